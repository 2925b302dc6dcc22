// Launchers for the reference's own CUDA kernels (TEST ORACLE ONLY).
//
// oracle/Makefile compiles this file together with the unmodified reference
// kernel sources (csrc/forward.cu, backward.cu, gradient_aware_rasterizer.cu,
// gradient_aware_upscaler.cu, read where they lie) into
// oracle/_ref/libgsplat2d_ref.so, with the reference's setup.py flags
// (-O3 --use_fast_math --expt-relaxed-constexpr).  Each launcher reproduces the
// allocation-and-launch step of one csrc/bindings.cu entry point without torch:
// outputs are zero-filled first (torch::zeros) and the kernel runs on the legacy
// default stream with the same grid/block shape.  The torch glue of
// gsplat2d/utils.py (cumsum, .item(), sort, gather) lives in oracle/ref.py.
#include <cstdint>
#include <cuda_runtime.h>

#include "backward.cuh"
#include "forward.cuh"
#include "helpers.cuh"
#include "upscale.cuh"

namespace {
constexpr int kThreads = N_THREADS;
inline int blocks_for(long n) { return (int)((n + kThreads - 1) / kThreads); }
inline dim3 tile_bounds(unsigned H, unsigned W, unsigned B) {
    return dim3((W + B - 1) / B, (H + B - 1) / B, 1);
}
}  // namespace

// Same per-element step as csrc/bindings.cu:19-39, calling the reference's
// own compute_cov2d_bounds device function.
__global__ void ref_cov2d_bounds_kernel(unsigned n, const float *covs, const float *opac,
                                        float *conics, float2 *extents) {
    unsigned row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    float3 conic = {0.f, 0.f, 0.f};
    float2 extent = {0.f, 0.f};
    float3 cov{covs[3 * row], covs[3 * row + 1], covs[3 * row + 2]};
    compute_cov2d_bounds(cov, opac ? opac[row] : 1.0f, conic, extent);
    conics[3 * row] = conic.x;
    conics[3 * row + 1] = conic.y;
    conics[3 * row + 2] = conic.z;
    extents[row] = extent;
}

extern "C" {

int ref_cov2d_bounds(int n, const float *cov, const float *opac, float *conics, float *extents) {
    cudaMemset(conics, 0, sizeof(float) * 3 * n);
    cudaMemset(extents, 0, sizeof(float) * 2 * n);
    ref_cov2d_bounds_kernel<<<blocks_for(n), kThreads>>>(n, cov, opac, conics, (float2 *)extents);
    return (int)cudaGetLastError();
}

// csrc/bindings.cu:73-117 (chol == 0) and :158-202 (chol == 1)
int ref_project_fwd(int n, int chol, const float *in3, const float *means, const float *opac,
                    int H, int W, int B, float *xys, float *extents, float *conics,
                    int32_t *counts) {
    cudaMemset(xys, 0, sizeof(float) * 2 * n);
    cudaMemset(extents, 0, sizeof(float) * 2 * n);
    cudaMemset(conics, 0, sizeof(float) * 3 * n);
    cudaMemset(counts, 0, sizeof(int32_t) * n);
    dim3 tb = tile_bounds(H, W, B);
    if (chol)
        project_gaussians_forward_kernel_cholesky<<<blocks_for(n), kThreads>>>(
            n, (const float3 *)in3, (const float2 *)means, opac, tb, B, (float2 *)xys,
            (float2 *)extents, (float3 *)conics, counts);
    else
        project_gaussians_forward_kernel<<<blocks_for(n), kThreads>>>(
            n, (const float3 *)in3, (const float2 *)means, opac, tb, B, (float2 *)xys,
            (float2 *)extents, (float3 *)conics, counts);
    return (int)cudaGetLastError();
}

// csrc/bindings.cu:122-151 (chol == 0) and :207-237 (chol == 1)
int ref_project_bwd(int n, int chol, const float *extents, const float *in3, const float *conics,
                    const float *v_xy, const float *v_conic, float *v_in3, float *v_mean) {
    cudaMemset(v_in3, 0, sizeof(float) * 3 * n);
    cudaMemset(v_mean, 0, sizeof(float) * 2 * n);
    if (chol)
        project_gaussians_backward_kernel_cholesky<<<blocks_for(n), kThreads>>>(
            n, (const float2 *)extents, (const float3 *)in3, (const float3 *)conics,
            (const float2 *)v_xy, (const float3 *)v_conic, (float3 *)v_in3, (float2 *)v_mean);
    else
        project_gaussians_backward_kernel<<<blocks_for(n), kThreads>>>(
            n, (const float2 *)extents, (const float3 *)conics, (const float2 *)v_xy,
            (const float3 *)v_conic, (float3 *)v_in3, (float2 *)v_mean);
    return (int)cudaGetLastError();
}

// csrc/bindings.cu:239-281
int ref_map_intersects(int n, int M, const float *xys, const float *depths, const float *extents,
                       const int32_t *cum, int tbx, int tby, int B, int64_t *isect_ids,
                       int32_t *gids) {
    cudaMemset(isect_ids, 0, sizeof(int64_t) * M);
    cudaMemset(gids, 0, sizeof(int32_t) * M);
    map_gaussian_to_intersects<<<blocks_for(n), kThreads>>>(
        n, (const float2 *)xys, depths, (const float2 *)extents, cum, dim3(tbx, tby, 1), B,
        isect_ids, gids);
    return (int)cudaGetLastError();
}

// csrc/bindings.cu:283-301
int ref_tile_bin_edges(int M, const int64_t *isect_sorted, int T, int32_t *bins) {
    cudaMemset(bins, 0, sizeof(int32_t) * 2 * T);
    if (M > 0) get_tile_bin_edges<<<blocks_for(M), kThreads>>>(M, isect_sorted, (int2 *)bins);
    return (int)cudaGetLastError();
}

// csrc/bindings.cu:304-401
int ref_raster_fwd(int H, int W, int B, const int32_t *gid_sorted, const int32_t *bins,
                   const float *xys, const float *conics, const float *colors, const float *opac,
                   int grad_aware, int32_t *final_idx, float *img, float *wsum, float *dx,
                   float *dy, float *dxy) {
    long P = (long)H * W;
    cudaMemset(final_idx, 0, sizeof(int32_t) * P);
    cudaMemset(img, 0, sizeof(float) * 3 * P);
    cudaMemset(wsum, 0, sizeof(float) * P);
    dim3 tb = tile_bounds(H, W, B), blk(B, B, 1), isz(W, H, 1);
    if (grad_aware) {
        cudaMemset(dx, 0, sizeof(float) * 3 * P);
        cudaMemset(dy, 0, sizeof(float) * 3 * P);
        cudaMemset(dxy, 0, sizeof(float) * 3 * P);
        gradient_aware_rasterize_forward<<<tb, blk>>>(
            tb, isz, gid_sorted, (const int2 *)bins, (const float2 *)xys, (const float3 *)conics,
            (const float3 *)colors, opac, final_idx, (float3 *)img, wsum, (float3 *)dx,
            (float3 *)dy, (float3 *)dxy);
    } else {
        rasterize_forward<<<tb, blk>>>(tb, isz, gid_sorted, (const int2 *)bins,
                                       (const float2 *)xys, (const float3 *)conics,
                                       (const float3 *)colors, opac, final_idx, (float3 *)img,
                                       wsum);
    }
    return (int)cudaGetLastError();
}

// csrc/bindings.cu:411-506 (v_dx == nullptr selects the sum kernel)
int ref_raster_bwd(int H, int W, int B, int N, const int32_t *gid_sorted, const int32_t *bins,
                   const float *xys, const float *conics, const float *colors, const float *opac,
                   const int32_t *final_idx, const float *v_out, const float *v_wsum,
                   const float *v_dx, const float *v_dy, const float *v_dxy, float *v_xy,
                   float *v_xy_abs, float *v_conic, float *v_rgb, float *v_opac) {
    cudaMemset(v_xy, 0, sizeof(float) * 2 * N);
    cudaMemset(v_xy_abs, 0, sizeof(float) * 2 * N);
    cudaMemset(v_conic, 0, sizeof(float) * 3 * N);
    cudaMemset(v_rgb, 0, sizeof(float) * 3 * N);
    if (v_opac) cudaMemset(v_opac, 0, sizeof(float) * N);
    dim3 tb = tile_bounds(H, W, B), blk(B, B, 1), isz(W, H, 1);
    if (v_dx)
        gradient_aware_rasterize_backward_kernel<<<tb, blk>>>(
            tb, isz, gid_sorted, (const int2 *)bins, (const float2 *)xys, (const float3 *)conics,
            (const float3 *)colors, opac, final_idx, (const float3 *)v_out, (const float3 *)v_dx,
            (const float3 *)v_dy, (const float3 *)v_dxy, v_wsum, (float2 *)v_xy,
            (float2 *)v_xy_abs, (float3 *)v_conic, (float3 *)v_rgb, v_opac);
    else
        rasterize_backward_kernel<<<tb, blk>>>(
            tb, isz, gid_sorted, (const int2 *)bins, (const float2 *)xys, (const float3 *)conics,
            (const float3 *)colors, opac, final_idx, (const float3 *)v_out, v_wsum,
            (float2 *)v_xy, (float2 *)v_xy_abs, (float3 *)v_conic, (float3 *)v_rgb, v_opac);
    return (int)cudaGetLastError();
}

// csrc/bindings.cu:508-559
int ref_upscale_fwd(int src_h, int src_w, int dst_h, int dst_w, float x1, float y1, float x2,
                    float y2, const float *f, const float *fx, const float *fy, const float *fxy,
                    float *out) {
    cudaMemset(out, 0, sizeof(float) * 3 * (long)dst_h * dst_w);
    dim3 blk(16, 16), grid((dst_w + 15) / 16, (dst_h + 15) / 16);
    gradient_aware_upscale_kernel<<<grid, blk>>>(dst_h, dst_w, src_h, src_w, x1, y1, x2, y2,
                                                 (const float3 *)f, (const float3 *)fx,
                                                 (const float3 *)fy, (const float3 *)fxy,
                                                 (float3 *)out);
    return (int)cudaGetLastError();
}

// csrc/bindings.cu:561-605
int ref_upscale_bwd(int src_h, int src_w, int dst_h, int dst_w, float x1, float y1, float x2,
                    float y2, const float *g, float *gf, float *gfx, float *gfy, float *gfxy) {
    long ns = 3L * src_h * src_w;
    cudaMemset(gf, 0, sizeof(float) * ns);
    cudaMemset(gfx, 0, sizeof(float) * ns);
    cudaMemset(gfy, 0, sizeof(float) * ns);
    cudaMemset(gfxy, 0, sizeof(float) * ns);
    dim3 blk(16, 16), grid((dst_w + 15) / 16, (dst_h + 15) / 16);
    gradient_aware_upscale_backward_kernel<<<grid, blk>>>(
        dst_h, dst_w, src_h, src_w, x1, y1, x2, y2, (const float3 *)g, (float3 *)gf,
        (float3 *)gfx, (float3 *)gfy, (float3 *)gfxy);
    return (int)cudaGetLastError();
}

}  // extern "C"
