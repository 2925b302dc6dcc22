// Fused L2 loss of the fit loop: mean((clamp(img, 0, 1) - target)^2) over an
// [H, W, 3] render — the value of gaussianlig.py:95-102 (clamp, then
// loss_fn 'L2' = F.mse_loss, utils.py:17-21) in one pass over the two images
// (HBM-bound, 8 B per element) with deterministic two-level reduction.
// Its gradient is computed inside the rasterizer backward (lig_raster_bwd_l2).
#include "common.cuh"

namespace lig {

constexpr int kLossThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kLossThreads)
l2_partial_kernel(int64_t n, const T *__restrict__ img, const T *__restrict__ target,
                  double *__restrict__ partials) {
    __shared__ double s_warp[kLossThreads / 32];
    double acc = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const T x = img[i];
        const T d = min(max(x, (T)0), (T)1) - target[i];
        acc += (double)(d * d);
    }
    for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s_warp[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < kLossThreads / 32; ++k) t += s_warp[k];
        partials[blockIdx.x] = t;
    }
}

// Sum of partials[k0, k1) by one warp in a fixed order (lane-strided
// sums, then a butterfly): deterministic, and the same for the single-image
// and the batched reduction.
__device__ __forceinline__ double warp_sum_range(const double *__restrict__ partials, int k0,
                                                 int k1) {
    const int lane = threadIdx.x & 31;
    double t = 0;
    for (int k = k0 + lane; k < k1; k += 32) t += partials[k];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    return t;
}

template <typename T>
__global__ void l2_final_kernel(int nblocks, int64_t n, const double *__restrict__ partials,
                                T *__restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    const double t = warp_sum_range(partials, 0, nblocks);
    if (threadIdx.x == 0) *out = (T)(t / (double)n);
}

inline int loss_blocks() { return 148 * 8; }

// Batched: loss = sum over images of mean_i((clamp(img_i) - target_i)^2).
// Image i gets its own run of blocks (about its share of loss_blocks(), at
// least one), each striding over that image's values only, so a block's
// partial belongs to one image and the reduction stays deterministic.  For a
// batch of one this is exactly the single-image reduction above.
struct LossSplit {
    int n_img;
    int blk_off[kMaxBatch + 1];
    long long elem_off[kMaxBatch + 1];
};

template <typename T>
__global__ void __launch_bounds__(kLossThreads)
l2_partial_batch_kernel(const LossSplit sp, const T *__restrict__ img,
                        const T *__restrict__ target, double *__restrict__ partials) {
    __shared__ double s_warp[kLossThreads / 32];
    const int b = blockIdx.x;
    int lo = 0, hi = sp.n_img - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sp.blk_off[mid] <= b) lo = mid; else hi = mid - 1;
    }
    const int im = lo;
    const int lb = b - sp.blk_off[im], nb = sp.blk_off[im + 1] - sp.blk_off[im];
    const int64_t e0 = sp.elem_off[im], n = sp.elem_off[im + 1] - e0;
    double acc = 0;
    for (int64_t i = (int64_t)lb * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)nb * blockDim.x) {
        const T x = img[e0 + i];
        const T d = min(max(x, (T)0), (T)1) - target[e0 + i];
        acc += (double)(d * d);
    }
    for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s_warp[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < kLossThreads / 32; ++k) t += s_warp[k];
        partials[b] = t;
    }
}

// One block of 32 warps: warp w reduces images w, w + 32, ...; thread 0
// then adds the per-image means in image order.
template <typename T>
__global__ void __launch_bounds__(1024)
l2_final_batch_kernel(const LossSplit sp, const double *__restrict__ partials,
                      T *__restrict__ out, T *__restrict__ per_image) {
    __shared__ double s_mean[kMaxBatch];
    const int w = threadIdx.x >> 5;
    for (int im = w; im < sp.n_img; im += 32) {
        const double t = warp_sum_range(partials, sp.blk_off[im], sp.blk_off[im + 1]);
        if ((threadIdx.x & 31) == 0) {
            const double m = t / (double)(sp.elem_off[im + 1] - sp.elem_off[im]);
            s_mean[im] = m;
            if (per_image) per_image[im] = (T)m;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double total = 0;
        for (int im = 0; im < sp.n_img; ++im) total += s_mean[im];
        *out = (T)total;
    }
}

inline bool make_split(int n_img, const int32_t *h, const int32_t *w, LossSplit &sp) {
    if (n_img < 1 || n_img > kMaxBatch || !h || !w) return false;
    long long tot = 0;
    for (int i = 0; i < n_img; ++i) {
        if (h[i] <= 0 || w[i] <= 0) return false;
        tot += 3ll * h[i] * w[i];
    }
    sp.n_img = n_img;
    sp.blk_off[0] = 0;
    sp.elem_off[0] = 0;
    for (int i = 0; i < n_img; ++i) {
        const long long e = 3ll * h[i] * w[i];
        long long nb = n_img == 1 ? loss_blocks() : (long long)loss_blocks() * e / tot;
        if (nb < 1) nb = 1;
        sp.blk_off[i + 1] = sp.blk_off[i] + (int)nb;
        sp.elem_off[i + 1] = sp.elem_off[i] + e;
    }
    return true;
}

}  // namespace lig

using namespace lig;

extern "C" size_t lig_l2_workspace_bytes(void) { return sizeof(double) * (size_t)loss_blocks(); }

extern "C" int lig_l2_clamped_loss(int dtype, int64_t n, const void *img, const void *target,
                                   void *loss, void *ws, size_t ws_bytes, void *stream) {
    if (n <= 0 || !img || !target || !loss || !ws) return LIG_ERR_INVALID;
    if (ws_bytes < lig_l2_workspace_bytes()) return LIG_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = loss_blocks();
    double *part = (double *)ws;
    if (dtype == LIG_F32) {
        l2_partial_kernel<float><<<nb, kLossThreads, 0, s>>>(n, (const float *)img,
                                                             (const float *)target, part);
        l2_final_kernel<float><<<1, 32, 0, s>>>(nb, n, part, (float *)loss);
    } else if (dtype == LIG_F64) {
        l2_partial_kernel<double><<<nb, kLossThreads, 0, s>>>(n, (const double *)img,
                                                              (const double *)target, part);
        l2_final_kernel<double><<<1, 32, 0, s>>>(nb, n, part, (double *)loss);
    } else {
        return LIG_ERR_INVALID;
    }
    note_launches(2);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

extern "C" size_t lig_l2_batch_workspace_bytes(int n_img) {
    return sizeof(double) * (size_t)(loss_blocks() + (n_img > 0 ? n_img : 0));
}

extern "C" int lig_l2_clamped_loss_batch(int dtype, int n_img, const int32_t *heights,
                                         const int32_t *widths, const void *img,
                                         const void *target, void *loss, void *per_image,
                                         void *ws, size_t ws_bytes, void *stream) {
    LossSplit sp;
    if (!make_split(n_img, heights, widths, sp) || !img || !target || !loss || !ws)
        return LIG_ERR_INVALID;
    if (ws_bytes < sizeof(double) * (size_t)sp.blk_off[n_img]) return LIG_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = sp.blk_off[n_img];
    double *part = (double *)ws;
    if (dtype == LIG_F32) {
        l2_partial_batch_kernel<float><<<nb, kLossThreads, 0, s>>>(sp, (const float *)img,
                                                                   (const float *)target, part);
        l2_final_batch_kernel<float><<<1, 1024, 0, s>>>(sp, part, (float *)loss,
                                                        (float *)per_image);
    } else if (dtype == LIG_F64) {
        l2_partial_batch_kernel<double><<<nb, kLossThreads, 0, s>>>(sp, (const double *)img,
                                                                    (const double *)target, part);
        l2_final_batch_kernel<double><<<1, 1024, 0, s>>>(sp, part, (double *)loss,
                                                         (double *)per_image);
    } else {
        return LIG_ERR_INVALID;
    }
    note_launches(2);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}
