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

template <typename T>
__global__ void l2_final_kernel(int nblocks, int64_t n, const double *__restrict__ partials,
                                T *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0;
    for (int k = 0; k < nblocks; ++k) t += partials[k];
    *out = (T)(t / (double)n);
}

inline int loss_blocks() { return 148 * 8; }

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
