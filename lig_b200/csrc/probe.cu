// FP32 throughput probe: the roofline denominator for the SIMT-bound
// rasterizer kernels, measured on the device at run time (the pool publishes
// HBM and tensor-core peaks only).  Each thread runs 8 independent FMA chains;
// 2 FLOP per FMA.
#include "common.cuh"

namespace lig {

__global__ void __launch_bounds__(256) fma_probe_kernel(int iters, float seed, float *out) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + (float)(threadIdx.x + k);
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace lig

// FLOPs issued = blocks * 256 threads * iters * 8 FMA * 2.
extern "C" int lig_probe_fp32(int blocks, int iters, float *out, void *stream) {
    if (blocks <= 0 || iters <= 0 || !out) return LIG_ERR_INVALID;
    lig::fma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 1.0f, out);
    lig::note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}
