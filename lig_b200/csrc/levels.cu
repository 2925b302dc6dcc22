// LIG level pipeline ops: the residual target between levels and the
// multi-level compose of a decode.
//
// Residual (train.py:113-126): resid = gt - up + 0.5, min-max normalised to
// [0, 1]; the level's store_min / store_max are the min and max.  Two passes
// over gt and up (the min/max reduction, then the normalised write) instead
// of six elementwise / reduction launches; every value is computed with the
// same IEEE operations in the same order as the torch expression
// ((gt - up) + 0.5, then (r - lo) / (hi - lo) with a correctly rounded
// division), so the result is bit-identical.
//
// Compose (train.py:188-200): for level s > 0 the running image is resized
// to the level's size with bilinear half-pixel sampling (F.interpolate mode
// 'bilinear', align_corners=False: src = max((dst + 0.5) * in/out - 0.5, 0),
// right/bottom neighbour clamped) and the de-normalised level render
// clamp(render, 0, 1) * (hi - lo) - 0.5 + lo is added; the last level is
// clamped to [0, 1].  One pass per level, no intermediate resized image.
#include <cfloat>

#include "common.cuh"

namespace lig {

constexpr int kLevelThreads = 256;

__device__ __forceinline__ float atomic_min_f(float *a, float v) {
    // order-preserving int mapping of finite floats
    int *ai = reinterpret_cast<int *>(a);
    int old = *ai;
    while (__int_as_float(old) > v) {
        const int prev = atomicCAS(ai, old, __float_as_int(v));
        if (prev == old) break;
        old = prev;
    }
    return __int_as_float(old);
}

__device__ __forceinline__ float atomic_max_f(float *a, float v) {
    int *ai = reinterpret_cast<int *>(a);
    int old = *ai;
    while (__int_as_float(old) < v) {
        const int prev = atomicCAS(ai, old, __float_as_int(v));
        if (prev == old) break;
        old = prev;
    }
    return __int_as_float(old);
}

__global__ void minmax_init_kernel(float *mm) {
    mm[0] = FLT_MAX;
    mm[1] = -FLT_MAX;
}

// pass 1: min / max of gt - up + 0.5 (NaNs are ignored by the comparisons)
__global__ void __launch_bounds__(kLevelThreads)
resid_minmax_kernel(int64_t n, const float *__restrict__ gt, const float *__restrict__ up,
                    float *__restrict__ mm) {
    float lo = FLT_MAX, hi = -FLT_MAX;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float r = __fadd_rn(__fsub_rn(gt[i], up[i]), 0.5f);
        lo = fminf(lo, r);
        hi = fmaxf(hi, r);
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __shared__ float s_lo[kLevelThreads / 32], s_hi[kLevelThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { s_lo[w] = lo; s_hi[w] = hi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kLevelThreads / 32; ++k) { lo = fminf(lo, s_lo[k]); hi = fmaxf(hi, s_hi[k]); }
        lo = fminf(lo, s_lo[0]);
        hi = fmaxf(hi, s_hi[0]);
        atomic_min_f(mm, lo);
        atomic_max_f(mm + 1, hi);
    }
}

// pass 2: (r - lo) / (hi - lo), correctly rounded
__global__ void __launch_bounds__(kLevelThreads)
resid_normalise_kernel(int64_t n, const float *__restrict__ gt, const float *__restrict__ up,
                       const float *__restrict__ mm, float *__restrict__ out) {
    const float lo = mm[0], hi = mm[1];
    const float den = __fsub_rn(hi, lo);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float r = __fadd_rn(__fsub_rn(gt[i], up[i]), 0.5f);
        out[i] = __fdiv_rn(__fsub_rn(r, lo), den);
    }
}

// Compose one level: out = base + (clamp(render) * (hi - lo) - 0.5 + lo),
// base = bilinear resize of prev [ph, pw, 3] to [H, W] (or prev itself when
// the sizes agree), clamp_out: final clamp to [0, 1].
__global__ void __launch_bounds__(kLevelThreads)
compose_kernel(int ph, int pw, const float *__restrict__ prev, int H, int W,
               const float *__restrict__ render, const float *__restrict__ mm, float lo_h,
               float hi_h, int clamp_render, int clamp_out, float *__restrict__ out) {
    const int64_t np = (int64_t)H * W;
    const float lo = mm ? mm[0] : lo_h, hi = mm ? mm[1] : hi_h;
    const float rng = __fsub_rn(hi, lo);
    const bool same = ph == H && pw == W;
    const float sh = __fdiv_rn((float)ph, (float)H), sw = __fdiv_rn((float)pw, (float)W);
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(p / W), x = (int)(p - (int64_t)y * W);
        float base[3];
        if (same || !prev) {
#pragma unroll
            for (int c = 0; c < 3; ++c) base[c] = prev ? prev[3 * p + c] : 0.f;
        } else {
            // the half-pixel source index and weights written as the bilinear
            // definition states them (src = s (d + 0.5) - 0.5, negative -> 0;
            // lambda1 = src - floor, lambda0 = 1 - lambda1), so that the
            // compiler contracts them as it does torch's upsample kernel
            float ry = sh * ((float)y + 0.5f) - 0.5f;
            float rx = sw * ((float)x + 0.5f) - 0.5f;
            ry = ry < 0.f ? 0.f : ry;
            rx = rx < 0.f ? 0.f : rx;
            const int y0 = (int)ry, x0 = (int)rx;
            const int y1 = y0 + (y0 < ph - 1 ? 1 : 0), x1 = x0 + (x0 < pw - 1 ? 1 : 0);
            const float ly1 = ry - (float)y0, lx1 = rx - (float)x0;
            const float ly0 = 1.f - ly1, lx0 = 1.f - lx1;
            const float *r0 = prev + 3 * ((int64_t)y0 * pw), *r1 = prev + 3 * ((int64_t)y1 * pw);
#pragma unroll
            for (int c = 0; c < 3; ++c)
                base[c] = ly0 * (lx0 * r0[3 * x0 + c] + lx1 * r0[3 * x1 + c]) +
                          ly1 * (lx0 * r1[3 * x0 + c] + lx1 * r1[3 * x1 + c]);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float r = render[3 * p + c];
            if (clamp_render) r = fminf(fmaxf(r, 0.f), 1.f);
            const float est = __fadd_rn(__fsub_rn(__fmul_rn(r, rng), 0.5f), lo);
            float v = __fadd_rn(base[c], est);
            if (clamp_out) v = fminf(fmaxf(v, 0.f), 1.f);
            out[3 * p + c] = v;
        }
    }
}

inline int level_blocks(int64_t n) {
    int64_t b = (n + kLevelThreads - 1) / kLevelThreads;
    const int64_t cap = 148 * 16;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace lig

using namespace lig;

extern "C" int lig_level_residual(int64_t n, const float *gt, const float *up, float *out,
                                  float *minmax, void *stream) {
    if (n <= 0 || !gt || !up || !out || !minmax) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    minmax_init_kernel<<<1, 1, 0, s>>>(minmax);
    resid_minmax_kernel<<<level_blocks(n), kLevelThreads, 0, s>>>(n, gt, up, minmax);
    resid_normalise_kernel<<<level_blocks(n), kLevelThreads, 0, s>>>(n, gt, up, minmax, out);
    note_launches(3);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

extern "C" int lig_level_compose(int prev_h, int prev_w, const float *prev, int H, int W,
                                 const float *render, const float *minmax, double store_min,
                                 double store_max, int clamp_render, int clamp_out, float *out,
                                 void *stream) {
    if (H <= 0 || W <= 0 || !render || !out || (prev && (prev_h <= 0 || prev_w <= 0)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t np = (int64_t)H * W;
    compose_kernel<<<level_blocks(np), kLevelThreads, 0, s>>>(
        prev_h, prev_w, prev, H, W, render, minmax, (float)store_min, (float)store_max,
        clamp_render, clamp_out, out);
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}
