// Fused Adam over one flat parameter buffer, guarded by the binning status.
//
// The fit loops keep every Gaussian parameter of a level (or of a batch of
// levels) in one flat fp32 buffer — means [N,2] | cholesky [N,3] | rgb [N,3] —
// with the gradient buffer laid out the same way, so one elementwise kernel
// updates them all (the optimiser of gaussianlig.py:64-68, Adam on every
// parameter, here without per-tensor launches).
//
// Guard: when the binning of this step overflowed its intersection capacity
// (status word has LIG_STATUS_OVERFLOW), the gradients are those of truncated
// tile lists.  The prologue then marks the step skipped — no moment update,
// no step increment, parameters untouched — and counts it, so a caller that
// captured the step in a CUDA graph with a fixed capacity can grow the
// capacity and redo exactly the skipped steps.
//
// Update rule: Adam (Kingma & Ba, "Adam: A Method for Stochastic
// Optimization", Algorithm 1) with the bias corrections folded as
// p -= (lr / (1 - b1^t)) * m / (sqrt(v) / sqrt(1 - b2^t) + eps), the form of
// torch.optim.Adam's update (which the fit loops used before).
#include "common.cuh"

namespace lig {

struct AdamScalars {
    float step_size;     // lr / (1 - b1^t)
    float bc2_sqrt;      // sqrt(1 - b2^t)
    int skip;            // 1: leave everything unchanged
    int pad;
};

// One element, in the form torch.optim.Adam evaluates it: m = lerp(m, g,
// 1 - b1), v = v b2 + (1 - b2) g g, p -= step_size * m / (sqrt(v) / bc2 +
// eps), with correctly rounded square root and divisions.
// c1 = 1 - b1 and c2 = 1 - b2 are formed in double on the host and rounded
// once, as torch does with its Python-float coefficients.
__device__ __forceinline__ void adam_update(float &p, float g, float &m, float &v, float c1,
                                            float b2, float c2, float eps,
                                            const AdamScalars &a) {
    m = __fadd_rn(m, __fmul_rn(c1, __fsub_rn(g, m)));
    v = __fadd_rn(__fmul_rn(v, b2), __fmul_rn(__fmul_rn(c2, g), g));
    const float den = __fadd_rn(__fdiv_rn(__fsqrt_rn(v), a.bc2_sqrt), eps);
    p = __fsub_rn(p, __fmul_rn(a.step_size, __fdiv_rn(m, den)));
}

__global__ void adam_prologue_kernel(const int32_t *__restrict__ status, int32_t *step,
                                     int32_t *skipped, double lr, double b1, double b2,
                                     AdamScalars *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    AdamScalars a{0.f, 1.f, 0, 0};
    if (status && (*status & LIG_STATUS_OVERFLOW)) {
        a.skip = 1;
        if (skipped) *skipped += 1;
    } else {
        const int t = *step + 1;
        *step = t;
        a.step_size = (float)(lr / (1.0 - pow(b1, (double)t)));
        a.bc2_sqrt = (float)sqrt(1.0 - pow(b2, (double)t));
    }
    *out = a;
}

__global__ void __launch_bounds__(256)
adam_kernel(int64_t n, float *__restrict__ p, const float *__restrict__ g,
            float *__restrict__ m, float *__restrict__ v, float c1, float b2, float c2,
            float eps, const AdamScalars *__restrict__ sc) {
    const AdamScalars a = *sc;
    if (a.skip) return;
    const int64_t n4 = n / 4;
    float4 *p4 = reinterpret_cast<float4 *>(p);
    const float4 *g4 = reinterpret_cast<const float4 *>(g);
    float4 *m4 = reinterpret_cast<float4 *>(m);
    float4 *v4 = reinterpret_cast<float4 *>(v);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 pp = p4[i], gg = g4[i], mm = m4[i], vv = v4[i];
        float *pe = &pp.x, *ge = &gg.x, *me = &mm.x, *ve = &vv.x;
#pragma unroll
        for (int k = 0; k < 4; ++k) adam_update(pe[k], ge[k], me[k], ve[k], c1, b2, c2, eps, a);
        p4[i] = pp; m4[i] = mm; v4[i] = vv;
    }
    for (int64_t i = n4 * 4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride) {
        float pi = p[i], mi = m[i], vi = v[i];
        adam_update(pi, g[i], mi, vi, c1, b2, c2, eps, a);
        p[i] = pi; m[i] = mi; v[i] = vi;
    }
}

// ---------------------------------------------------------------- batched
// A batch of fits in one flat buffer laid out [means 2N | cholesky 3N |
// rgb 3N] (N = total Gaussians, image i owning Gaussians [g_off[i],
// g_off[i+1])).  Every image keeps its own step count, so a fit that joins
// or leaves a running batch follows exactly the updates it would get alone.
struct AdamBatch {
    int n_img, n_pts;
    int g_off[kMaxBatch + 1];
};

__global__ void adam_batch_prologue_kernel(AdamBatch ab, const int32_t *__restrict__ status,
                                           int32_t *steps, int32_t *skipped, double lr,
                                           double b1, double b2, AdamScalars *out) {
    const int i = threadIdx.x;
    const bool skip = status && (*status & LIG_STATUS_OVERFLOW);
    if (i == 0 && skip && skipped) *skipped += 1;
    if (i >= ab.n_img) return;
    AdamScalars a{0.f, 1.f, skip ? 1 : 0, 0};
    if (!skip) {
        const int t = steps[i] + 1;
        steps[i] = t;
        a.step_size = (float)(lr / (1.0 - pow(b1, (double)t)));
        a.bc2_sqrt = (float)sqrt(1.0 - pow(b2, (double)t));
    }
    out[i] = a;
}

__device__ __forceinline__ int elem_image(const AdamBatch &ab, int64_t e) {
    const int64_t n = ab.n_pts;
    const int g = (int)(e < 2 * n ? e / 2 : (e < 5 * n ? (e - 2 * n) / 3 : (e - 5 * n) / 3));
    return BatchGeo::find(ab.g_off, ab.n_img, g);
}

__global__ void __launch_bounds__(256)
adam_batch_kernel(AdamBatch ab, float *__restrict__ p, const float *__restrict__ g,
                  float *__restrict__ m, float *__restrict__ v, float c1, float b2, float c2,
                  float eps, const AdamScalars *__restrict__ sc) {
    if (sc[0].skip) return;
    const int64_t n = 8ll * ab.n_pts;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const AdamScalars a = sc[elem_image(ab, i)];
        float pi = p[i], mi = m[i], vi = v[i];
        adam_update(pi, g[i], mi, vi, c1, b2, c2, eps, a);
        p[i] = pi; m[i] = mi; v[i] = vi;
    }
}

}  // namespace lig

using namespace lig;

extern "C" size_t lig_adam_batch_scratch_bytes(int n_img) {
    return sizeof(AdamScalars) * (size_t)(n_img > 0 ? n_img : 1);
}

extern "C" int lig_adam_step_batch(int n_img, const int32_t *counts, float *params,
                                   const float *grads, float *exp_avg, float *exp_avg_sq,
                                   double lr, double beta1, double beta2, double eps,
                                   const int32_t *status, int32_t *steps, int32_t *skipped,
                                   void *scratch, size_t scratch_bytes, void *stream) {
    if (n_img < 1 || n_img > kMaxBatch || !counts || !steps || !scratch) return LIG_ERR_INVALID;
    if (scratch_bytes < lig_adam_batch_scratch_bytes(n_img)) return LIG_ERR_WORKSPACE;
    AdamBatch ab;
    ab.n_img = n_img;
    ab.g_off[0] = 0;
    long long tot = 0;
    for (int i = 0; i < n_img; ++i) {
        if (counts[i] < 0) return LIG_ERR_INVALID;
        tot += counts[i];
        if (8 * tot > 0x7fffffffffffll) return LIG_ERR_INVALID;
        if (tot > 0x7fffffffll) return LIG_ERR_INVALID;
        ab.g_off[i + 1] = (int)tot;
    }
    ab.n_pts = (int)tot;
    if (tot > 0 && (!params || !grads || !exp_avg || !exp_avg_sq)) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    AdamScalars *sc = (AdamScalars *)scratch;
    adam_batch_prologue_kernel<<<1, kMaxBatch, 0, s>>>(ab, status, steps, skipped, lr, beta1,
                                                       beta2, sc);
    int launches = 1;
    if (tot > 0 && n_img == 1 && !((uintptr_t)params & 15) && !((uintptr_t)grads & 15) &&
        !((uintptr_t)exp_avg & 15) && !((uintptr_t)exp_avg_sq & 15)) {
        // one image: the float4 kernel with the image's scalars
        int64_t blocks = (2 * tot + 255) / 256;
        const int64_t cap = 148 * 16;
        if (blocks > cap) blocks = cap;
        adam_kernel<<<(int)blocks, 256, 0, s>>>(8 * tot, params, grads, exp_avg, exp_avg_sq,
                                               (float)(1.0 - beta1), (float)beta2,
                                               (float)(1.0 - beta2), (float)eps, sc);
        ++launches;
    } else if (tot > 0) {
        int64_t blocks = (8 * tot + 255) / 256;
        const int64_t cap = 148 * 16;
        if (blocks > cap) blocks = cap;
        adam_batch_kernel<<<(int)blocks, 256, 0, s>>>(ab, params, grads, exp_avg, exp_avg_sq,
                                                     (float)(1.0 - beta1), (float)beta2,
                                                     (float)(1.0 - beta2), (float)eps, sc);
        ++launches;
    }
    note_launches(launches);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

extern "C" size_t lig_adam_scratch_bytes(void) { return sizeof(AdamScalars); }

extern "C" int lig_adam_step(int64_t n, float *params, const float *grads, float *exp_avg,
                             float *exp_avg_sq, double lr, double beta1, double beta2,
                             double eps, const int32_t *status, int32_t *step, int32_t *skipped,
                             void *scratch, void *stream) {
    if (n < 0 || !step || !scratch || (n > 0 && (!params || !grads || !exp_avg || !exp_avg_sq)))
        return LIG_ERR_INVALID;
    // float4 path needs 16-byte aligned buffers
    const uintptr_t al = (uintptr_t)params | (uintptr_t)grads | (uintptr_t)exp_avg |
                         (uintptr_t)exp_avg_sq;
    if (al & 15) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    AdamScalars *sc = (AdamScalars *)scratch;
    adam_prologue_kernel<<<1, 32, 0, s>>>(status, step, skipped, lr, beta1, beta2, sc);
    int launches = 1;
    if (n > 0) {
        int64_t blocks = (n / 4 + 255) / 256;
        const int64_t cap = 148 * 16;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) blocks = 1;
        adam_kernel<<<(int)blocks, 256, 0, s>>>(n, params, grads, exp_avg, exp_avg_sq,
                                               (float)(1.0 - beta1), (float)beta2,
                                               (float)(1.0 - beta2), (float)eps, sc);
        ++launches;
    }
    note_launches(launches);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}
