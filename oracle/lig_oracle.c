/*
 * lig_oracle — CPU restatement of LIG's gsplat2d hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels in lig_b200/csrc
 * and the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library; the
 * product path (lig_b200) never does.
 *
 * Parity pinning: the float restatement is checked against golden vectors
 * produced by the reference's own CUDA kernels (compiled from the reference
 * sources into oracle/_ref by oracle/Makefile and run by
 * tests/golden/make_golden_ref.py) and against the reference's pure-torch
 * upscaler (tests/golden/make_golden_torch.py).
 *
 * The float/double bodies live in oracle_impl.inc; this file holds the
 * integer parts (scan, stable tile sort, tile ranges) and the FP64 dense
 * evaluator.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* float -> int32 conversion with the GPU's cvt.rzi.s32 semantics: truncate
 * toward zero, saturate to the int32 range, NaN -> 0.  The reference relies on
 * this in its tile bbox (csrc/helpers.cuh:39-42). */
static int32_t gpu_f2i(double v)
{
    if (v != v) return 0;
    if (v >= 2147483647.0) return INT32_MAX;
    if (v <= -2147483648.0) return INT32_MIN;
    return (int32_t)v;
}

/* min(max(0, v), bound) with the unsigned bound of csrc/helpers.cuh:39-42. */
static int32_t clamp_tile(int32_t v, int bound)
{
    if (v < 0) v = 0;
    if (v > bound) v = bound;
    return v;
}

#define R float
#define SFX f32
#define RLOG logf
#define RSQRT sqrtf
#define RCEIL ceilf
#define RFLOOR floorf
#define REXP expf
#define RMIN fminf
#define RABS fabsf
#include "oracle_impl.inc"
#undef R
#undef SFX
#undef RLOG
#undef RSQRT
#undef RCEIL
#undef RFLOOR
#undef REXP
#undef RMIN
#undef RABS

#define R double
#define SFX f64
#define RLOG log
#define RSQRT sqrt
#define RCEIL ceil
#define RFLOOR floor
#define REXP exp
#define RMIN fmin
#define RABS fabs
#include "oracle_impl.inc"

/* torch.cumsum(num_tiles_hit, dtype=int32), gsplat2d/gsplat2d/utils.py:65. */
void orc_cumsum_i32(int n, const int32_t *in, int32_t *out)
{
    int32_t acc = 0;
    for (int i = 0; i < n; ++i) { acc += in[i]; out[i] = acc; }
}

/*
 * Stable sort of intersections by key, gsplat2d/gsplat2d/utils.py:97-98
 * (torch.sort + gather).  Keys are (tile << 32) | depth-bits with depth 0, so
 * a stable counting sort on the tile gives the stable 64-bit order.  Returns
 * -1 if a key carries non-zero low bits or a tile >= T.
 */
int orc_sort_by_tile(int M, const int64_t *isect_ids, const int32_t *gids, int T,
                     int64_t *isect_sorted, int32_t *gid_sorted)
{
    int64_t *start = (int64_t *)calloc((size_t)T + 1, sizeof(int64_t));
    if (!start) return -2;
    for (int k = 0; k < M; ++k) {
        int64_t key = isect_ids[k];
        int64_t t = key >> 32;
        if ((key & 0xffffffffLL) != 0 || t < 0 || t >= T) { free(start); return -1; }
        start[t + 1]++;
    }
    for (int t = 0; t < T; ++t) start[t + 1] += start[t];
    for (int k = 0; k < M; ++k) {
        int64_t t = isect_ids[k] >> 32;
        int64_t pos = start[t]++;
        isect_sorted[pos] = isect_ids[k];
        gid_sorted[pos] = gids[k];
    }
    free(start);
    return 0;
}

/* Tile ranges from sorted keys, csrc/forward.cu:148-170; empty tiles (0,0). */
void orc_tile_bins(int M, const int64_t *isect_sorted, int T, int32_t *bins)
{
    memset(bins, 0, sizeof(int32_t) * 2 * (size_t)T);
    for (int k = 0; k < M; ++k) {
        int32_t cur = (int32_t)(isect_sorted[k] >> 32);
        if (k == 0) bins[2 * cur] = 0;
        if (k == M - 1) bins[2 * cur + 1] = M;
        if (k == 0) continue;
        int32_t prev = (int32_t)(isect_sorted[k - 1] >> 32);
        if (prev != cur) { bins[2 * prev + 1] = k; bins[2 * cur] = k; }
    }
}

/*
 * FP64 dense evaluator: every pixel against every Gaussian in ascending id,
 * with the reference's culling applied exactly (the pixel's tile inside the
 * Gaussian's tile bbox as in csrc/forward.cu:123-142, sigma < 0, alpha < 1/255,
 * alpha = min(0.999, o exp(-sigma)) as in csrc/forward.cu:249-270).  Gaussians
 * with extent <= 0 but a non-zero tile count contribute `counts[g]` zero-id
 * entries to tile 0 (the zero-initialised slots of csrc/bindings.cu:260-263),
 * which the evaluator reproduces as extra evaluations of Gaussian 0 in tile 0.
 * grad_aware selects the derivative outputs of
 * csrc/gradient_aware_rasterizer.cu:436-480.
 */
void orc_dense_fwd_f64(int H, int W, int B, int N, const double *xys, const double *extents,
                       const int32_t *counts, const double *conics, const double *colors,
                       const double *opac, int grad_aware, double *img, double *wsum,
                       double *odx, double *ody, double *odxy)
{
    int tbx = (W + B - 1) / B, tby = (H + B - 1) / B;
    int32_t *bb = (int32_t *)malloc(sizeof(int32_t) * 4 * (size_t)(N > 0 ? N : 1));
    int64_t phantom = 0;
    for (int g = 0; g < N; ++g) {
        bb[4 * g] = bb[4 * g + 1] = bb[4 * g + 2] = bb[4 * g + 3] = 0;
        if (extents[2 * g] <= 0 || extents[2 * g + 1] <= 0) {
            phantom += counts[g];
            continue;
        }
        int32_t tmin[2], tmax[2];
        tile_bbox_f64(xys[2 * g], xys[2 * g + 1], extents[2 * g], extents[2 * g + 1],
                      tbx, tby, B, tmin, tmax);
        bb[4 * g] = tmin[0]; bb[4 * g + 1] = tmin[1]; bb[4 * g + 2] = tmax[0]; bb[4 * g + 3] = tmax[1];
    }
    #pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < H; ++i) {
        for (int j = 0; j < W; ++j) {
            int tx = j / B, ty = i / B;
            double px = j + 0.5, py = i + 0.5;
            double out[3] = {0, 0, 0}, ax3[3] = {0, 0, 0}, ay3[3] = {0, 0, 0}, axy3[3] = {0, 0, 0};
            double ws = 0;
            for (int g = -1; g < N; ++g) {
                int gg = g;
                int64_t reps = 1;
                if (g < 0) {
                    if (!(tx == 0 && ty == 0) || phantom == 0 || N == 0) continue;
                    gg = 0;
                    reps = phantom;
                } else if (!(tx >= bb[4 * g] && tx < bb[4 * g + 2] && ty >= bb[4 * g + 1] && ty < bb[4 * g + 3])) {
                    continue;
                }
                double a = conics[3 * gg], b = conics[3 * gg + 1], c = conics[3 * gg + 2];
                double dx = px - xys[2 * gg], dy = py - xys[2 * gg + 1];
                double sigma = 0.5 * (a * dx * dx + c * dy * dy) + b * dx * dy;
                double o = opac ? opac[gg] : 1.0;
                double alpha = fmin(0.999, o * exp(-sigma));
                if (sigma < 0 || alpha < 1.0 / 255.0) continue;
                for (int64_t r = 0; r < reps; ++r) {
                    for (int ch = 0; ch < 3; ++ch) out[ch] += colors[3 * gg + ch] * alpha;
                    ws += alpha;
                    if (grad_aware) {
                        double sx = a * dx + b * dy, sy = b * dx + c * dy;
                        for (int ch = 0; ch < 3; ++ch) {
                            ax3[ch] += colors[3 * gg + ch] * (-alpha * sx);
                            ay3[ch] += colors[3 * gg + ch] * (-alpha * sy);
                            axy3[ch] += colors[3 * gg + ch] * (-alpha * (b - sx * sy));
                        }
                    }
                }
            }
            int64_t p = (int64_t)i * W + j;
            for (int ch = 0; ch < 3; ++ch) img[3 * p + ch] = out[ch];
            wsum[p] = ws;
            if (grad_aware)
                for (int ch = 0; ch < 3; ++ch) {
                    odx[3 * p + ch] = ax3[ch];
                    ody[3 * p + ch] = ay3[ch];
                    odxy[3 * p + ch] = axy3[ch];
                }
        }
    }
    free(bb);
}
