// Shared device helpers for the lig_b200 kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/lig_b200.h"

namespace lig {

constexpr int kWarp = 32;

// Precision-dependent math.  The float versions are the ones the reference
// gets from its --use_fast_math build (csrc/helpers.cuh, csrc/forward.cu:257):
// logf/sqrtf/division compile to the fast approximations under the same flag,
// and the exponential is the __expf intrinsic called by name.  The double
// versions are the IEEE functions, used by the FP64 checking path.
template <typename T> struct Math;
template <> struct Math<float> {
    static __device__ __forceinline__ float exp_(float x) { return __expf(x); }
    static __device__ __forceinline__ float log_(float x) { return logf(x); }
    static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float ceil_(float x) { return ceilf(x); }
    static __device__ __forceinline__ float floor_(float x) { return floorf(x); }
    static __device__ __forceinline__ float min_(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float abs_(float a) { return fabsf(a); }
    static __device__ __forceinline__ bool finite_(float a) { return isfinite(a); }
};
template <> struct Math<double> {
    static __device__ __forceinline__ double exp_(double x) { return exp(x); }
    static __device__ __forceinline__ double log_(double x) { return log(x); }
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double ceil_(double x) { return ceil(x); }
    static __device__ __forceinline__ double floor_(double x) { return floor(x); }
    static __device__ __forceinline__ double min_(double a, double b) { return fmin(a, b); }
    static __device__ __forceinline__ double abs_(double a) { return fabs(a); }
    static __device__ __forceinline__ bool finite_(double a) { return isfinite(a); }
};

// float/double -> int32, truncating toward zero, saturating, NaN -> 0 (the
// semantics of the (int) casts in the reference's tile bbox).
__device__ __forceinline__ int to_int_rz(float v) { return (int)v; }
__device__ __forceinline__ int to_int_rz(double v) { return (int)v; }

// Tile-space bbox of a Gaussian (inclusive min, exclusive max), following the
// reference's get_bbox/get_tile_bbox (csrc/helpers.cuh:29-62) operation for
// operation, so that the float results carry the same roundings.  `block` is
// a runtime value on purpose: the reference divides by a runtime block width.
template <typename T>
__device__ __forceinline__ void tile_bbox(T cx, T cy, T ex, T ey, unsigned tbx, unsigned tby,
                                          unsigned block, int &x0, int &y0, int &x1, int &y1) {
    T tcx = cx / (T)block, tcy = cy / (T)block;
    T tex = ex / (T)block, tey = ey / (T)block;
    x0 = (int)min((unsigned)max(0, to_int_rz(tcx - tex)), tbx);
    x1 = (int)min((unsigned)max(0, to_int_rz(tcx + tex + 1)), tbx);
    y0 = (int)min((unsigned)max(0, to_int_rz(tcy - tey)), tby);
    y1 = (int)min((unsigned)max(0, to_int_rz(tcy + tey + 1)), tby);
}

// Conic + SnugBox extent (csrc/helpers.cuh:64-98): same expressions in the same
// order.  Returns false when det == 0 (conic/extent untouched).
template <typename T>
__device__ __forceinline__ bool cov2d_bounds(T cx, T cy, T cz, T opacity, T &ca, T &cb, T &cc,
                                             T &ex, T &ey) {
    using M = Math<T>;
    T det = cx * cz - cy * cy;
    if (det == (T)0) return false;
    T inv_det = (T)1 / det;
    T a = cz * inv_det;
    T b = -cy * inv_det;
    T c = cx * inv_det;
    ca = a; cb = b; cc = c;
    T t = (T)2 * M::log_((T)255 * opacity);
    if (t <= (T)0) {
        ex = 0; ey = 0;
        return true;
    }
    ex = M::ceil_(M::sqrt_(t * c / inv_det));
    ey = M::ceil_(M::sqrt_(t * a / inv_det));
    return true;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31; }

// Geometry of a batch of images rasterised in one launch, passed by value as a
// kernel parameter (constant bank; ~1.6 KB).  Image i owns Gaussians
// [g_off[i], g_off[i+1]), tiles [tile_off[i], tile_off[i+1]) of the flattened
// tile list and pixels [pix_off[i], pix_off[i+1]) of the concatenated HWC
// buffers.  A single image is the batch {n_img = 1}.
constexpr int kMaxBatch = LIG_MAX_BATCH;
struct BatchGeo {
    int n_img, B;
    int tile_off[kMaxBatch + 1], g_off[kMaxBatch + 1], pix_off[kMaxBatch + 1];
    int H[kMaxBatch], W[kMaxBatch], tbx[kMaxBatch];

    // index i with off[i] <= x < off[i+1] (off non-decreasing, x < off[n])
    __host__ __device__ __forceinline__ static int find(const int *off, int n, int x) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (off[mid] <= x) lo = mid; else hi = mid - 1;
        }
        return lo;
    }
    __host__ __device__ __forceinline__ int image_of_tile(int t) const {
        return n_img == 1 ? 0 : find(tile_off, n_img, t);
    }
    __host__ __device__ __forceinline__ int image_of_gauss(int g) const {
        return n_img == 1 ? 0 : find(g_off, n_img, g);
    }
    __host__ __device__ __forceinline__ int image_of_pixel(int p) const {
        return n_img == 1 ? 0 : find(pix_off, n_img, p);
    }
    __host__ __device__ __forceinline__ int tby(int i) const { return (H[i] + B - 1) / B; }
    __host__ __device__ int total_tiles() const { return tile_off[n_img]; }
    __host__ __device__ int total_pixels() const { return pix_off[n_img]; }
    __host__ __device__ int total_points() const { return g_off[n_img]; }

    // host-side construction; false on bad sizes
    static bool make(int n_img, const int32_t *h, const int32_t *w, const int32_t *n_pts, int B,
                     BatchGeo &g) {
        if (n_img < 1 || n_img > kMaxBatch || B < 1) return false;
        g.n_img = n_img;
        g.B = B;
        long long t = 0, gp = 0, px = 0;
        g.tile_off[0] = g.g_off[0] = g.pix_off[0] = 0;
        for (int i = 0; i < n_img; ++i) {
            if (h[i] <= 0 || w[i] <= 0 || n_pts[i] < 0) return false;
            g.H[i] = h[i];
            g.W[i] = w[i];
            g.tbx[i] = (w[i] + B - 1) / B;
            t += (long long)g.tbx[i] * ((h[i] + B - 1) / B);
            gp += n_pts[i];
            px += (long long)h[i] * w[i];
            // batched pixel offsets index HWC buffers with 32-bit ints
            if (t > 0x7fffffffLL || gp > 0x7fffffffLL || (n_img > 1 && 3 * px > 0x7fffffffLL))
                return false;
            g.tile_off[i + 1] = (int)t;
            g.g_off[i + 1] = (int)gp;
            g.pix_off[i + 1] = (int)(px < 0x7fffffffLL ? px : 0x7fffffffLL);
        }
        return true;
    }
    static BatchGeo single(int H, int W, int B, int n) {
        BatchGeo g;
        int32_t h = H, w = W, np = n;
        make(1, &h, &w, &np, B, g);
        return g;
    }
};

// Process-wide count of kernel launches issued by this library.
void note_launches(int n);

}  // namespace lig

// Host-side launch check: every entry point returns a LIG_* status.
#define LIG_LAUNCH_CHECK()                                            \
    do {                                                              \
        cudaError_t e__ = cudaGetLastError();                         \
        if (e__ != cudaSuccess) return LIG_ERR_LAUNCH;                \
    } while (0)
