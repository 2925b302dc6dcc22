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

// Process-wide count of kernel launches issued by this library.
void note_launches(int n);

}  // namespace lig

// Host-side launch check: every entry point returns a LIG_* status.
#define LIG_LAUNCH_CHECK()                                            \
    do {                                                              \
        cudaError_t e__ = cudaGetLastError();                         \
        if (e__ != cudaSuccess) return LIG_ERR_LAUNCH;                \
    } while (0)
