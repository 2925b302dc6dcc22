// Projection: conic, SnugBox extent, tile bbox and tile-hit count per
// Gaussian, forward and backward, for cov2d and Cholesky inputs.
//
// One thread per Gaussian; the kernels are HBM-bound (52 B/Gaussian forward).
// Every output element is written, so callers need no zero-fill (the reference
// pre-zeroes with torch::zeros, csrc/bindings.cu:89-97).
#include <atomic>
#include <cmath>

#include "common.cuh"

namespace lig {

template <typename T> struct V2 { T x, y; };
template <typename T> struct V3 { T x, y, z; };

// Optional view transform of a render (region decode, scale_to): output
// pixel coordinates are ((x - ox) sx, (y - oy) sy) in the Gaussians' frame,
// so every Gaussian maps to means' = (means - origin) * (sx, sy) and
// L' = diag(sx, sy) L (Cholesky; the scale_to rule of
// minimal_trainer_upscale.py:139-157) or cov' = S cov S.  Off: inputs are used
// as they are.
template <typename T> struct View {
    T ox, oy, sx, sy;
    bool on;
};

// cov2d (a,b,c) from the input triple: pass-through, or the Cholesky product
// [l11^2, l11 l21, l21^2 + l22^2] written as in csrc/forward.cu:79-83.
// VIEW is a template parameter so that the plain projection compiles to
// exactly the reference's arithmetic (a runtime branch changes how the
// compiler contracts the products below, and with it the rounding).
template <typename T, bool VIEW = false>
__device__ __forceinline__ void input_cov(bool chol, const T *in3, int i, T &cx, T &cy, T &cz,
                                          const View<T> &v = View<T>{0, 0, 1, 1, false}) {
    T p = in3[3 * i], q = in3[3 * i + 1], r = in3[3 * i + 2];
    if constexpr (VIEW) {
        if (chol) { p *= v.sx; q *= v.sy; r *= v.sy; }
        else { p *= v.sx * v.sx; q *= v.sx * v.sy; r *= v.sy * v.sy; }
    }
    if (chol) {
        cx = p * p;
        cy = p * q;
        cz = q * q + r * r;
    } else {
        cx = p; cy = q; cz = r;
    }
}

// Forward: csrc/forward.cu:13-105 semantics.  xys holds the mean only where
// the tile area is positive (zero otherwise), conics are written whenever
// det != 0, extents only with a positive tile area.
template <typename T, bool VIEW>
__global__ void project_fwd_kernel(int n, bool chol, const T *__restrict__ in3,
                                   const T *__restrict__ means, const T *__restrict__ opac,
                                   BatchGeo geo, View<T> view, T *__restrict__ xys,
                                   T *__restrict__ extents, T *__restrict__ conics,
                                   int32_t *__restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int im = geo.image_of_gauss(i);
    const unsigned tbx = geo.tbx[im], tby = geo.tby(im), block = geo.B;
    T cx, cy, cz;
    input_cov<T, VIEW>(chol, in3, i, cx, cy, cz, view);
    T o = opac ? opac[i] : (T)1;
    T ca = 0, cb = 0, cc = 0, ex = 0, ey = 0;
    bool ok = cov2d_bounds(cx, cy, cz, o, ca, cb, cc, ex, ey);
    T mx = means[2 * i], my = means[2 * i + 1];
    if constexpr (VIEW) {
        mx = (mx - view.ox) * view.sx;
        my = (my - view.oy) * view.sy;
    }
    int32_t area = 0;
    if (ok) {
        int x0, y0, x1, y1;
        tile_bbox(mx, my, ex, ey, tbx, tby, block, x0, y0, x1, y1);
        area = (int32_t)((unsigned)(x1 - x0) * (unsigned)(y1 - y0));
    } else {
        ca = cb = cc = 0;
    }
    bool hit = area > 0;
    conics[3 * i] = ca;
    conics[3 * i + 1] = cb;
    conics[3 * i + 2] = cc;
    counts[i] = hit ? area : 0;
    extents[2 * i] = hit ? ex : (T)0;
    extents[2 * i + 1] = hit ? ey : (T)0;
    xys[2 * i] = hit ? mx : (T)0;
    xys[2 * i + 1] = hit ? my : (T)0;
}

// conic VJP (csrc/helpers.cuh:101-110): v_Sigma = -X G X for symmetric X
// (conic) and G (v_conic with halved off-diagonal), written out as the
// column-major 2x2 products in the same evaluation order.
template <typename T>
__device__ __forceinline__ void conic_vjp(T a, T b, T c, T va, T vb, T vc, T &oa, T &ob, T &oc) {
    T g01 = vb / (T)2;
    // N = -X
    T n00 = -a, n01 = -b, n10 = -b, n11 = -c;
    // P = N * G  (P[col][row] = N[0][row]*G[col][0] + N[1][row]*G[col][1])
    T p00 = n00 * va + n10 * g01;
    T p01 = n01 * va + n11 * g01;
    T p10 = n00 * g01 + n10 * vc;
    T p11 = n01 * g01 + n11 * vc;
    // Q = P * X
    T q00 = p00 * a + p10 * b;
    T q01 = p01 * a + p11 * b;
    T q10 = p00 * b + p10 * c;
    T q11 = p01 * b + p11 * c;
    oa = q00;
    ob = q10 + q01;
    oc = q11;
}

// Cholesky chain rule with non-finite -> 0 (csrc/backward.cu:228-246).
template <typename T>
__device__ __forceinline__ void chol_chain(T l11, T l21, T l22, T va, T vb, T vc, T &g11, T &g21,
                                           T &g22) {
    using M = Math<T>;
    T a = (T)2 * l11 * va + l21 * vb;
    T b = l11 * vb + (T)2 * l21 * vc;
    T c = (T)2 * l22 * vc;
    bool fin = M::finite_(a) & M::finite_(b) & M::finite_(c);
    g11 = fin ? a : (T)0;
    g21 = fin ? b : (T)0;
    g22 = fin ? c : (T)0;
}

// Backward recomputing conic/extent/bbox from the inputs: the validity test
// (extents > 0 in csrc/backward.cu:195, :217) is re-derived exactly because the
// forward math is re-run with the same code.
template <typename T>
__global__ void project_bwd_kernel(int n, bool chol, const T *__restrict__ in3,
                                   const T *__restrict__ means, const T *__restrict__ opac,
                                   BatchGeo geo, const T *__restrict__ v_xy, int64_t sxy,
                                   const T *__restrict__ v_conic, int64_t sco,
                                   T *__restrict__ v_in3, T *__restrict__ v_mean) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int im = geo.image_of_gauss(i);
    const unsigned tbx = geo.tbx[im], tby = geo.tby(im), block = geo.B;
    T cx, cy, cz;
    input_cov(chol, in3, i, cx, cy, cz);
    T o = opac ? opac[i] : (T)1;
    T ca = 0, cb = 0, cc = 0, ex = 0, ey = 0;
    bool valid = cov2d_bounds(cx, cy, cz, o, ca, cb, cc, ex, ey);
    if (valid) {
        int x0, y0, x1, y1;
        tile_bbox(means[2 * i], means[2 * i + 1], ex, ey, tbx, tby, block, x0, y0, x1, y1);
        int32_t area = (int32_t)((unsigned)(x1 - x0) * (unsigned)(y1 - y0));
        valid = area > 0 && ex > (T)0 && ey > (T)0;
    }
    T o0 = 0, o1 = 0, o2 = 0, m0 = 0, m1 = 0;
    if (valid) {
        m0 = v_xy[sxy * i];
        m1 = v_xy[sxy * i + 1];
        T va, vb, vc;
        conic_vjp(ca, cb, cc, v_conic[sco * i], v_conic[sco * i + 1], v_conic[sco * i + 2], va,
                  vb, vc);
        if (chol)
            chol_chain(in3[3 * i], in3[3 * i + 1], in3[3 * i + 2], va, vb, vc, o0, o1, o2);
        else {
            o0 = va; o1 = vb; o2 = vc;
        }
    }
    v_in3[3 * i] = o0;
    v_in3[3 * i + 1] = o1;
    v_in3[3 * i + 2] = o2;
    v_mean[2 * i] = m0;
    v_mean[2 * i + 1] = m1;
}

// Backward from saved extents/conics (csrc/backward.cu:185-246).
template <typename T>
__global__ void project_bwd_saved_kernel(int n, bool chol, const T *__restrict__ extents,
                                         const T *__restrict__ in3, const T *__restrict__ conics,
                                         const T *__restrict__ v_xy,
                                         const T *__restrict__ v_conic, T *__restrict__ v_in3,
                                         T *__restrict__ v_mean) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T o0 = 0, o1 = 0, o2 = 0, m0 = 0, m1 = 0;
    if (!(extents[2 * i] <= (T)0 || extents[2 * i + 1] <= (T)0)) {
        m0 = v_xy[2 * i];
        m1 = v_xy[2 * i + 1];
        T va, vb, vc;
        conic_vjp(conics[3 * i], conics[3 * i + 1], conics[3 * i + 2], v_conic[3 * i],
                  v_conic[3 * i + 1], v_conic[3 * i + 2], va, vb, vc);
        if (chol)
            chol_chain(in3[3 * i], in3[3 * i + 1], in3[3 * i + 2], va, vb, vc, o0, o1, o2);
        else {
            o0 = va; o1 = vb; o2 = vc;
        }
    }
    v_in3[3 * i] = o0;
    v_in3[3 * i + 1] = o1;
    v_in3[3 * i + 2] = o2;
    v_mean[2 * i] = m0;
    v_mean[2 * i + 1] = m1;
}

// compute_cov2d_bounds utility (csrc/bindings.cu:19-39); zeros where det == 0.
template <typename T>
__global__ void cov2d_bounds_kernel(int n, const T *__restrict__ cov, const T *__restrict__ opac,
                                    T *__restrict__ conics, T *__restrict__ extents) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T ca = 0, cb = 0, cc = 0, ex = 0, ey = 0;
    if (!cov2d_bounds(cov[3 * i], cov[3 * i + 1], cov[3 * i + 2], opac ? opac[i] : (T)1, ca, cb,
                      cc, ex, ey)) {
        ca = cb = cc = ex = ey = 0;
    }
    conics[3 * i] = ca;
    conics[3 * i + 1] = cb;
    conics[3 * i + 2] = cc;
    extents[2 * i] = ex;
    extents[2 * i + 1] = ey;
}

constexpr int kProjThreads = 256;
inline int proj_blocks(int n) { return (n + kProjThreads - 1) / kProjThreads; }

inline bool valid_geometry(int n, int h, int w, int b) {
    return n >= 0 && h > 0 && w > 0 && b >= 1;
}

template <typename T>
int project_fwd(int n, int chol, const void *in3, const void *means, const void *opac,
                const BatchGeo &geo, void *xys, void *ext, void *con, int32_t *cnt,
                cudaStream_t s, View<T> view = View<T>{0, 0, 1, 1, false}) {
    if (n == 0) return LIG_OK;
    if (view.on)
        project_fwd_kernel<T, true><<<proj_blocks(n), kProjThreads, 0, s>>>(
            n, chol != 0, (const T *)in3, (const T *)means, (const T *)opac, geo, view,
            (T *)xys, (T *)ext, (T *)con, cnt);
    else
        project_fwd_kernel<T, false><<<proj_blocks(n), kProjThreads, 0, s>>>(
            n, chol != 0, (const T *)in3, (const T *)means, (const T *)opac, geo, view,
            (T *)xys, (T *)ext, (T *)con, cnt);
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

template <typename T>
int project_bwd(int n, int chol, const void *in3, const void *means, const void *opac,
                const BatchGeo &geo, const void *v_xy, int64_t sxy, const void *v_con,
                int64_t sco, void *v_in3, void *v_mean, cudaStream_t s) {
    if (n == 0) return LIG_OK;
    project_bwd_kernel<T><<<proj_blocks(n), kProjThreads, 0, s>>>(
        n, chol != 0, (const T *)in3, (const T *)means, (const T *)opac, geo, (const T *)v_xy,
        sxy, (const T *)v_con, sco, (T *)v_in3, (T *)v_mean);
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

}  // namespace lig

using namespace lig;

namespace lig {
static std::atomic<long long> g_launches{0};
void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace lig

extern "C" int lig_abi_version(void) { return 1; }

extern "C" int64_t lig_kernel_launches(void) { return (int64_t)lig::g_launches.load(); }

extern "C" int lig_project_fwd(int dtype, int n, int chol, const void *in3, const void *means,
                               const void *opac, int h, int w, int b, void *xys, void *ext,
                               void *con, int32_t *cnt, void *stream) {
    if (!valid_geometry(n, h, w, b) || (n > 0 && (!in3 || !means || !xys || !ext || !con || !cnt)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const BatchGeo geo = BatchGeo::single(h, w, b, n);
    if (dtype == LIG_F32) return project_fwd<float>(n, chol, in3, means, opac, geo, xys, ext, con, cnt, s);
    if (dtype == LIG_F64) return project_fwd<double>(n, chol, in3, means, opac, geo, xys, ext, con, cnt, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_project_bwd(int dtype, int n, int chol, const void *in3, const void *means,
                               const void *opac, int h, int w, int b, const void *v_xy,
                               int64_t sxy, const void *v_con, int64_t sco, void *v_in3,
                               void *v_mean, void *stream) {
    if (!valid_geometry(n, h, w, b) || sxy < 2 || sco < 3 ||
        (n > 0 && (!in3 || !means || !v_xy || !v_con || !v_in3 || !v_mean)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const BatchGeo geo = BatchGeo::single(h, w, b, n);
    if (dtype == LIG_F32)
        return project_bwd<float>(n, chol, in3, means, opac, geo, v_xy, sxy, v_con, sco, v_in3, v_mean, s);
    if (dtype == LIG_F64)
        return project_bwd<double>(n, chol, in3, means, opac, geo, v_xy, sxy, v_con, sco, v_in3, v_mean, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_project_bwd_saved(int dtype, int n, int chol, const void *ext,
                                     const void *in3, const void *con, const void *v_xy,
                                     const void *v_con, void *v_in3, void *v_mean,
                                     void *stream) {
    if (n < 0 || (n > 0 && (!ext || !con || !v_xy || !v_con || !v_in3 || !v_mean)) ||
        (n > 0 && chol && !in3))
        return LIG_ERR_INVALID;
    if (n == 0) return LIG_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        project_bwd_saved_kernel<float><<<proj_blocks(n), kProjThreads, 0, s>>>(
            n, chol != 0, (const float *)ext, (const float *)in3, (const float *)con,
            (const float *)v_xy, (const float *)v_con, (float *)v_in3, (float *)v_mean);
    else if (dtype == LIG_F64)
        project_bwd_saved_kernel<double><<<proj_blocks(n), kProjThreads, 0, s>>>(
            n, chol != 0, (const double *)ext, (const double *)in3, (const double *)con,
            (const double *)v_xy, (const double *)v_con, (double *)v_in3, (double *)v_mean);
    else
        return LIG_ERR_INVALID;
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

extern "C" int lig_cov2d_bounds(int dtype, int n, const void *cov, const void *opac,
                                void *con, void *ext, void *stream) {
    if (n < 0 || (n > 0 && (!cov || !con || !ext))) return LIG_ERR_INVALID;
    if (n == 0) return LIG_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        cov2d_bounds_kernel<float><<<proj_blocks(n), kProjThreads, 0, s>>>(
            n, (const float *)cov, (const float *)opac, (float *)con, (float *)ext);
    else if (dtype == LIG_F64)
        cov2d_bounds_kernel<double><<<proj_blocks(n), kProjThreads, 0, s>>>(
            n, (const double *)cov, (const double *)opac, (double *)con, (double *)ext);
    else
        return LIG_ERR_INVALID;
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

extern "C" int lig_project_fwd_batch(int dtype, int n_img, const int32_t *heights,
                                     const int32_t *widths, const int32_t *counts_per_image,
                                     int chol, const void *in3, const void *means,
                                     const void *opac, int b, void *xys, void *ext, void *con,
                                     int32_t *cnt, void *stream) {
    BatchGeo geo;
    if (!heights || !widths || !counts_per_image ||
        !BatchGeo::make(n_img, heights, widths, counts_per_image, b, geo))
        return LIG_ERR_INVALID;
    const int n = geo.total_points();
    if (n > 0 && (!in3 || !means || !xys || !ext || !con || !cnt)) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32) return project_fwd<float>(n, chol, in3, means, opac, geo, xys, ext, con, cnt, s);
    if (dtype == LIG_F64) return project_fwd<double>(n, chol, in3, means, opac, geo, xys, ext, con, cnt, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_project_bwd_batch(int dtype, int n_img, const int32_t *heights,
                                     const int32_t *widths, const int32_t *counts_per_image,
                                     int chol, const void *in3, const void *means,
                                     const void *opac, int b, const void *v_xy, int64_t sxy,
                                     const void *v_con, int64_t sco, void *v_in3, void *v_mean,
                                     void *stream) {
    BatchGeo geo;
    if (!heights || !widths || !counts_per_image || sxy < 2 || sco < 3 ||
        !BatchGeo::make(n_img, heights, widths, counts_per_image, b, geo))
        return LIG_ERR_INVALID;
    const int n = geo.total_points();
    if (n > 0 && (!in3 || !means || !v_xy || !v_con || !v_in3 || !v_mean)) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return project_bwd<float>(n, chol, in3, means, opac, geo, v_xy, sxy, v_con, sco, v_in3, v_mean, s);
    if (dtype == LIG_F64)
        return project_bwd<double>(n, chol, in3, means, opac, geo, v_xy, sxy, v_con, sco, v_in3, v_mean, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_project_fwd_view(int dtype, int n, int chol, const void *in3,
                                    const void *means, const void *opac, int h, int w, int b,
                                    double origin_x, double origin_y, double scale_x,
                                    double scale_y, void *xys, void *ext, void *con,
                                    int32_t *cnt, void *stream) {
    if (n < 0 || h <= 0 || w <= 0 || b < 1 || !(scale_x > 0.0) || !(scale_y > 0.0) ||
        !std::isfinite(scale_x) || !std::isfinite(scale_y) || !std::isfinite(origin_x) ||
        !std::isfinite(origin_y) ||
        (n > 0 && (!in3 || !means || !xys || !ext || !con || !cnt)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const BatchGeo geo = BatchGeo::single(h, w, b, n);
    if (dtype == LIG_F32)
        return project_fwd<float>(n, chol, in3, means, opac, geo, xys, ext, con, cnt, s,
                                  View<float>{(float)origin_x, (float)origin_y, (float)scale_x,
                                              (float)scale_y, true});
    if (dtype == LIG_F64)
        return project_fwd<double>(n, chol, in3, means, opac, geo, xys, ext, con, cnt, s,
                                   View<double>{origin_x, origin_y, scale_x, scale_y, true});
    return LIG_ERR_INVALID;
}
