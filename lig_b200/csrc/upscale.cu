// Gradient-aware Hermite-bicubic upscale (value, d/dx, d/dy, d2/dxdy planes,
// HWC with 3 channels, or 1 for the single-channel form of
// upscaler_torch.py:91-165), forward and backward.
//
// Coordinate maps:
//   mode 0  half-pixel over a ROI with the ROI extent truncated to int,
//           csrc/gradient_aware_upscaler.cu:201-218;
//   mode 1  align-corners (torch.linspace(0, n-1, steps)), upscaler_torch.py:108-122.
// Weights: C^-1 transposed times [1, t, t^2, t^3] (the Hermite basis),
// csrc/gradient_aware_upscaler.cu:137-154.
//
// Forward (HBM-bound: 48 B per source pixel + 12 B per output pixel): a CTA
// owns an 8 x 64 output tile.  It stages the source window of all four planes
// in shared memory with coalesced row loads, forms for every (output row,
// source column) the column products F*cy of the reference
// (csrc/gradient_aware_upscaler.cu:172-175), and finishes each pixel with the
// four cx products.  The expressions match the reference's, so results match
// to rounding.  Windows too large for shared memory (down-scaling) fall back to
// a direct per-pixel gather.
//
// Backward: a gather.  A CTA owns an 8 x 16 block of source texels, finds the
// output rows/columns whose cell corners touch it (monotone maps -> binary
// search), stages that patch of the incoming gradient in shared memory, reduces
// along x then y with the separable weights, and writes each texel's four
// gradients once.  The reference scatters 48 float atomics per output pixel
// (csrc/gradient_aware_upscaler.cu:313-370).
#include "common.cuh"

namespace lig {

__constant__ float kCinvF[16] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f,
                                 -3.f, 3.f, -2.f, -1.f, 2.f, -2.f, 1.f, 1.f};
__constant__ double kCinvD[16] = {1., 0., 0., 0., 0., 0., 1., 0.,
                                  -3., 3., -2., -1., 2., -2., 1., 1.};
template <typename T> __device__ __forceinline__ const T *cinv();
template <> __device__ __forceinline__ const float *cinv<float>() { return kCinvF; }
template <> __device__ __forceinline__ const double *cinv<double>() { return kCinvD; }

template <typename T>
__device__ __forceinline__ void hermite(T t, T (&w)[4]) {
    const T *C = cinv<T>();
    const T t2 = t * t;
    const T t3 = t2 * t;
    w[0] = C[0] * (T)1 + C[4] * t + C[8] * t2 + C[12] * t3;
    w[1] = C[1] * (T)1 + C[5] * t + C[9] * t2 + C[13] * t3;
    w[2] = C[2] * (T)1 + C[6] * t + C[10] * t2 + C[14] * t3;
    w[3] = C[3] * (T)1 + C[7] * t + C[11] * t2 + C[15] * t3;
}

struct UpMap {
    int mode, dst_n, src_n, roi_n;
    double lo;
};

// Source coordinate of output index d (float arithmetic for T=float).
template <typename T>
__device__ __forceinline__ T src_coord(const UpMap &m, int d) {
    if (m.mode == 0) {
        return (T)m.lo + ((T)d + (T)0.5) * (T)m.roi_n / (T)m.dst_n - (T)0.5;
    }
    // torch.linspace(0, n-1, steps): two-sided evaluation, IEEE division
    if (m.dst_n == 1) return (T)0;
    T end = (T)(m.src_n - 1);
    T step;
    if (sizeof(T) == 4) step = (T)__fdiv_rn((float)end, (float)(m.dst_n - 1));
    else step = end / (T)(m.dst_n - 1);
    if (d < m.dst_n / 2) return step * (T)d;
    return end - step * (T)(m.dst_n - 1 - d);
}

template <typename T>
__device__ __forceinline__ void coord(const UpMap &m, int d, int &i0, int &i1, T (&w)[4]) {
    T s = src_coord<T>(m, d);
    int f = (int)Math<T>::floor_(s);
    T t = s - (T)f;
    i1 = max(0, min(f + 1, m.src_n - 1));
    i0 = max(0, min(f, m.src_n - 1));
    hermite<T>(t, w);
}

template <typename T>
__device__ __forceinline__ void coord_idx(const UpMap &m, int d, int &i0, int &i1) {
    T s = src_coord<T>(m, d);
    int f = (int)Math<T>::floor_(s);
    i1 = max(0, min(f + 1, m.src_n - 1));
    i0 = max(0, min(f, m.src_n - 1));
}

// ---------------------------------------------------------------- forward
constexpr int kFwdRows = 8, kFwdCols = 64, kFwdThreads = 256;
constexpr int kFwdMaxSW = kFwdCols + 4;   // staged source columns (scale <= 1 fits)
constexpr int kFwdMaxSH = kFwdRows + 4;   // staged source rows

template <typename T, int C>
struct FwdSmem {
    int x0[kFwdCols], x1[kFwdCols];
    T cx[kFwdCols][4];
    int y0[kFwdRows], y1[kFwdRows];
    T cy[kFwdRows][4];
    T src[4][kFwdMaxSH][kFwdMaxSW * C];   // f, fx, fy, fxy
    T vf[kFwdRows][kFwdMaxSW * C];        // F*cy columns 0/1 (value)
    T vd[kFwdRows][kFwdMaxSW * C];        // F*cy columns 2/3 (x-derivative)
};

template <typename T, int C>
__global__ void __launch_bounds__(kFwdThreads)
upscale_fwd_kernel(UpMap mx, UpMap my, int src_w, const T *__restrict__ f,
                   const T *__restrict__ fx, const T *__restrict__ fy,
                   const T *__restrict__ fxy, T *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FwdSmem<T, C> &S = *reinterpret_cast<FwdSmem<T, C> *>(smem_raw);
    const int dst_w = mx.dst_n, dst_h = my.dst_n;
    const int c0 = blockIdx.x * kFwdCols, r0 = blockIdx.y * kFwdRows;
    const int ncol = min(kFwdCols, dst_w - c0), nrow = min(kFwdRows, dst_h - r0);
    const int tid = threadIdx.x;
    if (tid < ncol) coord<T>(mx, c0 + tid, S.x0[tid], S.x1[tid], S.cx[tid]);
    if (tid >= 128 && tid - 128 < nrow) {
        int r = tid - 128;
        coord<T>(my, r0 + r, S.y0[r], S.y1[r], S.cy[r]);
    }
    __syncthreads();
    const int xs_lo = S.x0[0], xs_hi = S.x1[ncol - 1];
    const int ys_lo = S.y0[0], ys_hi = S.y1[nrow - 1];
    const int SW = xs_hi - xs_lo + 1, SH = ys_hi - ys_lo + 1;
    const T *planes[4] = {f, fx, fy, fxy};
    if (SW >= 1 && SH >= 1 && SW <= kFwdMaxSW && SH <= kFwdMaxSH) {
        // stage source window (coalesced: one contiguous 3*SW segment per row)
        const int seg = C * SW;
        for (int idx = tid; idx < 4 * SH * seg; idx += kFwdThreads) {
            int p = idx / (SH * seg), rem = idx % (SH * seg);
            int r = rem / seg, q = rem % seg;
            S.src[p][r][q] = planes[p][((int64_t)(ys_lo + r) * src_w + xs_lo) * C + q];
        }
        __syncthreads();
        // column products per (output row, source column): the reference's
        // Fcy0/Fcy1 (value planes) and Fcy2/Fcy3 (x-derivative planes)
        for (int idx = tid; idx < nrow * SW; idx += kFwdThreads) {
            int r = idx / SW, x = idx % SW;
            int ya = min(max(S.y0[r] - ys_lo, 0), SH - 1);
            int yb = min(max(S.y1[r] - ys_lo, 0), SH - 1);
            const T *cy = S.cy[r];
#pragma unroll
            for (int ch = 0; ch < C; ++ch) {
                int q = C * x + ch;
                S.vf[r][q] = S.src[0][ya][q] * cy[0] + S.src[0][yb][q] * cy[1] +
                             S.src[2][ya][q] * cy[2] + S.src[2][yb][q] * cy[3];
                S.vd[r][q] = S.src[1][ya][q] * cy[0] + S.src[1][yb][q] * cy[1] +
                             S.src[3][ya][q] * cy[2] + S.src[3][yb][q] * cy[3];
            }
        }
        __syncthreads();
        for (int idx = tid; idx < nrow * kFwdCols; idx += kFwdThreads) {
            int r = idx / kFwdCols, c = idx % kFwdCols;
            if (c >= ncol) continue;
            int xa = min(max(S.x0[c] - xs_lo, 0), SW - 1);
            int xb = min(max(S.x1[c] - xs_lo, 0), SW - 1);
            const T *cx = S.cx[c];
            T *o = out + ((int64_t)(r0 + r) * dst_w + c0 + c) * C;
#pragma unroll
            for (int ch = 0; ch < C; ++ch)
                o[ch] = cx[0] * S.vf[r][C * xa + ch] + cx[1] * S.vf[r][C * xb + ch] +
                        cx[2] * S.vd[r][C * xa + ch] + cx[3] * S.vd[r][C * xb + ch];
        }
        return;
    }
    // direct gather (large source windows)
    for (int idx = tid; idx < nrow * kFwdCols; idx += kFwdThreads) {
        int r = idx / kFwdCols, c = idx % kFwdCols;
        if (c >= ncol) continue;
        const T *cx = S.cx[c], *cy = S.cy[r];
        int64_t i00 = (int64_t)S.y0[r] * src_w + S.x0[c], i01 = (int64_t)S.y0[r] * src_w + S.x1[c];
        int64_t i10 = (int64_t)S.y1[r] * src_w + S.x0[c], i11 = (int64_t)S.y1[r] * src_w + S.x1[c];
        T *o = out + ((int64_t)(r0 + r) * dst_w + c0 + c) * C;
#pragma unroll
        for (int ch = 0; ch < C; ++ch) {
            T F0 = f[C * i00 + ch] * cy[0] + f[C * i10 + ch] * cy[1] + fy[C * i00 + ch] * cy[2] + fy[C * i10 + ch] * cy[3];
            T F1 = f[C * i01 + ch] * cy[0] + f[C * i11 + ch] * cy[1] + fy[C * i01 + ch] * cy[2] + fy[C * i11 + ch] * cy[3];
            T F2 = fx[C * i00 + ch] * cy[0] + fx[C * i10 + ch] * cy[1] + fxy[C * i00 + ch] * cy[2] + fxy[C * i10 + ch] * cy[3];
            T F3 = fx[C * i01 + ch] * cy[0] + fx[C * i11 + ch] * cy[1] + fxy[C * i01 + ch] * cy[2] + fxy[C * i11 + ch] * cy[3];
            o[ch] = cx[0] * F0 + cx[1] * F1 + cx[2] * F2 + cx[3] * F3;
        }
    }
}

// --------------------------------------------------------------- backward
constexpr int kBwdTexH = 8, kBwdTexW = 16, kBwdThreads = 256;
constexpr int kBwdMaxDW = 72, kBwdMaxDH = 40;   // staged output patch (scale <= 4 fits)

template <typename T, int C>
struct BwdSmem {
    int i_lo, i_hi, j_lo, j_hi;
    int x0[kBwdMaxDW], x1[kBwdMaxDW];
    T cx[kBwdMaxDW][4];
    int y0[kBwdMaxDH], y1[kBwdMaxDH];
    T cy[kBwdMaxDH][4];
    int ia[kBwdTexW], ib[kBwdTexW], ja[kBwdTexH], jb[kBwdTexH];
    T g[kBwdMaxDH][kBwdMaxDW * C];
    T uv[kBwdMaxDH][kBwdTexW * C];   // x-reduced with value weights
    T ud[kBwdMaxDH][kBwdTexW * C];   // x-reduced with derivative weights
};

// first index in [0, n) whose map (i0 or i1) satisfies pred, binary search
template <typename T>
__device__ int first_x1_ge(const UpMap &m, int s) {
    int lo = 0, hi = m.dst_n;  // answer in [lo, hi]
    while (lo < hi) {
        int mid = (lo + hi) >> 1, a, b;
        coord_idx<T>(m, mid, a, b);
        if (b >= s) hi = mid; else lo = mid + 1;
    }
    return lo;
}
template <typename T>
__device__ int last_x0_le(const UpMap &m, int s) {
    int lo = -1, hi = m.dst_n - 1;  // answer in [lo, hi]
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1, a, b;
        coord_idx<T>(m, mid, a, b);
        if (a <= s) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <typename T>
__device__ __forceinline__ void wx_of(int s, int a, int b, const T *w, T &wv, T &wd) {
    wv = (a == s ? w[0] : (T)0) + (b == s ? w[1] : (T)0);
    wd = (a == s ? w[2] : (T)0) + (b == s ? w[3] : (T)0);
}

template <typename T, int C>
__global__ void __launch_bounds__(kBwdThreads)
upscale_bwd_kernel(UpMap mx, UpMap my, int src_w, int src_h, const T *__restrict__ g,
                   T *__restrict__ gf, T *__restrict__ gfx, T *__restrict__ gfy,
                   T *__restrict__ gfxy) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BwdSmem<T, C> &S = *reinterpret_cast<BwdSmem<T, C> *>(smem_raw);
    const int dst_w = mx.dst_n;
    const int sx0 = blockIdx.x * kBwdTexW, sy0 = blockIdx.y * kBwdTexH;
    const int nsx = min(kBwdTexW, src_w - sx0), nsy = min(kBwdTexH, src_h - sy0);
    const int tid = threadIdx.x;
    if (tid == 0) {
        S.i_lo = first_x1_ge<T>(mx, sx0);
        S.i_hi = last_x0_le<T>(mx, sx0 + nsx - 1);
    } else if (tid == 32) {
        S.j_lo = first_x1_ge<T>(my, sy0);
        S.j_hi = last_x0_le<T>(my, sy0 + nsy - 1);
    }
    __syncthreads();
    const int i_lo = S.i_lo, i_hi = S.i_hi, j_lo = S.j_lo, j_hi = S.j_hi;
    const int DW = i_hi - i_lo + 1, DH = j_hi - j_lo + 1;
    const bool staged = DW <= kBwdMaxDW && DH <= kBwdMaxDH;
    if (DW <= 0 || DH <= 0) {
        for (int idx = tid; idx < nsy * nsx * C; idx += kBwdThreads) {
            int r = idx / (nsx * C), q = idx % (nsx * C);
            int64_t o = ((int64_t)(sy0 + r) * src_w + sx0) * C + q;
            gf[o] = 0; gfx[o] = 0; gfy[o] = 0; gfxy[o] = 0;
        }
        return;
    }
    if (staged) {
        for (int i = tid; i < DW; i += kBwdThreads) coord<T>(mx, i_lo + i, S.x0[i], S.x1[i], S.cx[i]);
        for (int j = tid; j < DH; j += kBwdThreads) coord<T>(my, j_lo + j, S.y0[j], S.y1[j], S.cy[j]);
        const int seg = C * DW;
        for (int idx = tid; idx < DH * seg; idx += kBwdThreads) {
            int r = idx / seg, q = idx % seg;
            S.g[r][q] = g[((int64_t)(j_lo + r) * dst_w + i_lo) * C + q];
        }
        __syncthreads();
        // candidate output ranges per source column / row (monotone maps)
        if (tid < nsx) {
            int s = sx0 + tid, a = DW, b = -1;
            for (int i = 0; i < DW; ++i)
                if (S.x0[i] == s || S.x1[i] == s) { a = min(a, i); b = max(b, i); }
            S.ia[tid] = a; S.ib[tid] = b;
        } else if (tid >= 64 && tid - 64 < nsy) {
            int r = tid - 64, s = sy0 + r, a = DH, b = -1;
            for (int j = 0; j < DH; ++j)
                if (S.y0[j] == s || S.y1[j] == s) { a = min(a, j); b = max(b, j); }
            S.ja[r] = a; S.jb[r] = b;
        }
        __syncthreads();
        // x-reduction: for each staged output row and source column
        for (int idx = tid; idx < DH * nsx; idx += kBwdThreads) {
            int r = idx / nsx, sc = idx % nsx, s = sx0 + sc;
            T av[C] = {}, ad[C] = {};
            for (int i = S.ia[sc]; i <= S.ib[sc]; ++i) {
                T wv, wd;
                wx_of<T>(s, S.x0[i], S.x1[i], S.cx[i], wv, wd);
#pragma unroll
                for (int ch = 0; ch < C; ++ch) {
                    T gv = S.g[r][C * i + ch];
                    av[ch] += gv * wv;
                    ad[ch] += gv * wd;
                }
            }
#pragma unroll
            for (int ch = 0; ch < C; ++ch) {
                S.uv[r][C * sc + ch] = av[ch];
                S.ud[r][C * sc + ch] = ad[ch];
            }
        }
        __syncthreads();
        // y-reduction and write-out
        for (int idx = tid; idx < nsy * nsx; idx += kBwdThreads) {
            int rr = idx / nsx, sc = idx % nsx, s = sy0 + rr;
            T a0[C] = {}, a1[C] = {}, a2[C] = {}, a3[C] = {};
            for (int j = S.ja[rr]; j <= S.jb[rr]; ++j) {
                T wv, wd;
                wx_of<T>(s, S.y0[j], S.y1[j], S.cy[j], wv, wd);
#pragma unroll
                for (int ch = 0; ch < C; ++ch) {
                    T uv = S.uv[j][C * sc + ch], ud = S.ud[j][C * sc + ch];
                    a0[ch] += uv * wv;   // value plane
                    a1[ch] += ud * wv;   // x-derivative plane
                    a2[ch] += uv * wd;   // y-derivative plane
                    a3[ch] += ud * wd;   // mixed plane
                }
            }
            int64_t o = ((int64_t)s * src_w + sx0 + sc) * C;
#pragma unroll
            for (int ch = 0; ch < C; ++ch) {
                gf[o + ch] = a0[ch]; gfx[o + ch] = a1[ch]; gfy[o + ch] = a2[ch]; gfxy[o + ch] = a3[ch];
            }
        }
        return;
    }
    // large patches (strong down-scaling): per texel, straight from global memory
    for (int idx = tid; idx < nsy * nsx; idx += kBwdThreads) {
        int rr = idx / nsx, sc = idx % nsx, sy = sy0 + rr, sx = sx0 + sc;
        T a0[C] = {}, a1[C] = {}, a2[C] = {}, a3[C] = {};
        int jl = first_x1_ge<T>(my, sy), jh = last_x0_le<T>(my, sy);
        int il = first_x1_ge<T>(mx, sx), ih = last_x0_le<T>(mx, sx);
        for (int j = jl; j <= jh; ++j) {
            int ya, yb;
            T cy[4];
            coord<T>(my, j, ya, yb, cy);
            T yv, yd;
            wx_of<T>(sy, ya, yb, cy, yv, yd);
            if (yv == (T)0 && yd == (T)0) continue;
            for (int i = il; i <= ih; ++i) {
                int xa, xb;
                T cx[4];
                coord<T>(mx, i, xa, xb, cx);
                T xv, xd;
                wx_of<T>(sx, xa, xb, cx, xv, xd);
                const T *gp = g + ((int64_t)j * dst_w + i) * C;
#pragma unroll
                for (int ch = 0; ch < C; ++ch) {
                    T gv = gp[ch];
                    a0[ch] += gv * xv * yv;
                    a1[ch] += gv * xd * yv;
                    a2[ch] += gv * xv * yd;
                    a3[ch] += gv * xd * yd;
                }
            }
        }
        int64_t o = ((int64_t)sy * src_w + sx) * C;
#pragma unroll
        for (int ch = 0; ch < C; ++ch) {
            gf[o + ch] = a0[ch]; gfx[o + ch] = a1[ch]; gfy[o + ch] = a2[ch]; gfxy[o + ch] = a3[ch];
        }
    }
}

inline bool set_smem(const void *fn, size_t bytes) {
    if (bytes <= 48 * 1024) return true;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
           cudaSuccess;
}

template <typename T, int C>
int upscale_fwd(int mode, int src_h, int src_w, int dst_h, int dst_w, double x1, double y1,
                double x2, double y2, const void *f, const void *fx, const void *fy,
                const void *fxy, void *out, cudaStream_t s) {
    // the reference truncates the ROI extent to int (csrc/gradient_aware_upscaler.cu:201-202)
    UpMap mx{mode, dst_w, src_w, (int)((T)x2 - (T)x1), (double)(T)x1};
    UpMap my{mode, dst_h, src_h, (int)((T)y2 - (T)y1), (double)(T)y1};
    size_t sm = sizeof(FwdSmem<T, C>);
    if (!set_smem((const void *)upscale_fwd_kernel<T, C>, sm)) return LIG_ERR_LAUNCH;
    dim3 grid((dst_w + kFwdCols - 1) / kFwdCols, (dst_h + kFwdRows - 1) / kFwdRows);
    upscale_fwd_kernel<T, C><<<grid, kFwdThreads, sm, s>>>(mx, my, src_w, (const T *)f, (const T *)fx,
                                                       (const T *)fy, (const T *)fxy, (T *)out);
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

template <typename T, int C>
int upscale_bwd(int mode, int src_h, int src_w, int dst_h, int dst_w, double x1, double y1,
                double x2, double y2, const void *g, void *gf, void *gfx, void *gfy, void *gfxy,
                cudaStream_t s) {
    UpMap mx{mode, dst_w, src_w, (int)((T)x2 - (T)x1), (double)(T)x1};
    UpMap my{mode, dst_h, src_h, (int)((T)y2 - (T)y1), (double)(T)y1};
    size_t sm = sizeof(BwdSmem<T, C>);
    if (!set_smem((const void *)upscale_bwd_kernel<T, C>, sm)) return LIG_ERR_LAUNCH;
    dim3 grid((src_w + kBwdTexW - 1) / kBwdTexW, (src_h + kBwdTexH - 1) / kBwdTexH);
    upscale_bwd_kernel<T, C><<<grid, kBwdThreads, sm, s>>>(mx, my, src_w, src_h, (const T *)g,
                                                       (T *)gf, (T *)gfx, (T *)gfy, (T *)gfxy);
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

inline bool up_args_ok(int mode, int sh, int sw, int dh, int dw) {
    return (mode == 0 || mode == 1) && sh > 0 && sw > 0 && dh > 0 && dw > 0;
}

}  // namespace lig

using namespace lig;

namespace lig {
template <int C>
int upscale_fwd_dt(int dtype, int mode, int sh, int sw, int dh, int dw, double x1, double y1,
                   double x2, double y2, const void *f, const void *fx, const void *fy,
                   const void *fxy, void *out, cudaStream_t s) {
    if (dtype == LIG_F32)
        return upscale_fwd<float, C>(mode, sh, sw, dh, dw, x1, y1, x2, y2, f, fx, fy, fxy, out, s);
    if (dtype == LIG_F64)
        return upscale_fwd<double, C>(mode, sh, sw, dh, dw, x1, y1, x2, y2, f, fx, fy, fxy, out, s);
    return LIG_ERR_INVALID;
}
template <int C>
int upscale_bwd_dt(int dtype, int mode, int sh, int sw, int dh, int dw, double x1, double y1,
                   double x2, double y2, const void *g, void *gf, void *gfx, void *gfy,
                   void *gfxy, cudaStream_t s) {
    if (dtype == LIG_F32)
        return upscale_bwd<float, C>(mode, sh, sw, dh, dw, x1, y1, x2, y2, g, gf, gfx, gfy, gfxy, s);
    if (dtype == LIG_F64)
        return upscale_bwd<double, C>(mode, sh, sw, dh, dw, x1, y1, x2, y2, g, gf, gfx, gfy, gfxy,
                                      s);
    return LIG_ERR_INVALID;
}
}  // namespace lig

extern "C" int lig_upscale_fwd_nc(int dtype, int mode, int channels, int sh, int sw, int dh,
                                  int dw, double x1, double y1, double x2, double y2,
                                  const void *f, const void *fx, const void *fy, const void *fxy,
                                  void *out, void *stream) {
    if (!up_args_ok(mode, sh, sw, dh, dw) || !f || !fx || !fy || !fxy || !out) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (channels == 3)
        return upscale_fwd_dt<3>(dtype, mode, sh, sw, dh, dw, x1, y1, x2, y2, f, fx, fy, fxy, out, s);
    if (channels == 1)
        return upscale_fwd_dt<1>(dtype, mode, sh, sw, dh, dw, x1, y1, x2, y2, f, fx, fy, fxy, out, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_upscale_bwd_nc(int dtype, int mode, int channels, int sh, int sw, int dh,
                                  int dw, double x1, double y1, double x2, double y2,
                                  const void *g, void *gf, void *gfx, void *gfy, void *gfxy,
                                  void *stream) {
    if (!up_args_ok(mode, sh, sw, dh, dw) || !g || !gf || !gfx || !gfy || !gfxy) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (channels == 3)
        return upscale_bwd_dt<3>(dtype, mode, sh, sw, dh, dw, x1, y1, x2, y2, g, gf, gfx, gfy, gfxy, s);
    if (channels == 1)
        return upscale_bwd_dt<1>(dtype, mode, sh, sw, dh, dw, x1, y1, x2, y2, g, gf, gfx, gfy, gfxy, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_upscale_fwd(int dtype, int mode, int sh, int sw, int dh, int dw, double x1,
                               double y1, double x2, double y2, const void *f, const void *fx,
                               const void *fy, const void *fxy, void *out, void *stream) {
    return lig_upscale_fwd_nc(dtype, mode, 3, sh, sw, dh, dw, x1, y1, x2, y2, f, fx, fy, fxy, out,
                              stream);
}

extern "C" int lig_upscale_bwd(int dtype, int mode, int sh, int sw, int dh, int dw, double x1,
                               double y1, double x2, double y2, const void *g, void *gf,
                               void *gfx, void *gfy, void *gfxy, void *stream) {
    return lig_upscale_bwd_nc(dtype, mode, 3, sh, sw, dh, dw, x1, y1, x2, y2, g, gf, gfx, gfy,
                              gfxy, stream);
}
