// Weighted-sum rasterizer, forward and backward, plain and gradient-aware.
//
// Work decomposition (B200): one CTA per tile (or per work item of a
// batch's flattened (image, tile) list); the tile is split into <= 32
// regions of 32 lanes and warp w owns region w: 8x8 pixels with two pixels
// per lane in the sum forward, 8x4 pixels in the gradient-aware forward and
// the sum backward, the reference's warp in the gradient-aware backward,
// whose v_xy_abs is |sum over that warp| per Gaussian
// (csrc/gradient_aware_rasterizer.cu:317-341).
//
// Gaussian data: a pack kernel writes one 16-byte-aligned 48-byte record per
// Gaussian (mean, conic, opacity, colour, cull half-widths, sigma
// threshold).  The tile's sorted id list is consumed in batches of blockDim
// Gaussians: each thread parks one record in shared memory (fetched into
// registers while the previous batch was processed) together with that
// Gaussian's region mask.
//
// Culling: a warp runs only the Gaussians whose mask has its region bit
// (forward: one ballot per 32 Gaussians, then the set bits in ascending, i.e.
// list, order; backward: a compacted per-warp list).  The mask comes from a
// conservative box around the Gaussian's alpha >= 1/255 ellipse, built with
// margin (see pack_kernel), refined in the backward by an exact
// ellipse-over-rectangle test, so every skipped pixel would have failed the
// reference's own `alpha < 1/255` test (csrc/forward.cu:258): results are
// unchanged.
//
// Per-pixel arithmetic follows the reference (csrc/forward.cu:250-269,
// csrc/backward.cu:102-150, csrc/gradient_aware_rasterizer.cu:201-315,
// :434-482), sigma with explicit roundings in its compiled form (sigma_ref),
// so that the alpha-threshold decisions are the same, and each pixel adds its
// terms in list order.
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "pair.cuh"

namespace lig {

// The fields every evaluation reads come first (two 16-byte loads); opacity
// and the cull data, read at staging or only with opacities, last.
template <typename T> struct alignas(16) Rec {
    T x, y, a, b;      // mean, conic (a, b)
    T c, r, g, bl;     // conic c, colour
    T o, wx, wy, thr;  // opacity, cull half-widths (negative: never cull), sigma threshold
};

// ------------------------------------------------------------ alpha cut
// The reference's per-pixel test rejects a term when sigma < 0 or
// min(clamp, __expf(-sigma)) < 1/255 (csrc/forward.cu:255-258,
// csrc/backward.cu:104-111); for clamp >= 1/255 the second half depends on
// __expf(-sigma) alone.  Over the non-negative floats that decision is a step
// in sigma's bit pattern: it passes below one pattern (the cut) and fails from
// it on, and every negative sigma (sign bit set) fails.  So for a sigma that
// is neither NaN nor -0, the whole test is one unsigned compare,
//   pass  <=>  bits(sigma) < cut.
// The cut is found on the device by the same expression: between 5.5
// (__expf(-5.5) = 0.00409, 4% above 1/255 — far beyond __expf's error) and 5.6
// (6% below) a warp narrows the bracket 32 ways per round (four rounds).
// lig_alpha_cut scans every non-negative float to show the decision is that
// step and that the search finds its edge (a GPU test).
__device__ __forceinline__ bool alpha_passes(float s) {
    return !(s < 0.f || fminf(0.999f, __expf(-s)) < 1.f / 255.f);
}

// One full warp; returns the cut (the first failing bit pattern) in every lane.
__device__ __forceinline__ uint32_t alpha_cut_search() {
    uint32_t lo = __float_as_uint(5.5f), hi = __float_as_uint(5.6f);  // pass(lo), fail(hi)
    const int lane = threadIdx.x & 31;
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t cand = min(lo + (uint32_t)(lane + 1) * step, hi);
        const uint32_t fails = __ballot_sync(0xffffffffu, !alpha_passes(__uint_as_float(cand)));
        const int f = __ffs(fails) - 1;  // hi itself fails, so some lane does
        const uint32_t new_hi = __shfl_sync(0xffffffffu, cand, f);
        if (f > 0) lo = __shfl_sync(0xffffffffu, cand, f - 1);
        hi = new_hi;
    }
    return hi;
}

// The cut on this device, written by every pack launch for the fused forward
// (always the same value) and read by that forward, launched after it on the
// same stream.
__device__ uint32_t g_alpha_cut;

// ------------------------------------------------------------------ pack
// Culling data: the alpha >= 1/255 region of a positive-definite conic is the
// ellipse sigma <= t/2, t = 2 ln(255 o), whose x half-extent is sqrt(t Sxx).
// With t_c = max(t, 0.01) the record carries the box half-widths
// w = 1.001 sqrt(t_c Sxx) + 2 px and the sigma threshold
// thr = 1.001 t_c/2 + 0.02: a pixel with sigma > thr has
// alpha < exp(-0.02)/255, i.e. 2% below the reference's 1/255 cut, far beyond
// the rounding of sigma and __expf, so skipping it changes nothing.  No culling (w < 0) for non-finite inputs, non-positive
// opacity, non-positive-definite or nearly degenerate conics (b^2 > 0.999 ac),
// where the reference's per-pixel tests must run everywhere in the tile, nor
// where a conic entry times the squared reach of the box (plus a 16-pixel
// region) could approach the float range.  A record with culling data
// (w >= 0) therefore has a finite positive-definite conic and finite sigma
// terms, so at every pixel it is evaluated on, sigma is finite and not -0
// (every term of sigma_ref / sigma_half is >= +0 except b dx dy, and their
// sum is +0 or a positive normal or negative float): the alpha cut's compare
// applies.
// HALF: the record carries a/2 and c/2 in place of a and c (the fused-loss
// forward, see sigma_half); the cull data are computed from the full conic.
// zero (backward): also clears the Gaussian's zero_stride accumulators there
// (zero_stride * sizeof(T) a multiple of 16 bytes, 16-byte aligned).
// HALF (float): block 0's first warp also publishes the alpha cut.
template <typename T, bool HALF>
__global__ void pack_kernel(int n, const T *__restrict__ xys, const T *__restrict__ conics,
                            const T *__restrict__ colors, const T *__restrict__ opac,
                            Rec<T> *__restrict__ recs, T *__restrict__ zero, int zero_stride) {
    if (HALF && sizeof(T) == 4 && blockIdx.x == 0 && threadIdx.x < 32) {
        const uint32_t cut = alpha_cut_search();
        if (threadIdx.x == 0) g_alpha_cut = cut;
    }
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (zero) {
        float4 *z = reinterpret_cast<float4 *>(zero + (size_t)i * zero_stride);
        const int nv = zero_stride * (int)sizeof(T) / 16;
        for (int k = 0; k < nv; ++k) z[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    Rec<T> r;
    r.x = xys[2 * i];
    r.y = xys[2 * i + 1];
    r.a = conics[3 * i];
    r.b = conics[3 * i + 1];
    r.c = conics[3 * i + 2];
    r.o = opac ? opac[i] : (T)1;
    r.r = colors[3 * i];
    r.g = colors[3 * i + 1];
    r.bl = colors[3 * i + 2];
    r.thr = 0;
    double a = r.a, b = r.b, c = r.c, o = r.o;
    double det = a * c - b * b;
    bool ok = isfinite((double)r.x) && isfinite((double)r.y) && isfinite(a) && isfinite(b) &&
              isfinite(c) && isfinite(o) && o > 0.0 && a > 0.0 && c > 0.0 && det > 0.0 &&
              b * b <= 0.999 * a * c && fabs(r.x) < 1e7 && fabs(r.y) < 1e7;
    T wx = (T)-1, wy = (T)-1;
    if (ok) {
        double t = 2.0 * log(255.0 * o);
        double tc = t > 0.01 ? t : 0.01;
        double sxx = c / det, syy = a / det;
        double hx = 1.001 * sqrt(tc * sxx) + 2.0, hy = 1.001 * sqrt(tc * syy) + 2.0;
        const float reach = (float)fmax(hx, hy) + 16.f;
        if (hx < 1e7 && hy < 1e7 &&
            fmaxf(fmaxf((float)r.a, (float)r.c), fabsf((float)r.b)) * reach * reach < 1e36f) {
            wx = (T)hx;
            wy = (T)hy;
            r.thr = (T)(0.5 * tc * 1.001 + 0.02);
        }
    }
    r.wx = wx;
    r.wy = wy;
    if (HALF) {
        r.a *= (T)0.5;
        r.c *= (T)0.5;
    }
    recs[i] = r;
}

// ---------------------------------------------------------------- regions
// A tile is split into R <= 32 regions of 32 pixels; warp w of the CTA owns
// region w and each lane owns PPL pixels of it.
//   kind 0: 8x4 blocks, PPL 1               (backward; gradient-aware forward)
//   kind 1: 8x8 blocks, lane owns (x, y) and (x, y + 4)  (sum forward)
//   kind 3: 8x16 blocks, lane owns (x, y + 4p), p < 4   (sum forward, large images)
//   kind 2: the reference's warps, thread ranks 32w..32w+31 with
//           rank = ty*B + tx, PPL 1                    (gradient-aware backward)
struct Regions {
    int kind, B, nbx, nby, count;
    __host__ __device__ static Regions make(int kind, int B) {
        Regions r{kind, B, 1, 1, 1};
        if (kind == 0) { r.nbx = (B + 7) / 8; r.nby = (B + 3) / 4; }
        else if (kind == 1) { r.nbx = (B + 7) / 8; r.nby = (B + 7) / 8; }
        else if (kind == 3) { r.nbx = (B + 7) / 8; r.nby = (B + 15) / 16; }
        else { r.nbx = 1; r.nby = (B * B + 31) / 32; }
        r.count = r.nbx * r.nby;
        return r;
    }
    __device__ __forceinline__ void pixel(int w, int lane, int p, int &lx, int &ly) const {
        if (kind == 0) {
            lx = (w % nbx) * 8 + (lane & 7);
            ly = (w / nbx) * 4 + (lane >> 3);
        } else if (kind == 1 || kind == 3) {
            lx = (w % nbx) * 8 + (lane & 7);
            ly = (w / nbx) * block_h() + (lane >> 3) + 4 * p;
        } else {
            int r = w * 32 + lane;
            lx = r % B;
            ly = r < B * B ? r / B : B;  // B marks "no pixel"
        }
    }
    // rows of a block region (kinds 0, 1, 3)
    __host__ __device__ __forceinline__ int block_h() const {
        return kind == 0 ? 4 : (kind == 1 ? 8 : 16);
    }
    // tile-local pixel-centre rectangle of region w (conservative)
    template <typename T>
    __device__ __forceinline__ void rect(int w, T &x0, T &x1, T &y0, T &y1) const {
        int ix0, ix1, iy0, iy1;
        if (kind == 2) {
            const int r0 = w * 32, r1 = min(w * 32 + 31, B * B - 1);
            iy0 = r0 / B; iy1 = r1 / B;
            if (iy0 == iy1) { ix0 = r0 % B; ix1 = r1 % B; }
            else { ix0 = 0; ix1 = B - 1; }
        } else {
            const int hb = block_h();
            ix0 = (w % nbx) * 8; ix1 = min(ix0 + 7, B - 1);
            iy0 = (w / nbx) * hb; iy1 = min(iy0 + hb - 1, B - 1);
        }
        x0 = (T)ix0 + (T)0.5; x1 = (T)ix1 + (T)0.5;
        y0 = (T)iy0 + (T)0.5; y1 = (T)iy1 + (T)0.5;
    }
    __device__ __forceinline__ uint32_t all() const {
        return count >= 32 ? 0xffffffffu : ((1u << count) - 1u);
    }
    // Regions whose pixel centres (tile-local, pixel i at i + 0.5) can lie in
    // the box [x0, x1] x [y0, y1].  Conservative.
    template <typename T>
    __device__ __forceinline__ uint32_t bits(T x0, T x1, T y0, T y1) const {
        if (kind == 2) {
            // rows j with centre in [y0, y1]; a region spans rows r0/B .. r1/B
            T fy0 = Math<T>::ceil_(y0 - (T)0.5), fy1 = Math<T>::floor_(y1 - (T)0.5);
            if (!(fy0 <= fy1) || fy1 < (T)0 || fy0 > (T)(B - 1)) return 0u;
            int j0 = (int)max(fy0, (T)0), j1 = (int)min(fy1, (T)(B - 1));
            uint32_t m = 0;
            for (int w = 0; w < count; ++w) {
                int r0 = (w * 32) / B, r1 = min(w * 32 + 31, B * B - 1) / B;
                if (r0 <= j1 && r1 >= j0) m |= 1u << w;
            }
            return m;
        }
        const int hb = block_h();
        T c0 = Math<T>::ceil_((x0 - (T)7.5) / (T)8), c1 = Math<T>::floor_((x1 - (T)0.5) / (T)8);
        T r0 = Math<T>::ceil_((y0 - ((T)hb - (T)0.5)) / (T)hb);
        T r1 = Math<T>::floor_((y1 - (T)0.5) / (T)hb);
        c0 = max(c0, (T)0); r0 = max(r0, (T)0);
        c1 = min(c1, (T)(nbx - 1)); r1 = min(r1, (T)(nby - 1));
        if (!(c0 <= c1) || !(r0 <= r1)) return 0u;
        int ic0 = (int)c0, ic1 = (int)c1, ir0 = (int)r0, ir1 = (int)r1;
        uint32_t cols = ((1u << (ic1 - ic0 + 1)) - 1u) << ic0;
        uint32_t m = 0;
        for (int r = ir0; r <= ir1; ++r) m |= cols << (r * nbx);
        return m;
    }
};

// Minimum of sigma(d) = 0.5 (a dx^2 + c dy^2) + b dx dy over the rectangle
// [dx0, dx1] x [dy0, dy1] (positive-definite conic): zero if the rectangle
// holds the origin, else the least of the edge minima (each a clamped 1-D
// quadratic minimum).
// With the centre outside the rectangle the minimum lies on an edge that
// faces the centre (at the minimiser every active bound's inward move must
// not decrease sigma, while the direction to the centre does; that direction
// points outward only across facing edges), so at most one vertical and one
// horizontal edge are evaluated: x = dx0 when dx0 > 0, x = dx1 when dx1 < 0,
// and likewise in y.
template <typename T>
__device__ __forceinline__ T sigma_min_rect(T a, T b, T c, T dx0, T dx1, T dy0, T dy1) {
    const bool ox = dx0 > (T)0 || dx1 < (T)0, oy = dy0 > (T)0 || dy1 < (T)0;
    if (!ox && !oy) return (T)0;
    T best = (T)3.0e38;
    if (ox) {
        const T dx = dx0 > (T)0 ? dx0 : dx1;
        const T dy = min(max(-b * dx / c, dy0), dy1);
        best = (T)0.5 * (a * dx * dx + c * dy * dy) + b * dx * dy;
    }
    if (oy) {
        const T dy = dy0 > (T)0 ? dy0 : dy1;
        const T dx = min(max(-b * dy / a, dx0), dx1);
        best = min(best, (T)0.5 * (a * dx * dx + c * dy * dy) + b * dx * dy);
    }
    return best;
}

// Region mask of one Gaussian for the tile at pixel origin (tx0, ty0): the
// regions whose pixel-centre rectangle meets the Gaussian's cull box and, on
// it, reaches sigma <= thr (see pack_kernel: every pixel with sigma > thr
// fails the reference's own alpha >= 1/255 test).  Records without culling
// data (wx < 0) touch every region.
// ELLIPSE = false stops at the box test.  HALF: the record carries the
// halved conic (fused-loss forward).
template <typename T, bool ELLIPSE = true, bool HALF = false>
__device__ __forceinline__ uint32_t region_bits(const Rec<T> &g, const Regions &R, int tx0,
                                                int ty0) {
    if (!(g.wx >= (T)0)) return R.all();
    const T cx = g.x - (T)tx0, cy = g.y - (T)ty0;
    uint32_t m = R.bits<T>(cx - g.wx, cx + g.wx, cy - g.wy, cy + g.wy);
    if (!ELLIPSE) return m;
    uint32_t keep = m;
    while (m) {
        const int w = __ffs(m) - 1;
        m &= m - 1;
        T x0, x1, y0, y1;
        R.rect<T>(w, x0, x1, y0, y1);
        const T a = HALF ? (T)2 * g.a : g.a, c = HALF ? (T)2 * g.c : g.c;
        if (sigma_min_rect<T>(a, g.b, c, x0 - cx, x1 - cx, y0 - cy, y1 - cy) > g.thr)
            keep &= ~(1u << w);
    }
    return keep;
}

// One region's test of region_bits: does the Gaussian reach region w?
template <typename T, bool ELLIPSE, bool HALF>
__device__ __forceinline__ bool region_hit(const Rec<T> &g, const Regions &R, int w, int tx0,
                                           int ty0) {
    if (!(g.wx >= (T)0)) return true;
    T x0, x1, y0, y1;
    R.rect<T>(w, x0, x1, y0, y1);
    const T cx = g.x - (T)tx0, cy = g.y - (T)ty0;
    if (cx + g.wx < x0 || cx - g.wx > x1 || cy + g.wy < y0 || cy - g.wy > y1) return false;
    if (!ELLIPSE) return true;
    const T a = HALF ? (T)2 * g.a : g.a, c = HALF ? (T)2 * g.c : g.c;
    return !(sigma_min_rect<T>(a, g.b, c, x0 - cx, x1 - cx, y0 - cy, y1 - cy) > g.thr);
}

// ------------------------------------------------------------ tile setup
// Work item -> image and tile origin.  Work items index the flattened
// (image, tile) list of a BatchGeo; a single image is a batch of one.
struct TileCtx {
    int im, H, W, B, tx0, ty0, poff;
    bool empty;  // the image has no intersections (reference empty-list branch)
};

// Intersections of image im: from the inclusive prefix sum of per-Gaussian
// counts when given (batched), else the whole list's total.
__device__ __forceinline__ bool image_empty(const BatchGeo &geo, const int32_t *cum,
                                            const int32_t *d_total, int im) {
    if (!cum) return *d_total == 0;
    const int g0 = geo.g_off[im], g1 = geo.g_off[im + 1];
    if (g1 <= g0) return true;
    const int hi = cum[g1 - 1], lo = g0 > 0 ? cum[g0 - 1] : 0;
    return hi - lo == 0;
}

__device__ __forceinline__ TileCtx tile_ctx(const BatchGeo &geo, const int32_t *cum,
                                            const int32_t *d_total, int tile) {
    TileCtx t;
    t.im = geo.image_of_tile(tile);
    const int lt = tile - geo.tile_off[t.im];
    const int tbx = geo.tbx[t.im];
    t.H = geo.H[t.im];
    t.W = geo.W[t.im];
    t.B = geo.B;
    t.tx0 = (lt % tbx) * t.B;
    t.ty0 = (lt / tbx) * t.B;
    t.poff = geo.pix_off[t.im];
    t.empty = image_empty(geo, cum, d_total, t.im);
    return t;
}

// Next work item: blockIdx.x in a plain launch (one CTA per tile); in a
// persistent launch (work != null) the CTA pulls items from a global counter
// until the list is exhausted.  The loop ends because the counter only grows.
__device__ __forceinline__ int next_tile(int *work, int &s_slot, bool first) {
    if (!work) return first ? (int)blockIdx.x : 0x7fffffff;
    __syncthreads();  // everyone is done with the previous item
    if (threadIdx.x == 0) s_slot = atomicAdd(work, 1);
    __syncthreads();
    return s_slot;
}

// --------------------------------------------------------------- forward
#ifndef LIG_RASTER_FWD_WARPS
#define LIG_RASTER_FWD_WARPS 1  // sum forward: warps stream the tile list independently
#endif
#ifndef LIG_RASTER_FWD_ELLIPSE
#define LIG_RASTER_FWD_ELLIPSE 1  // sum forward: exact ellipse test per region
#endif
#ifndef LIG_RASTER_FWD_ELLIPSE_GA
#define LIG_RASTER_FWD_ELLIPSE_GA 1  // the same in the gradient-aware forward
#endif
#ifndef LIG_RASTER_FWD_FUSED
#define LIG_RASTER_FWD_FUSED 1  // specialised fused-loss forward (no opacities)
#endif
#ifndef LIG_RASTER_ALPHA_CUT
#define LIG_RASTER_ALPHA_CUT 1  // fused forward: alpha test by the cut's compare
#endif
// One CTA per tile, warp w = region w (8x4 pixels), one pixel per lane.
// Batches of blockDim Gaussians (list order) are staged in shared memory, one
// record per thread, with the next batch's record fetched into registers
// while the current batch is processed.  Each thread also stores its
// Gaussian's region mask; a warp then walks only the Gaussians whose mask has
// its bit (ballot over the batch, set bits in ascending order = list order),
// two per iteration so the two sigma/alpha chains overlap, accumulating in
// list order — per pixel exactly the reference's sequence of additions.
// sigma = 0.5 (a dx^2 + c dy^2) + b dx dy (csrc/forward.cu:250-251,
// csrc/backward.cu:102-104, csrc/gradient_aware_rasterizer.cu:201-203),
// rounded step by step as the reference's expression compiles under
// --use_fast_math: fma(b dx, dy, 0.5 fma(a dx, dx, (c dy) dy)) — established by
// comparing the compiled expression against each explicit form on 4M random
// inputs.  Written explicitly so that the surrounding code (several pixels
// per lane sharing products) cannot change the contraction, and with it the
// alpha >= 1/255 decisions.
// Rounded product / fused multiply-add, spelled out so that the compiler
// cannot contract or reassociate them.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) {
    return __fma_rn(a, b, c);
}

template <typename T>
__device__ __forceinline__ T sigma_ref(T a, T b, T c, T dx, T dy);
template <>
__device__ __forceinline__ float sigma_ref<float>(float a, float b, float c, float dx, float dy) {
    const float ta = __fmul_rn(a, dx), tc = __fmul_rn(c, dy), tb = __fmul_rn(b, dx);
    return __fmaf_rn(tb, dy, __fmul_rn(0.5f, __fmaf_rn(ta, dx, __fmul_rn(tc, dy))));
}
template <>
__device__ __forceinline__ double sigma_ref<double>(double a, double b, double c, double dx,
                                                    double dy) {
    const double ta = __dmul_rn(a, dx), tc = __dmul_rn(c, dy), tb = __dmul_rn(b, dx);
    return __fma_rn(tb, dy, __dmul_rn(0.5, __fma_rn(ta, dx, __dmul_rn(tc, dy))));
}

// sigma_ref from the halved conic (ha = a/2, hc = c/2):
//   fma(b dx, dy, fma(ha dx, dx, (hc dy) dy)) == fma(b dx, dy, 0.5 fma(a dx, dx, (c dy) dy))
// bit for bit — halving is exact and commutes with rounding (away from the
// subnormal range, where every term is far below any alpha decision) — with
// one product fewer.
template <typename T>
__device__ __forceinline__ T sigma_half(T ha, T b, T hc, T dx, T dy) {
    return fma_rn(mul_rn(b, dx), dy, fma_rn(mul_rn(ha, dx), dx, mul_rn(mul_rn(hc, dy), dy)));
}

template <typename T>
struct PixelEval {
    // csrc/forward.cu:250-259 (sum) / csrc/gradient_aware_rasterizer.cu:436-445
    // (gradient-aware: d = p - mu); returns false when the term is skipped.
    template <bool GA>
    static __device__ __forceinline__ bool alpha(const Rec<T> &g, T px, T py, T &dx, T &dy,
                                                 T &a) {
        using M = Math<T>;
        if (!GA) { dx = g.x - px; dy = g.y - py; }
        else { dx = px - g.x; dy = py - g.y; }
        const T sigma = sigma_ref<T>(g.a, g.b, g.c, dx, dy);
        a = M::min_((T)0.999, g.o * M::exp_(-sigma));
        return !(sigma < (T)0 || a < (T)1 / (T)255);
    }
    // the fused-loss forward: halved conic in the record, no opacities (o = 1,
    // so o * exp(-sigma) is exp(-sigma) exactly)
    static __device__ __forceinline__ bool alpha_fused(const Rec<T> &g, T px, T py, T &a) {
        using M = Math<T>;
        const T sigma = sigma_half<T>(g.a, g.b, g.c, g.x - px, g.y - py);
        a = M::min_((T)0.999, M::exp_(-sigma));
        return !(sigma < (T)0 || a < (T)1 / (T)255);
    }
};

template <typename T, bool GA>
struct FwdAcc {
    T r = 0, g = 0, b = 0, w = 0;
    T dx[GA ? 3 : 1] = {}, dy[GA ? 3 : 1] = {}, dxy[GA ? 3 : 1] = {};
    int cur = 0;
    // fused-loss forward: colour and, with FIN, the final index (no wsum, not GA)
    template <bool FIN = true>
    __device__ __forceinline__ void add_fused(const Rec<T> &q, T a, int idx) {
        r += q.r * a;
        g += q.g * a;
        b += q.bl * a;
        if constexpr (FIN) cur = idx;
    }
    __device__ __forceinline__ void add(const Rec<T> &q, T dxp, T dyp, T a, int idx) {
        // csrc/forward.cu:264-269, csrc/gradient_aware_rasterizer.cu:451-482
        r += q.r * a;
        g += q.g * a;
        b += q.bl * a;
        if (GA) {
            const T sdx = q.a * dxp + q.b * dyp;
            const T sdy = q.b * dxp + q.c * dyp;
            const T s2 = q.b;
            const T adx = -a * sdx;
            const T ady = -a * sdy;
            const T adxy = -a * (s2 - sdx * sdy);
            dx[0] += q.r * adx; dx[1] += q.g * adx; dx[2] += q.bl * adx;
            dy[0] += q.r * ady; dy[1] += q.g * ady; dy[2] += q.bl * ady;
            dxy[0] += q.r * adxy; dxy[1] += q.g * adxy; dxy[2] += q.bl * adxy;
        }
        w += a;
        cur = idx;
    }
};

// Fused clamped-L2 loss in the forward (fit loops): instead of the image the
// forward writes the masked difference diff = (0 <= x <= 1) ? clamp(x) - t : 0
// (what the loss gradient needs per pixel) and each tile adds
// (clamp(x) - t)^2 over its pixels into one fp64 partial (fixed-order block
// reduction, so the loss is deterministic).  No target: plain forward.
// An 8-bit target (an RGB image as stored) is read as t = byte / 255 rounded
// to nearest: the float value torchvision's ToTensor gives (train.py's image
// loading), so the result equals the fp32 path fed that float target.  In
// float the quotient is q = b * r (r = 1/255 rounded) refined by one
// residual-correction step (Markstein): e = fma(-q, 255, b), t = fma(e, r, q)
// — equal to the correctly rounded b / 255 for every byte b (checked against
// the host's division for all 256 values), with no division.
template <typename T> struct L2Fwd {
    const T *target;
    double *tile_partial;  // [total tiles]
    const uint8_t *target_u8 = nullptr;
    __device__ __forceinline__ bool on() const { return target || target_u8; }
    __device__ __forceinline__ T at(int i) const;
};
template <> __device__ __forceinline__ float L2Fwd<float>::at(int i) const {
    if (!target_u8) return target[i];
    constexpr float r = 0.003921568859368563f;  // 1/255 rounded to nearest (0x3b808081)
    const float b = (float)target_u8[i];
    const float q = __fmul_rn(b, r);
    return __fmaf_rn(__fmaf_rn(-q, 255.0f, b), r, q);
}
template <> __device__ __forceinline__ double L2Fwd<double>::at(int i) const {
    return target_u8 ? __ddiv_rn((double)target_u8[i], 255.0) : target[i];
}

template <typename T>
__device__ __forceinline__ void block_sum_to(double v, double *dst) {
    __shared__ double s_part[32];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s_part[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += s_part[k];
        *dst = t;
    }
    __syncthreads();
}

// Writes one pixel's forward outputs, or in the fused-L2 mode its masked
// difference; returns the pixel's (clamp(x) - t)^2 sum for the tile partial.
template <typename T, bool GA>
__device__ __forceinline__ double fwd_write(const FwdAcc<T, GA> &acc, bool inside, int pix,
                                            T *__restrict__ img, T *__restrict__ wsum,
                                            T *__restrict__ odx, T *__restrict__ ody,
                                            T *__restrict__ odxy,
                                            int32_t *__restrict__ final_idx,
                                            const L2Fwd<T> &l2) {
    if (!inside) return 0.0;
    if (final_idx) final_idx[pix] = acc.cur;
    if (l2.on()) {
        double sq = 0;
        const T x[3] = {acc.r, acc.g, acc.b};
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            const T d = min(max(x[ch], (T)0), (T)1) - l2.at(3 * pix + ch);
            sq += (double)(d * d);
            img[3 * pix + ch] = (x[ch] >= (T)0 && x[ch] <= (T)1) ? d : (T)0;
        }
        return sq;
    }
    img[3 * pix] = acc.r;
    img[3 * pix + 1] = acc.g;
    img[3 * pix + 2] = acc.b;
    wsum[pix] = acc.w;
    if (GA) {
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            odx[3 * pix + ch] = acc.dx[ch];
            ody[3 * pix + ch] = acc.dy[ch];
            odxy[3 * pix + ch] = acc.dxy[ch];
        }
    }
    return 0.0;
}

// PPL pixels per lane: 1 (8x4 regions, two Gaussians per iteration), 2 (8x8
// regions, lane owns (x, y) and (x, y + 4)) or 4 (8x16, (x, y + 4p)); each
// Gaussian's record and loop overhead are shared by the lane's evaluations,
// whose independent sigma / exp chains overlap.  Per pixel the terms are
// added in list order either way.
// FL: the fused-loss forward without opacities (records carry the halved
// conic; no wsum): per pixel the same alphas and colour sums, fewer operations.
template <typename T, bool GA, int PPL, bool FL, bool FIN = true>
__device__ __forceinline__ void fwd_tile(const TileCtx &tc, int tile, const int32_t *__restrict__ ids,
                                         const int2 *__restrict__ tile_bins,
                                         const Rec<T> *__restrict__ recs, T *__restrict__ img,
                                         T *__restrict__ wsum, T *__restrict__ odx,
                                         T *__restrict__ ody, T *__restrict__ odxy,
                                         int32_t *__restrict__ final_idx, Rec<T> *s_rec,
                                         uint32_t *s_bits, const L2Fwd<T> &l2, uint32_t cut) {
    // the alpha cut's compare: the fused forward's pixel pairs (float)
    constexpr bool kCut = FL && PPL > 1 && sizeof(T) == 4 && LIG_RASTER_ALPHA_CUT;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int B = tc.B, tx0 = tc.tx0, ty0 = tc.ty0;
    static_assert(PPL == 1 || PPL == 2 || PPL == 4, "one, two or four pixels per lane");
    const Regions R = Regions::make(PPL == 1 ? 0 : (PPL == 2 ? 1 : 3), B);
    // a warp lists only the Gaussians whose alpha >= 1/255 ellipse meets
    // its region (one test per Gaussian and region)
    constexpr bool ELL = LIG_RASTER_FWD_ELLIPSE && (!GA || LIG_RASTER_FWD_ELLIPSE_GA);
    bool inside[PPL];
    int pix[PPL];
    T px[PPL], py[PPL];
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
        int lx, ly;
        R.pixel(w, lane, p, lx, ly);
        const int gx = tx0 + lx, gy = ty0 + ly;
        inside[p] = lx < B && ly < B && gx < tc.W && gy < tc.H;
        pix[p] = tc.poff + gy * tc.W + gx;
        px[p] = (T)gx + (T)0.5;
        py[p] = (T)gy + (T)0.5;
    }

    FwdAcc<T, GA> acc[PPL];
    // walk the Gaussians of `mask` (bits of the 32 records at rb, list
    // indices ib + bit) in list order; fast_tag true: every record has
    // culling data, so the fused forward tests alpha by the cut's compare
    auto walk = [&](uint32_t mask, const Rec<T> *rb, int ib, auto fast_tag) {
        [[maybe_unused]] constexpr bool FAST = decltype(fast_tag)::value;
        if constexpr (FL && PPL == 1) {
            while (mask) {
                const int b1 = __ffs(mask) - 1;
                mask &= mask - 1;
                const Rec<T> g1 = rb[b1];
                T a1;
                const bool ok1 = PixelEval<T>::alpha_fused(g1, px[0], py[0], a1);
                if (mask) {
                    const int b2 = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const Rec<T> g2 = rb[b2];
                    T a2;
                    const bool ok2 = PixelEval<T>::alpha_fused(g2, px[0], py[0], a2);
                    if (ok1) acc[0].template add_fused<FIN>(g1, a1, ib + b1);
                    if (ok2) acc[0].template add_fused<FIN>(g2, a2, ib + b2);
                } else if (ok1) {
                    acc[0].template add_fused<FIN>(g1, a1, ib + b1);
                }
            }
        } else if constexpr (FL) {
            // a lane's pixels share their column: dx, (a/2) dx and
            // b dx once per Gaussian (sigma_half's products)
            using M = Math<T>;
            while (mask) {
                const int b1 = __ffs(mask) - 1;
                mask &= mask - 1;
                const Rec<T> g1 = rb[b1];
                const T dx = g1.x - px[0];
                const T hadx = mul_rn(g1.a, dx), bdx = mul_rn(g1.b, dx);
                T ap[PPL];
                bool okp[PPL];
#pragma unroll
                for (int p = 0; p < PPL; ++p) {
                    const T dy = g1.y - py[p];
                    const T sg = fma_rn(bdx, dy, fma_rn(hadx, dx, mul_rn(mul_rn(g1.c, dy), dy)));
                    ap[p] = M::min_((T)0.999, M::exp_(-sg));
                    if constexpr (FAST) okp[p] = __float_as_uint((float)sg) < cut;
                    else okp[p] = !(sg < (T)0 || ap[p] < (T)1 / (T)255);
                }
#pragma unroll
                for (int p = 0; p < PPL; ++p)
                    if (okp[p]) acc[p].template add_fused<FIN>(g1, ap[p], ib + b1);
            }
        } else if constexpr (PPL == 1) {
            while (mask) {
                const int b1 = __ffs(mask) - 1;
                mask &= mask - 1;
                const Rec<T> g1 = rb[b1];
                T dx1, dy1, a1;
                const bool ok1 =
                    PixelEval<T>::template alpha<GA>(g1, px[0], py[0], dx1, dy1, a1);
                if (mask) {
                    const int b2 = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const Rec<T> g2 = rb[b2];
                    T dx2, dy2, a2;
                    const bool ok2 =
                        PixelEval<T>::template alpha<GA>(g2, px[0], py[0], dx2, dy2, a2);
                    if (ok1) acc[0].add(g1, dx1, dy1, a1, ib + b1);
                    if (ok2) acc[0].add(g2, dx2, dy2, a2, ib + b2);
                } else if (ok1) {
                    acc[0].add(g1, dx1, dy1, a1, ib + b1);
                }
            }
        } else {
            while (mask) {
                const int b1 = __ffs(mask) - 1;
                mask &= mask - 1;
                const Rec<T> g1 = rb[b1];
                T dxp[PPL], dyp[PPL], ap[PPL];
                bool okp[PPL];
#pragma unroll
                for (int p = 0; p < PPL; ++p)
                    okp[p] = PixelEval<T>::template alpha<GA>(g1, px[p], py[p], dxp[p],
                                                              dyp[p], ap[p]);
#pragma unroll
                for (int p = 0; p < PPL; ++p)
                    if (okp[p]) acc[p].add(g1, dxp[p], dyp[p], ap[p], ib + b1);
            }
        }
    };
    if (!tc.empty) {
        const int2 range = tile_bins[tile];
        if constexpr (LIG_RASTER_FWD_WARPS) {
            // each warp streams the tile's list in chunks of 32 on its own
            // (its region's test only, no block barriers: warps whose
            // regions have short lists do not wait for the others)
            Rec<T> *w_rec = s_rec + w * 32;
            Rec<T> pre;
            if (range.x + lane < range.y) pre = recs[__ldg(ids + range.x + lane)];
            for (int base = range.x; base < range.y; base += 32) {
                const bool hit =
                    base + lane < range.y && region_hit<T, ELL, FL>(pre, R, w, tx0, ty0);
                // a chunk whose records all carry culling data takes the cut
                bool fast = false;
                if constexpr (kCut)
                    fast = !__any_sync(FULL, base + lane < range.y && !(pre.wx >= (T)0));
                __syncwarp();
                w_rec[lane] = pre;
                __syncwarp();
                if (base + 32 + lane < range.y) pre = recs[__ldg(ids + base + 32 + lane)];
                const uint32_t mask = __ballot_sync(FULL, hit);
                if (fast) walk(mask, w_rec, base, std::true_type{});
                else walk(mask, w_rec, base, std::false_type{});
            }
        } else {
            const int nt = blockDim.x;
            Rec<T> pre;
            if (range.x + tid < range.y) pre = recs[__ldg(ids + range.x + tid)];
            for (int base = range.x; base < range.y; base += nt) {
                const int cnt = min(nt, range.y - base);
                __syncthreads();
                if (tid < cnt) {
                    s_rec[tid] = pre;
                    s_bits[tid] = region_bits<T, ELL, FL>(pre, R, tx0, ty0);
                }
                __syncthreads();
                if (base + nt + tid < range.y) pre = recs[__ldg(ids + base + nt + tid)];
                for (int m = 0; m * 32 < cnt; ++m) {
                    const int t = m * 32 + lane;
                    walk(__ballot_sync(FULL, t < cnt && ((s_bits[t] >> w) & 1u)), s_rec + m * 32,
                         base + m * 32, std::false_type{});
                }
            }
        }
    } else {  // the reference's empty-list branch (rasterize.py:80-90)
#pragma unroll
        for (int p = 0; p < PPL; ++p) acc[p].r = acc[p].g = acc[p].b = (T)1;
    }
    double sq = 0.0;
#pragma unroll
    for (int p = 0; p < PPL; ++p)
        sq += fwd_write<T, GA>(acc[p], inside[p], pix[p], img, wsum, odx, ody, odxy, final_idx, l2);
    if (l2.on()) block_sum_to<T>(sq, l2.tile_partial + tile);
}

// Launch bounds: tiles of B <= 16 launch <= 256 threads, and their
// instantiation asks for LIG_RASTER_FWD_MINB / LIG_RASTER_BWD_MINB resident
// CTAs per SM (the register budget follows); larger tiles use the 1024-thread
// instantiation.
#ifndef LIG_RASTER_FWD_MINB
#define LIG_RASTER_FWD_MINB 4
#endif
#ifndef LIG_RASTER_BWD_LEAN_MINB
#define LIG_RASTER_BWD_LEAN_MINB 4  // the paired loop wants the larger register budget
#endif
// From LIG_RASTER_BWD_LARGE_MIN_TILES tiles on, the lean backward asks for
// LIG_RASTER_BWD_LEAN_MINB_LARGE resident CTAs per SM (fewer registers, a few
// spilled, more warps to hide latency): measured 4% faster at 8192^2 and
// 1% at 2048^2, but 14% slower at 512^2 (1024 tiles).
#ifndef LIG_RASTER_BWD_LEAN_MINB_LARGE
#define LIG_RASTER_BWD_LEAN_MINB_LARGE 5  // pairs + bulk-staged records (48 registers)
#endif
#ifndef LIG_RASTER_BWD_LARGE_MIN_TILES
#define LIG_RASTER_BWD_LARGE_MIN_TILES 4096
#endif
#ifndef LIG_RASTER_BWD_RROWS
#define LIG_RASTER_BWD_RROWS 0  // float lean walks of large images: region rows (4, 8, 16; 0: by density)
#endif
// Region rows by density (Gaussians per pixel): taller regions save per-pair
// work, but evaluate more pixels a pair cannot reach, which costs more when
// the tile lists are long.  Measured (lean backward, 16x16 tiles): at 0.03
// Gaussians per pixel (8192^2, 2M) 8x16 2.05 ms, 8x8 2.18, 8x4 2.79; at 0.06
// (4096^2, 1M) 8x16 0.99, 8x8 0.89; at 0.12 (4096^2, 2M) 1.86 / 1.63 / 1.67;
// at 0.24 (2048^2, 1M) 0.94 / 0.79 / 0.81.  The crossover is near 0.04.
#ifndef LIG_RASTER_BWD_R16_MAX_DENSITY
#define LIG_RASTER_BWD_R16_MAX_DENSITY 0.04
#endif
#ifndef LIG_RASTER_BWD_RROWS_MINB
#define LIG_RASTER_BWD_RROWS_MINB 8  // resident CTAs per SM of the 8x8 walk (128 threads)
#endif
#ifndef LIG_RASTER_BWD_R16_MINB
#define LIG_RASTER_BWD_R16_MINB 14  // resident CTAs per SM of the 8x16 walk (64 threads, 72 registers)
#endif
#ifndef LIG_RASTER_BWD_SPLIT2
#define LIG_RASTER_BWD_SPLIT2 8  // with up to this many Gaussians left, 4 lanes take one
#endif
#ifndef LIG_RASTER_BWD_R16_SPLIT1
#define LIG_RASTER_BWD_R16_SPLIT1 32  // the 8x16 walk: 2 lanes per Gaussian at least
#endif
#ifndef LIG_RASTER_BWD_R16_SPLIT3
#define LIG_RASTER_BWD_R16_SPLIT3 8  // the 8x16 walk: 8 lanes per Gaussian from this many left
#endif
#ifndef LIG_RASTER_BWD_SPLIT3
#define LIG_RASTER_BWD_SPLIT3 4  // with up to this many Gaussians left, 8 lanes take one
#endif
#ifndef LIG_RASTER_BWD_SPLIT
#define LIG_RASTER_BWD_SPLIT 1  // split a short list's Gaussians across lanes (measured faster)
#endif
#ifndef LIG_RASTER_BWD_SPLIT1
#define LIG_RASTER_BWD_SPLIT1 24  // with up to this many Gaussians left, 2 lanes take one
#endif
#ifndef LIG_RASTER_BWD_LANE_ELLIPSE
#define LIG_RASTER_BWD_LANE_ELLIPSE 1  // ellipse culling by the warp's lanes (measured faster)
#endif
#ifndef LIG_RASTER_BWD_MINB
#define LIG_RASTER_BWD_MINB 5
#endif

// Sum forward: two pixels per lane from LIG_RASTER_PPL2_MIN_TILES tiles on,
// four from LIG_RASTER_PPL4_MIN_TILES on (fewer warps per tile, so small
// images keep more pixels in flight with fewer pixels per lane).
#ifndef LIG_RASTER_PPL2_MIN_TILES
#define LIG_RASTER_PPL2_MIN_TILES 0
#endif
#ifndef LIG_RASTER_PPL4_MIN_TILES
#define LIG_RASTER_PPL4_MIN_TILES 4096  // measured: faster from 2048^2 up, not at 512^2
#endif

template <typename T, bool GA, int PPL, int MAXT, int MINB, bool FL = false, bool FIN = true>
__global__ void __launch_bounds__(MAXT, MINB)
raster_fwd_kernel(const BatchGeo geo, const int32_t *__restrict__ cum, int *work,
                  const int32_t *__restrict__ ids, const int2 *__restrict__ tile_bins,
                  const int32_t *__restrict__ d_total, const Rec<T> *__restrict__ recs,
                  T *__restrict__ img, T *__restrict__ wsum, T *__restrict__ odx,
                  T *__restrict__ ody, T *__restrict__ odxy, int32_t *__restrict__ final_idx,
                  L2Fwd<T> l2) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_slot;
    Rec<T> *s_rec = reinterpret_cast<Rec<T> *>(smem_raw);
    uint32_t *s_bits = reinterpret_cast<uint32_t *>(s_rec + blockDim.x);
    const int n_tiles = geo.total_tiles();
    const uint32_t cut = FL && sizeof(T) == 4 ? g_alpha_cut : 0u;
    for (int tile = next_tile(work, s_slot, true); tile < n_tiles;
         tile = next_tile(work, s_slot, false)) {
        const TileCtx tc = tile_ctx(geo, cum, d_total, tile);
        fwd_tile<T, GA, PPL, FL, FIN>(tc, tile, ids, tile_bins, recs, img, wsum, odx, ody, odxy,
                                      final_idx, s_rec, s_bits, l2, cut);
    }
}

// Loss from the tile partials, deterministic.  Pass 1: each CTA sums a
// chunk of kLossChunk tile partials of one image (thread-strided, then a
// fixed-order block reduction); image i owns CTAs [chunk_off[i],
// chunk_off[i+1]).  Pass 2: one warp per image adds its chunk sums in order
// (lane-strided + butterfly) and divides by 3 H_i W_i; thread 0 adds the
// image means in order.
constexpr int kLossChunk = 4096;

struct TileChunks {
    int n_img;
    int chunk_off[kMaxBatch + 1];
};

inline TileChunks tile_chunks(const BatchGeo &geo) {
    TileChunks c;
    c.n_img = geo.n_img;
    c.chunk_off[0] = 0;
    for (int i = 0; i < geo.n_img; ++i) {
        const int t = geo.tile_off[i + 1] - geo.tile_off[i];
        c.chunk_off[i + 1] = c.chunk_off[i] + (t + kLossChunk - 1) / kLossChunk;
    }
    return c;
}

__global__ void __launch_bounds__(256)
l2_tiles_chunk_kernel(const BatchGeo geo, const TileChunks ch, const double *__restrict__ partial,
                      double *__restrict__ chunk_sum) {
    __shared__ double s_w[8];
    const int b = blockIdx.x;
    const int im = BatchGeo::find(ch.chunk_off, ch.n_img, b);
    const int k0 = geo.tile_off[im] + (b - ch.chunk_off[im]) * kLossChunk;
    const int k1 = min(k0 + kLossChunk, geo.tile_off[im + 1]);
    double t = 0;
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) t += partial[k];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s_w[w] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double u = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) u += s_w[k];
        chunk_sum[b] = u;
    }
}

template <typename T>
__global__ void __launch_bounds__(1024)
l2_chunks_final_kernel(const BatchGeo geo, const TileChunks ch,
                       const double *__restrict__ chunk_sum, T *__restrict__ loss,
                       T *__restrict__ per_image) {
    __shared__ double s_mean[kMaxBatch];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int im = w; im < geo.n_img; im += 32) {
        double t = 0;
        for (int k = ch.chunk_off[im] + lane; k < ch.chunk_off[im + 1]; k += 32) t += chunk_sum[k];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) {
            const double m = t / (3.0 * (double)geo.H[im] * (double)geo.W[im]);
            s_mean[im] = m;
            if (per_image) per_image[im] = (T)m;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double total = 0;
        for (int im = 0; im < geo.n_img; ++im) total += s_mean[im];
        *loss = (T)total;
    }
}

// ------------------------------------------------------------- backward
template <typename T>
struct Grads {  // the ABI's per-Gaussian gradient arrays (v_opac may be null)
    T *v_xy, *v_abs, *v_conic, *v_rgb, *v_opac;
};

// Backward, transposed: one CTA per tile, warp w owns region w (an 8x4 block in
// the sum variant; in the gradient-aware variant the reference's warp w, whose
// v_xy_abs is |sum over that warp| per Gaussian,
// csrc/gradient_aware_rasterizer.cu:317-341).  The tile's pixel cotangents,
// pixel centres and final indices are staged in shared memory once, region
// by region.  Per batch each warp compacts the batch slots whose region box it
// meets (exact ellipse test by the lanes); lanes then take one such Gaussian
// each — or, for a short list, 2 / 4 / 8 lanes share one and take interleaved
// pixels — and loop over the region's pixels (pixel data read by broadcast),
// accumulating the Gaussian's gradient terms in registers; a lane group is
// combined with shuffles, and the terms go to the packed per-Gaussian buffer
// with 16-byte atomics per (Gaussian, region) — [N][12], three atomics, in
// general; [N][8], two, in the lean fused-loss variant.  Entries past every
// pixel's final index are skipped.
//
// Pixel cotangent source of the backward: explicit dL/dimg (+ optional
// dL/dwsum), or — fused L2 — computed on the fly from the render and the target
// as the gradient of mean((clamp(img, 0, 1) - target)^2): the value torch's
// mse_loss + clamp backward produce, 2/N (clamp(x) - t) g where 0 <= x <= 1.
template <typename T>
struct CotSrc {
    const T *v_img, *v_wsum;              // explicit (v_wsum may be null: zero)
    const T *img, *target, *grad_loss;    // fused L2 (v_img == null)
    T scale;                              // 2 / numel
    const T *diff = nullptr;              // fused L2 from the forward's masked difference
    __device__ __forceinline__ void get(int p, T &r, T &g, T &b, T &w) const {
        w = v_wsum ? v_wsum[p] : (T)0;
        if (v_img) {
            r = v_img[3 * p];
            g = v_img[3 * p + 1];
            b = v_img[3 * p + 2];
            return;
        }
        const T s = scale * *grad_loss;
        if (diff) {
            r = diff[3 * p] * s;
            g = diff[3 * p + 1] * s;
            b = diff[3 * p + 2] * s;
            return;
        }
        T v[3];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            const T x = img[3 * p + ch];
            const T d = min(max(x, (T)0), (T)1) - target[3 * p + ch];
            v[ch] = (x >= (T)0 && x <= (T)1) ? d * s : (T)0;
        }
        r = v[0]; g = v[1]; b = v[2];
    }
};

template <typename T, bool GA>
struct alignas(16) PixRec {
    T vo0, vo1, vo2, vw;  // first: one 16-byte load in the lean loop
    T px, py;
    int fin;
    T vd[GA ? 9 : 1];  // vdx.rgb, vdy.rgb, vdxy.rgb
};

#ifndef LIG_RASTER_BWD_COLS
#define LIG_RASTER_BWD_COLS 1  // lean backward: column-major region walk
#endif

// Lean backward of one Gaussian over the pixels of one 8x4 region that this
// lane takes: columns part, part + 2^LS, ... (8 >> LS of them) in each of the
// four rows, column by column.  The separable pieces of sigma are shared:
// per row dy and (c/2 dy) dy, per column dx, (a/2) dx and b dx, so that
//   sigma = fma(b dx, dy, fma((a/2) dx, dx, ((c/2) dy) dy))
// which equals sigma_ref's fma(b dx, dy, 0.5 fma(a dx, dx, (c dy) dy)) bit for
// bit (halving is exact and commutes with rounding away from the subnormal
// range) with one product fewer.  No opacities on this path (o = 1, so
// alpha = min(clamp, exp(-sigma)) is the reference's o * exp(-sigma) clamped).
// No final-index test either: a Gaussian after a pixel's final index fails
// that pixel's alpha test here exactly as it did in the forward.  A skipped
// pair adds zeros.  The moment sums of v_sigma dx^i dy^j (v_sigma =
// -alpha v_alpha) use dx constant along a column: Sx, Sxx and Sxy take one
// term per column.  Leaves Sx, Sy, Sxx, Sxy, Syy in acc[0, 1, 4, 5, 6] and the
// colour sums in acc[7..9].
template <typename T, int LS>
__device__ __forceinline__ void lean_region(const Rec<T> &g, T clamp,
                                            const PixRec<T, false> *__restrict__ pix, int part,
                                            T px0, T py0, T (&acc)[11]) {
    using M = Math<T>;
    constexpr int NC = 8 >> LS, JS = 1 << LS;
    const T ha = (T)0.5 * g.a, hc = (T)0.5 * g.c;
    T dy[4], cdd[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        dy[r] = g.y - (py0 + (T)r);
        cdd[r] = mul_rn(mul_rn(hc, dy[r]), dy[r]);
    }
    T sx = 0, sy = 0, sxx = 0, sxy = 0, syy = 0, c0 = 0, c1 = 0, c2 = 0;
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        const T dx = g.x - (px0 + (T)(k * JS));
        const T hadx = mul_rn(ha, dx), bdx = mul_rn(g.b, dx);
        T wc = 0, yc = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const PixRec<T, false> &c = pix[r * 8 + part + k * JS];
            const T s = fma_rn(bdx, dy[r], fma_rn(hadx, dx, cdd[r]));
            const T al = M::min_(clamp, M::exp_(-s));
            const T a = (s < (T)0 || al < (T)1 / (T)255) ? (T)0 : al;
            c0 += a * c.vo0;
            c1 += a * c.vo1;
            c2 += a * c.vo2;
            const T wv = a * (g.r * c.vo0 + g.g * c.vo1 + g.bl * c.vo2);  // -v_sigma
            wc += wv;
            const T ty = wv * dy[r];
            yc += ty;
            syy += ty * dy[r];
        }
        const T tx = wc * dx;
        sx += tx;
        sxx += tx * dx;
        sy += yc;
        sxy += yc * dx;
    }
    acc[0] = -sx; acc[1] = -sy; acc[4] = -sxx; acc[5] = -sxy; acc[6] = -syy;
    acc[7] = c0; acc[8] = c1; acc[9] = c2;
}

#ifndef LIG_RASTER_BWD_F2
#define LIG_RASTER_BWD_F2 1  // lean backward (float): pixel pairs in f32x2 arithmetic
#endif

// The lean backward's pixel cotangents in pair layout: region entry
// row * 4 + cp holds columns cp and cp + 4 of that row, channel by channel,
// so one 16-byte and one 8-byte load give three ready (column cp, cp + 4)
// pairs.
struct alignas(16) PixPair {
    float v[8];  // v0 (cp, cp+4), v1 (cp, cp+4), v2 (cp, cp+4), unused
};

// lean_region in f32x2 form (float): the lane takes NCP column pairs
// c0, c0 + CSTEP, ... (columns cp and cp + 4 of each) in NR rows r0.. of the
// 8-column region, and evaluates the two pixels of a pair with one packed
// operation where lean_region uses two.  Per pixel the operations and their
// roundings are lean_region's — sigma = fma(b dx, dy, fma((a/2) dx, dx,
// ((c/2) dy) dy)), alpha = min(clamp, exp(-sigma)) and the same alpha test —
// so the alpha decisions are bit-identical; only the order in which the
// moment and colour sums are added differs.  Same quantities as lean_region,
// added to acc[] (zeroed by the caller).  NH > 1 walks NH blocks of NR rows
// (rows r0 .. r0 + NH NR - 1 of a taller region, 4 pair entries a row in pp).
// ABS: also the per-pixel absolute values of the mean gradient summed over
// the pixels (the reference's v_xy_abs, csrc/backward.cu:146-150), in acc[2],
// acc[3]: per pixel v_sigma (a dx + b dy) and v_sigma (b dx + c dy).
template <int NCP, int CSTEP, int NR, bool ABS = false, int NH = 1>
__device__ __forceinline__ void lean_region_f2(const Rec<float> &g, float clamp,
                                               const PixPair *__restrict__ pp, int c0, int r0,
                                               float px0, float py0, float (&acc)[11]) {
    const float ha = 0.5f * g.a, hc = 0.5f * g.c;
    const f2 HA = f2_dup(ha), BB = f2_dup(g.b);
    f2 AA, CC;
    float ax = 0.f, ay = 0.f;
    if constexpr (ABS) {
        AA = f2_dup(g.a);
        CC = f2_dup(g.c);
    }
    const f2 CR = f2_dup(g.r), CG = f2_dup(g.g), CB = f2_dup(g.bl);
    f2 sx = f2_zero(), sy = f2_zero(), sxx = f2_zero(), sxy = f2_zero(), syy = f2_zero();
    f2 sr = f2_zero(), sg = f2_zero(), sb = f2_zero();
    // NH blocks of NR rows, one after the other (not interleaved: the sums
    // carry over, the row and column products are rebuilt per block)
#pragma unroll 1
    for (int hh = 0; hh < NH; ++hh) {
        const int rb = r0 + hh * NR;
        f2 DY[NR], CDD[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const float dy = g.y - (py0 + (float)(rb + r));
            DY[r] = f2_dup(dy);
            CDD[r] = f2_dup(__fmul_rn(__fmul_rn(hc, dy), dy));
        }
#pragma unroll
        for (int k = 0; k < NCP; ++k) {
            const int cp = c0 + k * CSTEP;
            const f2 DX = f2_pack(g.x - (px0 + (float)cp), g.x - (px0 + (float)(cp + 4)));
            const f2 HADX = f2_mul(HA, DX), BDX = f2_mul(BB, DX);
            f2 AX;
            if constexpr (ABS) AX = f2_mul(AA, DX);
            f2 wc = f2_zero(), yc = f2_zero();
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const PixPair *e = pp + (rb + r) * 4 + cp;
                const ulonglong2 v01 = *reinterpret_cast<const ulonglong2 *>(e->v);
                const f2 V0{v01.x}, V1{v01.y};
                const f2 V2{*reinterpret_cast<const unsigned long long *>(e->v + 4)};
                const f2 S = f2_fma(BDX, DY[r], f2_fma(HADX, DX, CDD[r]));
                float s0, s1;
                f2_unpack(S, s0, s1);
                const float al0 = fminf(clamp, __expf(-s0)), al1 = fminf(clamp, __expf(-s1));
                const float a0 = (s0 < 0.f || al0 < 1.f / 255.f) ? 0.f : al0;
                const float a1 = (s1 < 0.f || al1 < 1.f / 255.f) ? 0.f : al1;
                const f2 A = f2_pack(a0, a1);
                sr = f2_fma(A, V0, sr);
                sg = f2_fma(A, V1, sg);
                sb = f2_fma(A, V2, sb);
                // -v_sigma per pixel
                const f2 WV = f2_mul(A, f2_fma(CB, V2, f2_fma(CG, V1, f2_mul(CR, V0))));
                wc = f2_add(wc, WV);
                const f2 TY = f2_mul(WV, DY[r]);
                yc = f2_add(yc, TY);
                syy = f2_fma(TY, DY[r], syy);
                if constexpr (ABS) {
                    float gx0, gx1, gy0, gy1;
                    f2_unpack(f2_mul(WV, f2_fma(BB, DY[r], AX)), gx0, gx1);
                    f2_unpack(f2_mul(WV, f2_fma(CC, DY[r], BDX)), gy0, gy1);
                    ax += fabsf(gx0) + fabsf(gx1);
                    ay += fabsf(gy0) + fabsf(gy1);
                }
            }
            const f2 TX = f2_mul(wc, DX);
            sx = f2_add(sx, TX);
            sxx = f2_fma(TX, DX, sxx);
            sy = f2_add(sy, yc);
            sxy = f2_fma(yc, DX, sxy);
        }
    }
    acc[0] -= f2_sum(sx); acc[1] -= f2_sum(sy);
    acc[4] -= f2_sum(sxx); acc[5] -= f2_sum(sxy); acc[6] -= f2_sum(syy);
    acc[7] += f2_sum(sr); acc[8] += f2_sum(sg); acc[9] += f2_sum(sb);
    if constexpr (ABS) {
        acc[2] += ax;
        acc[3] += ay;
    }
}

#ifndef LIG_RASTER_BWD_BULK
#define LIG_RASTER_BWD_BULK 1  // lean backward (float): records staged by bulk async copies
#endif
// Bounded device waits that gave up (a malfunction; read by lig_wait_timeouts).
__device__ unsigned int g_wait_timeouts;
// SM clock cycles (about 1 ms) before an mbarrier wait is abandoned: a
// normal wait ends within microseconds, and a malfunction then costs a
// launch at most about a millisecond per wave of CTAs instead of a hang.
constexpr long long kWaitCycles = 2000000;

// Bulk asynchronous copies of gathered 48-byte records into shared memory,
// completing on one mbarrier per CTA (cp.async.bulk, this GPU's memory only,
// no multicast).  Thread 0 announces the batch's bytes; each thread < cnt
// copies its record.  The transaction count may be completed before it is
// announced (its range includes negative values), so no barrier is needed
// between the two.
__device__ __forceinline__ void bulk_records(uint32_t bar, Rec<float> *s_rec, int32_t *s_ids,
                                             const int32_t *__restrict__ ids,
                                             const Rec<float> *__restrict__ recs, int base,
                                             int cnt) {
    const int tid = threadIdx.x;
    if (tid == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(cnt * (int)sizeof(Rec<float>))
                     : "memory");
    if (tid < cnt) {
        const int id = __ldg(ids + base + tid);
        s_ids[tid] = id;
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(s_rec + tid);
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(dst),
            "l"(recs + id), "r"((int)sizeof(Rec<float>)), "r"(bar)
            : "memory");
    }
}

// Wait for the mbarrier's phase `phase` for at most kWaitCycles.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    uint32_t done = 0;
    const long long t0 = clock64();
    for (;;) {
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
            "selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done || clock64() - t0 > kWaitCycles) break;
    }
    return done != 0;
}

// LEAN (sum backward of the fused fit loss, no opacities, no wsum
// cotangent): only the gradients the fit needs — v_xy, v_conic, v_rgb — are
// accumulated (no |v_xy| sums, no opacity gradient) and each (Gaussian,
// region) pair adds them with two 16-byte atomics into an [N][8] buffer.
// RR (float pair walk only): region rows, 4 (8x4 regions, eight warps per
// 16x16 tile), 8 (8x8, four warps, each thread staging two pixels) or 16
// (8x16, two warps, four pixels a thread); a lane group walks a taller region
// in blocks of four rows.
// Against 8x4 regions a Gaussian meets fewer regions, so the per-pair costs —
// the warps' region tests, the per-round set-up, the lane-group reduction and
// the atomics — are paid fewer times, for more pixel evaluations per pair.
template <typename T, bool GA, bool LEAN, bool ABS = false, int RR = 4>
__device__ __forceinline__ void bwd_tile(const TileCtx &tc, int tile,
                                         const int32_t *__restrict__ ids,
                                         const int2 *__restrict__ tile_bins,
                                         const Rec<T> *__restrict__ recs,
                                         const int32_t *__restrict__ final_idx, CotSrc<T> cot,
                                         const T *__restrict__ v_dx, const T *__restrict__ v_dy,
                                         const T *__restrict__ v_dxy, T clamp,
                                         T *__restrict__ packed, int &s_end, uint32_t bar,
                                         uint32_t &phase) {
    using M = Math<T>;
    // float lean backward: pixel pairs in f32x2 arithmetic (lean_region_f2)
    constexpr bool kPairs = LEAN && !GA && LIG_RASTER_BWD_F2 && sizeof(T) == 4;
    static_assert(!ABS || kPairs, "the |v_xy| sums of the lean walk need its pair form");
    // records staged by bulk async copies (no register prefetch, no region
    // masks: the warps test the box and ellipse themselves)
    constexpr bool kBulk = kPairs && LIG_RASTER_BWD_BULK;
    static_assert(RR == 4 || kPairs, "taller regions are walked by the pair form only");
    static_assert(RR == 4 || RR == 8 || RR == 16, "region rows");
    constexpr int kRows = RR;  // pair entries per region: kRows * 4
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nt = blockDim.x;  // = 32 * regions: region-major pixel slots
    PixRec<T, GA> *s_pix = reinterpret_cast<PixRec<T, GA> *>(smem_raw);
    // (8x16 regions: two pixel slots a thread hold the pair entries)
    Rec<T> *s_rec = reinterpret_cast<Rec<T> *>(s_pix + nt * (RR == 16 ? 2 : 1));
    uint32_t *s_bits = reinterpret_cast<uint32_t *>(s_rec + nt);
    int32_t *s_ids = reinterpret_cast<int32_t *>(s_bits + nt);
    uint16_t *s_list = reinterpret_cast<uint16_t *>(s_ids + nt);
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tc.empty) return;  // gradients stay zero (rasterize.py:156-161)
    const int B = tc.B, H = tc.H, W = tc.W, tx0 = tc.tx0, ty0 = tc.ty0;
    // fused L2: mean over this image's 3HW values (a batch sums per-image means)
    if (!cot.v_img) cot.scale = (T)(2.0 / (3.0 * (double)H * (double)W));
    const Regions R = Regions::make(GA ? 2 : (RR == 8 ? 1 : RR == 16 ? 3 : 0), B);
    T rx0 = 0, rx1 = 0, ry0 = 0, ry1 = 0;  // this warp's region (tile-local centres)
    if (LIG_RASTER_BWD_LANE_ELLIPSE) R.rect<T>(w, rx0, rx1, ry0, ry1);
    uint16_t *my_list = s_list + w * nt;
    const PixRec<T, GA> *my_pix = s_pix + w * 32;

    const int2 range = tile_bins[tile];
    int end = range.y;
    Rec<T> pre;
    int pre_id = -1;
    if constexpr (kBulk) {
        // first batch in flight while the pixels are staged
        if (range.x < end)
            bulk_records(bar, reinterpret_cast<Rec<float> *>(s_rec), s_ids, ids,
                         reinterpret_cast<const Rec<float> *>(recs), range.x,
                         min(nt, end - range.x));
    } else if constexpr (LEAN) {
        // the lean walk has no final-index test (see lean_region), so the list
        // is not cut at the tile's last final index: the first batch's gather
        // is issued before the pixels are staged and no barrier precedes it
        if (range.x + tid < end) {
            pre_id = __ldg(ids + range.x + tid);
            pre = recs[pre_id];
        }
    }
    // stage this thread's pixel (region w, slot lane)
    if (!LEAN && tid == 0) s_end = -1;
    if constexpr (RR > 4) {
        // pixels (x, y + 4 p2) of region w; pair entries as below with RR rows
        // per region
#pragma unroll
        for (int p2 = 0; p2 < RR / 4; ++p2) {
            int lx, ly;
            R.pixel(w, lane, p2, lx, ly);
            const int gx = tx0 + lx, gy = ty0 + ly;
            const bool inside = lx < B && ly < B && gx < W && gy < H;
            T v0 = (T)0, v1 = (T)0, v2 = (T)0, vw;
            if (inside) cot.get(tc.poff + gy * W + gx, v0, v1, v2, vw);
            PixPair *e = reinterpret_cast<PixPair *>(smem_raw) + w * RR * 4 +
                         ((lane >> 3) + 4 * p2) * 4 + (lane & 3);
            const int h = (lane >> 2) & 1;
            e->v[h] = v0;
            e->v[2 + h] = v1;
            e->v[4 + h] = v2;
        }
    } else {
        int lx, ly;
        R.pixel(w, lane, 0, lx, ly);
        const int gx = tx0 + lx, gy = ty0 + ly;
        const bool inside = lx < B && ly < B && gx < W && gy < H;
        const int p = inside ? tc.poff + gy * W + gx : 0;
        PixRec<T, GA> c;
        c.px = (T)gx + (T)0.5;
        c.py = (T)gy + (T)0.5;
        c.vo0 = c.vo1 = c.vo2 = c.vw = (T)0;
        if (inside) cot.get(p, c.vo0, c.vo1, c.vo2, c.vw);
        c.fin = (!LEAN && inside) ? final_idx[p] : -1;  // -1: never valid (unread when lean)
        if constexpr (GA) {
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                c.vd[ch] = inside ? v_dx[3 * p + ch] : (T)0;
                c.vd[3 + ch] = inside ? v_dy[3 * p + ch] : (T)0;
                c.vd[6 + ch] = inside ? v_dxy[3 * p + ch] : (T)0;
            }
        }
        if constexpr (kPairs) {
            // region w's pair entries: (row, column) -> entry row * 4 + col % 4,
            // half col / 4 (the pixel slots are row-major 8x4, kind 0)
            PixPair *e = reinterpret_cast<PixPair *>(smem_raw) + w * 16 + (lane >> 3) * 4 +
                         (lane & 3);
            const int h = (lane >> 2) & 1;
            e->v[h] = c.vo0;
            e->v[2 + h] = c.vo1;
            e->v[4 + h] = c.vo2;
        } else {
            s_pix[tid] = c;
        }
        if constexpr (!LEAN) {
            int my_max = c.fin;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1)
                my_max = max(my_max, __shfl_xor_sync(FULL, my_max, o));
            __syncthreads();
            if (lane == 0) atomicMax(&s_end, my_max);
        }
    }
    if constexpr (!LEAN) {
        __syncthreads();
        end = min(range.y, s_end + 1);
        if (range.x + tid < end) {
            pre_id = __ldg(ids + range.x + tid);
            pre = recs[pre_id];
        }
    }
    for (int base = range.x; base < end; base += nt) {
        const int cnt = min(nt, end - base);
        if constexpr (kBulk) {
            if (base != range.x) {  // everyone is done with the previous batch
                __syncthreads();
                bulk_records(bar, reinterpret_cast<Rec<float> *>(s_rec), s_ids, ids,
                             reinterpret_cast<const Rec<float> *>(recs), base, cnt);
            }
            const bool ok = mbar_wait(bar, phase);
            phase ^= 1u;
            // all threads agree: a wait that gave up counts once, then every
            // thread lets its copies drain (bounded) and the tile is abandoned
            if (__syncthreads_or(!ok)) {
                if (tid == 0) atomicAdd(&g_wait_timeouts, 1u);
                (void)mbar_wait(bar, phase ^ 1u);
                return;
            }
        } else {
            __syncthreads();
            if (tid < cnt) {
                s_rec[tid] = pre;
                s_bits[tid] = region_bits<T, !LIG_RASTER_BWD_LANE_ELLIPSE>(pre, R, tx0, ty0);
                s_ids[tid] = pre_id;
            }
            __syncthreads();
            if (base + nt + tid < end) {
                pre_id = __ldg(ids + base + nt + tid);
                pre = recs[pre_id];
            }
        }
        // compact the batch slots touching this region (ascending)
        int nmine = 0;
        for (int m = 0; m * 32 < cnt; ++m) {
            const int t = m * 32 + lane;
            bool hit;
            if constexpr (kBulk) hit = t < cnt && region_hit<T, false, false>(s_rec[t], R, w, tx0, ty0);
            else hit = t < cnt && ((s_bits[t] >> w) & 1u);
            if (LIG_RASTER_BWD_LANE_ELLIPSE && hit) {
                // exact ellipse test of Gaussian t against this warp's region,
                // one Gaussian per lane (the staging only tested the box)
                const Rec<T> &g = s_rec[t];
                if (g.wx >= (T)0) {
                    const T cx = g.x - (T)tx0, cy = g.y - (T)ty0;
                    hit = !(sigma_min_rect<T>(g.a, g.b, g.c, rx0 - cx, rx1 - cx, ry0 - cy,
                                              ry1 - cy) > g.thr);
                }
            }
            const uint32_t mask = __ballot_sync(FULL, hit);
            if (hit) my_list[nmine + __popc(mask & ((1u << lane) - 1u))] = (uint16_t)t;
            nmine += __popc(mask);
        }
        __syncwarp();
        for (int g0 = 0, lsplit = 0; g0 < nmine; g0 += 32 >> lsplit) {
            // lanes per Gaussian: with at most LIG_RASTER_BWD_SPLIT3 / SPLIT2 /
            // SPLIT1 Gaussians left, 8 / 4 / 2 lanes share one Gaussian (a round
            // then takes 4 / 8 / 16 of them), lane part p taking pixels
            // p, p + 2^lsplit, ... of the region (interleaved, so the group's
            // pixel records sit in different shared-memory banks); their
            // sums are combined below
            const int left = min(32, nmine - g0);
            // (the 8x16 walk: its own first and last thresholds, 64-pixel
            // regions favour more lanes per Gaussian)
            constexpr int kS1 = RR == 16 ? LIG_RASTER_BWD_R16_SPLIT1 : LIG_RASTER_BWD_SPLIT1;
            constexpr int kS3 = RR == 16 ? LIG_RASTER_BWD_R16_SPLIT3 : LIG_RASTER_BWD_SPLIT3;
            lsplit = !LIG_RASTER_BWD_SPLIT             ? 0
                     : left <= kS3                     ? 3
                     : left <= LIG_RASTER_BWD_SPLIT2   ? 2
                     : left <= kS1                     ? 1 : 0;
            const int gi = lane >> lsplit, part = lane & ((1 << lsplit) - 1);
            const int jstep = 1 << lsplit;
            const int slot = gi < left ? (int)my_list[g0 + gi] : -1;
            const bool act = slot >= 0;
            const Rec<T> g = s_rec[act ? slot : 0];
            const int k = act ? base + slot : 0x7fffffff;
            T acc[11];
#pragma unroll
            for (int q = 0; q < 11; ++q) acc[q] = 0;
            bool touched = false;
            if constexpr (kPairs) {
                // as below, two pixels per packed operation: lanes of a group
                // take column pairs (1 / 2 / 4 lanes) or column pairs and row
                // halves (8 lanes)
                touched = act;
                const float px0 = (float)(tx0 + (w % R.nbx) * 8) + 0.5f;
                const float py0 = (float)(ty0 + (w / R.nbx) * kRows) + 0.5f;
                const PixPair *pp = reinterpret_cast<const PixPair *>(smem_raw) + w * kRows * 4;
                if (act && RR > 4) {
                    // the region in blocks of four rows (8 lanes: one half each)
                    constexpr int NB = RR / 4;
                    switch (lsplit) {
                    case 0:
                        lean_region_f2<4, 1, 4, ABS, NB>(g, clamp, pp, 0, 0, px0, py0, acc);
                        break;
                    case 1:
                        lean_region_f2<2, 2, 4, ABS, NB>(g, clamp, pp, part, 0, px0, py0, acc);
                        break;
                    case 2:
                        lean_region_f2<1, 1, 4, ABS, NB>(g, clamp, pp, part, 0, px0, py0, acc);
                        break;
                    default:
                        lean_region_f2<1, 1, 4, ABS, NB / 2>(g, clamp, pp, part & 3,
                                                             (RR / 2) * (part >> 2), px0, py0,
                                                             acc);
                        break;
                    }
                } else if (act) {
                    switch (lsplit) {
                    case 0:
                        lean_region_f2<4, 1, 4, ABS>(g, clamp, pp, 0, 0, px0, py0, acc);
                        break;
                    case 1:
                        lean_region_f2<2, 2, 4, ABS>(g, clamp, pp, part, 0, px0, py0, acc);
                        break;
                    case 2:
                        lean_region_f2<1, 1, 4, ABS>(g, clamp, pp, part, 0, px0, py0, acc);
                        break;
                    default:
                        lean_region_f2<1, 1, 2, ABS>(g, clamp, pp, part & 3, 2 * (part >> 2),
                                                     px0, py0, acc);
                        break;
                    }
                }
            } else if constexpr (LEAN && !GA && LIG_RASTER_BWD_COLS) {
                // every listed (Gaussian, region) pair met the region's
                // ellipse test; an untouched one adds zeros
                touched = act;
                const T px0 = (T)(tx0 + (w % R.nbx) * 8 + part) + (T)0.5;
                const T py0 = (T)(ty0 + (w / R.nbx) * 4) + (T)0.5;
                if (act) {
                    switch (lsplit) {
                    case 0: lean_region<T, 0>(g, clamp, my_pix, part, px0, py0, acc); break;
                    case 1: lean_region<T, 1>(g, clamp, my_pix, part, px0, py0, acc); break;
                    case 2: lean_region<T, 2>(g, clamp, my_pix, part, px0, py0, acc); break;
                    default: lean_region<T, 3>(g, clamp, my_pix, part, px0, py0, acc); break;
                    }
                }
            } else {
            for (int j = part; j < 32; j += jstep) {
                const PixRec<T, GA> &c = my_pix[j];
                if (k > c.fin) continue;
                if constexpr (!GA) {
                    // csrc/backward.cu:102-150
                    const T dx = g.x - c.px;
                    const T dy = g.y - c.py;
                    const T sigma = sigma_ref<T>(g.a, g.b, g.c, dx, dy);
                    const T vis = M::exp_(-sigma);
                    const T alpha = M::min_(clamp, g.o * vis);
                    if (sigma < (T)0 || alpha < (T)1 / (T)255) continue;
                    touched = true;
                    T v_alpha = 0;
                    acc[7] += alpha * c.vo0;
                    acc[8] += alpha * c.vo1;
                    acc[9] += alpha * c.vo2;
                    v_alpha += g.r * c.vo0;
                    v_alpha += g.g * c.vo1;
                    v_alpha += g.bl * c.vo2;
                    if constexpr (!LEAN) {
                        v_alpha += c.vw;
                        acc[10] += vis * v_alpha;
                    }
                    const T v_sigma = -alpha * v_alpha;
                    if constexpr (LEAN) {
                        // the gradients are linear in five per-pixel sums
                        // (Sx, Sy, Sxx, Sxy, Syy of v_sigma dx^i dy^j); the
                        // conic is applied once per Gaussian after the loop
                        const T tx = v_sigma * dx, ty = v_sigma * dy;
                        acc[0] += tx;
                        acc[1] += ty;
                        acc[4] += tx * dx;
                        acc[5] += tx * dy;
                        acc[6] += ty * dy;
                    } else {
                        acc[4] += (T)0.5 * v_sigma * dx * dx;
                        acc[5] += v_sigma * dx * dy;
                        acc[6] += (T)0.5 * v_sigma * dy * dy;
                        const T gx = v_sigma * (g.a * dx + g.b * dy);
                        const T gy = v_sigma * (g.b * dx + g.c * dy);
                        acc[0] += gx;
                        acc[1] += gy;
                        acc[2] += M::abs_(gx);
                        acc[3] += M::abs_(gy);
                    }
                } else {
                    // csrc/gradient_aware_rasterizer.cu:201-315
                    const T dx = c.px - g.x;
                    const T dy = c.py - g.y;
                    const T sigma = sigma_ref<T>(g.a, g.b, g.c, dx, dy);
                    const T vis = M::exp_(-sigma);
                    const T alpha = M::min_(clamp, g.o * vis);
                    if (sigma < (T)0 || alpha < (T)1 / (T)255) continue;
                    touched = true;
                    const T sx = g.a * dx + g.b * dy;
                    const T sy = g.b * dx + g.c * dy;
                    const T a = g.a, b = g.b, cc = g.c;
                    const T ax = -alpha * sx;
                    const T ay = -alpha * sy;
                    const T axy = alpha * (sx * sy - b);
                    const T vo[3] = {c.vo0, c.vo1, c.vo2};
                    const T *vdx = c.vd, *vdy = c.vd + 3, *vdxy = c.vd + 6;
                    acc[7] += vo[0] * alpha + vdx[0] * ax + vdy[0] * ay + vdxy[0] * axy;
                    acc[8] += vo[1] * alpha + vdx[1] * ax + vdy[1] * ay + vdxy[1] * axy;
                    acc[9] += vo[2] * alpha + vdx[2] * ax + vdy[2] * ay + vdxy[2] * axy;
                    const T va = (vo[0] * g.r + vo[1] * g.g + vo[2] * g.bl) + c.vw;
                    const T vax = vdx[0] * g.r + vdx[1] * g.g + vdx[2] * g.bl;
                    const T vay = vdy[0] * g.r + vdy[1] * g.g + vdy[2] * g.bl;
                    const T vaxy = vdxy[0] * g.r + vdxy[1] * g.g + vdxy[2] * g.bl;
                    const T sx2 = sx * sx, sy2 = sy * sy, sxsy = sx * sy;
                    acc[0] += alpha * (va * sx + vax * (a - sx2) + vay * (b - sxsy) +
                                       vaxy * (sx2 * sy - (T)2 * b * sx - a * sy));
                    acc[1] += alpha * (va * sy + vax * (b - sxsy) + vay * (cc - sy2) +
                                       vaxy * (sx * sy2 - (T)2 * b * sy - cc * sx));
                    const T dx2 = dx * dx, dy2 = dy * dy, dxdy = dx * dy;
                    const T P = sxsy - b;
                    acc[4] += alpha * (va * (-(T)0.5 * dx2) + vax * ((T)0.5 * dx2 * sx - dx) +
                                       vay * ((T)0.5 * dx2 * sy) +
                                       vaxy * (-(T)0.5 * dx2 * P + dx * sy));
                    acc[5] += alpha * (va * (-dxdy) + vax * (dxdy * sx - dy) +
                                       vay * (dxdy * sy - dx) +
                                       vaxy * (-dxdy * P + dy * sy + dx * sx - (T)1));
                    acc[6] += alpha * (va * (-(T)0.5 * dy2) + vax * ((T)0.5 * dy2 * sx) +
                                       vay * ((T)0.5 * dy2 * sy - dy) +
                                       vaxy * (-(T)0.5 * dy2 * P + dy * sx));
                    acc[10] += vis * va;
                }
            }
            }
            for (int o = 1; o < (1 << lsplit); o <<= 1) {  // combine the lane group
#pragma unroll
                for (int q = 0; q < 11; ++q) {
                    if (LEAN && (q == 10 || (!ABS && (q == 2 || q == 3)))) continue;
                    acc[q] += __shfl_xor_sync(FULL, acc[q], o);
                }
                touched = __shfl_xor_sync(FULL, (int)touched, o) || touched;
            }
            if (touched && part == 0) {
                if constexpr (LEAN && !GA) {
                    // v_xy = (a Sx + b Sy, b Sx + c Sy); v_conic = (Sxx/2, Sxy, Syy/2)
                    const T sx = acc[0], sy = acc[1];
                    acc[0] = g.a * sx + g.b * sy;
                    acc[1] = g.b * sx + g.c * sy;
                    acc[4] *= (T)0.5;
                    acc[6] *= (T)0.5;
                }
                if (GA) {  // |sum over the reference warp| (= this region)
                    acc[2] = M::abs_(acc[0]);
                    acc[3] = M::abs_(acc[1]);
                }
                if constexpr (LEAN && ABS) {
                    // the general [N][12] layout, no opacity gradient
                    float4 *d4 = reinterpret_cast<float4 *>(packed + (size_t)s_ids[slot] * 12);
                    atomicAdd(d4, make_float4(acc[0], acc[1], acc[2], acc[3]));
                    atomicAdd(d4 + 1, make_float4(acc[4], acc[5], acc[6], acc[7]));
                    atomicAdd(d4 + 2, make_float4(acc[8], acc[9], 0.f, 0.f));
                } else if constexpr (LEAN) {
                    // [xy, conic, rgb]
                    T *dst = packed + (size_t)s_ids[slot] * 8;
                    if constexpr (sizeof(T) == 4) {
                        float4 *d4 = reinterpret_cast<float4 *>(dst);
                        atomicAdd(d4, make_float4(acc[0], acc[1], acc[4], acc[5]));
                        atomicAdd(d4 + 1, make_float4(acc[6], acc[7], acc[8], acc[9]));
                    } else {
                        const T v[8] = {acc[0], acc[1], acc[4], acc[5],
                                        acc[6], acc[7], acc[8], acc[9]};
#pragma unroll
                        for (int q = 0; q < 8; ++q) atomicAdd(dst + q, v[q]);
                    }
                } else {
                    T *dst = packed + (size_t)s_ids[slot] * 12;
                    if constexpr (sizeof(T) == 4) {
                        float4 *d4 = reinterpret_cast<float4 *>(dst);
                        atomicAdd(d4, make_float4(acc[0], acc[1], acc[2], acc[3]));
                        atomicAdd(d4 + 1, make_float4(acc[4], acc[5], acc[6], acc[7]));
                        atomicAdd(d4 + 2, make_float4(acc[8], acc[9], acc[10], 0.f));
                    } else {
#pragma unroll
                        for (int q = 0; q < 11; ++q) atomicAdd(dst + q, acc[q]);
                    }
                }
            }
        }
    }
}

template <typename T, bool GA, bool LEAN, int MAXT, int MINB, bool ABS = false, int RR = 4>
__global__ void __launch_bounds__(MAXT, MINB)
raster_bwd_kernel(const BatchGeo geo, const int32_t *__restrict__ cum, int *work,
                  const int32_t *__restrict__ ids, const int2 *__restrict__ tile_bins,
                  const int32_t *__restrict__ d_total, const Rec<T> *__restrict__ recs,
                  const int32_t *__restrict__ final_idx, CotSrc<T> cot,
                  const T *__restrict__ v_dx, const T *__restrict__ v_dy,
                  const T *__restrict__ v_dxy, T clamp, T *__restrict__ packed) {
    __shared__ int s_end, s_slot;
    __shared__ __align__(8) unsigned long long s_mbar;
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&s_mbar);
    uint32_t phase = 0;
    if (LIG_RASTER_BWD_BULK && LEAN && !GA && sizeof(T) == 4) {
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
            asm volatile("fence.mbarrier_init.release.cluster;");
        }
        __syncthreads();
    }
    const int n_tiles = geo.total_tiles();
    for (int tile = next_tile(work, s_slot, true); tile < n_tiles;
         tile = next_tile(work, s_slot, false)) {
        const TileCtx tc = tile_ctx(geo, cum, d_total, tile);
        bwd_tile<T, GA, LEAN, ABS, RR>(tc, tile, ids, tile_bins, recs, final_idx, cot, v_dx, v_dy,
                                   v_dxy, clamp, packed, s_end, bar, phase);
    }
}

// Packed per-Gaussian gradients [N][12] -> the five output arrays of the ABI.
template <typename T>
__global__ void unpack_lean_grads_kernel(int n, const T *__restrict__ packed, Grads<T> out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T *g = packed + (size_t)i * 8;
    out.v_xy[2 * i] = g[0];
    out.v_xy[2 * i + 1] = g[1];
    out.v_abs[2 * i] = 0;
    out.v_abs[2 * i + 1] = 0;
    out.v_conic[3 * i] = g[2];
    out.v_conic[3 * i + 1] = g[3];
    out.v_conic[3 * i + 2] = g[4];
    out.v_rgb[3 * i] = g[5];
    out.v_rgb[3 * i + 1] = g[6];
    out.v_rgb[3 * i + 2] = g[7];
}

template <typename T>
__global__ void unpack_grads_kernel(int n, const T *__restrict__ packed, Grads<T> out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T *g = packed + (size_t)i * 12;
    out.v_xy[2 * i] = g[0];
    out.v_xy[2 * i + 1] = g[1];
    out.v_abs[2 * i] = g[2];
    out.v_abs[2 * i + 1] = g[3];
    out.v_conic[3 * i] = g[4];
    out.v_conic[3 * i + 1] = g[5];
    out.v_conic[3 * i + 2] = g[6];
    out.v_rgb[3 * i] = g[7];
    out.v_rgb[3 * i + 1] = g[8];
    out.v_rgb[3 * i + 2] = g[9];
    if (out.v_opac) out.v_opac[i] = g[10];
}

// ------------------------------------------------------------------ host
template <typename T>
int pack(int n, const void *xys, const void *con, const void *col, const void *op, void *ws,
         size_t ws_bytes, cudaStream_t s, bool half = false, T *zero = nullptr,
         int zero_stride = 0) {
    if (ws_bytes < sizeof(Rec<T>) * (size_t)n) return LIG_ERR_WORKSPACE;
    if ((reinterpret_cast<uintptr_t>(ws) & 15) != 0) return LIG_ERR_INVALID;  // 16-byte records
    if (n > 0) {
        auto k = half ? pack_kernel<T, true> : pack_kernel<T, false>;
        k<<<(n + 255) / 256, 256, 0, s>>>(n, (const T *)xys, (const T *)con, (const T *)col,
                                          (const T *)op, (Rec<T> *)ws, zero, zero_stride);
    }
    note_launches(n > 0 ? 1 : 0);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

// Opt a kernel into `bytes` of dynamic shared memory, once per (kernel,
// device, size): repeated calls cost nothing, and none is made during a
// stream capture after the first eager call.
#ifndef LIG_RASTER_CARVEOUT
#define LIG_RASTER_CARVEOUT -1  // shared-memory carveout percent; -1: driver default
#endif

inline bool set_dyn_smem(const void *fn, size_t bytes) {
    if (bytes <= 48 * 1024 && LIG_RASTER_CARVEOUT < 0) return true;
    static std::mutex mu;
    static std::vector<std::tuple<const void *, int, size_t>> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    std::lock_guard<std::mutex> lock(mu);
    for (auto &e : done)
        if (std::get<0>(e) == fn && std::get<1>(e) == dev && std::get<2>(e) >= bytes) return true;
    if (bytes > 48 * 1024 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
            cudaSuccess)
        return false;
    if (LIG_RASTER_CARVEOUT >= 0 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                             LIG_RASTER_CARVEOUT) != cudaSuccess)
        return false;
    done.emplace_back(fn, dev, bytes);
    return true;
}

// Grid of a persistent launch: every CTA that fits on the device at once.
inline int persistent_grid(const void *fn, int threads, size_t smem) {
    static std::mutex mu;
    static std::vector<std::tuple<const void *, int, int, size_t, int>> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    std::lock_guard<std::mutex> lock(mu);
    for (auto &e : cache)
        if (std::get<0>(e) == fn && std::get<1>(e) == dev && std::get<2>(e) == threads &&
            std::get<3>(e) == smem)
            return std::get<4>(e);
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    const int g = per_sm * sms;
    cache.emplace_back(fn, dev, threads, smem, g);
    return g;
}

// How a raster kernel walks the flattened (image, tile) list.
struct TileWalk {
    const int32_t *cum = nullptr;  // per-image empty test (batched); null: *d_total
    int *work = nullptr;           // persistent: global work counter; null: CTA per tile
};

// Loss outputs of the fused-L2 forward (with a target).
template <typename T> struct L2Out {
    T *loss = nullptr, *per_image = nullptr;
};

template <typename T>
int raster_fwd(const BatchGeo &geo, TileWalk walk, const int32_t *ids, const int32_t *bins,
               const int32_t *d_total, const void *xys, const void *con, const void *col,
               const void *op, void *ws, size_t ws_bytes, void *img, void *wsum, void *dx,
               void *dy, void *dxy, int32_t *fin, cudaStream_t s,
               L2Fwd<T> l2 = L2Fwd<T>{nullptr, nullptr}, L2Out<T> l2o = L2Out<T>{}) {
    const int n = geo.total_points();
    const bool ga = dx != nullptr;
    // fused loss without opacities: the specialised forward (halved conic)
    const bool fl = !ga && (l2.target || l2.target_u8) && !op && LIG_RASTER_FWD_FUSED;
    int rc = pack<T>(n, xys, con, col, op, ws, ws_bytes, s, fl);
    if (rc) return rc;
    const bool ppl4 = !ga && geo.total_tiles() >= LIG_RASTER_PPL4_MIN_TILES;
    const bool ppl2 = !ga && !ppl4 && geo.total_tiles() >= LIG_RASTER_PPL2_MIN_TILES;
    const int nt = 32 * Regions::make(ppl4 ? 3 : (ppl2 ? 1 : 0), geo.B).count;
    const size_t sm = (size_t)nt * (sizeof(Rec<T>) + sizeof(uint32_t));
    using K = void (*)(const BatchGeo, const int32_t *, int *, const int32_t *, const int2 *,
                       const int32_t *, const Rec<T> *, T *, T *, T *, T *, T *, int32_t *,
                       L2Fwd<T>);
    const bool small = nt <= 256;
    constexpr int FM = LIG_RASTER_FWD_MINB;
    K fn = ga ? (small ? raster_fwd_kernel<T, true, 1, 256, FM>
                       : raster_fwd_kernel<T, true, 1, 1024, 1>)
         : fl && fin ? (ppl4 ? (small ? raster_fwd_kernel<T, false, 4, 256, FM, true>
                                      : raster_fwd_kernel<T, false, 4, 1024, 1, true>)
                        : ppl2 ? (small ? raster_fwd_kernel<T, false, 2, 256, FM, true>
                                        : raster_fwd_kernel<T, false, 2, 1024, 1, true>)
                               : (small ? raster_fwd_kernel<T, false, 1, 256, FM, true>
                                        : raster_fwd_kernel<T, false, 1, 1024, 1, true>))
         : fl ? (ppl4 ? (small ? raster_fwd_kernel<T, false, 4, 256, FM, true, false>
                               : raster_fwd_kernel<T, false, 4, 1024, 1, true, false>)
                 : ppl2 ? (small ? raster_fwd_kernel<T, false, 2, 256, FM, true, false>
                                 : raster_fwd_kernel<T, false, 2, 1024, 1, true, false>)
                        : (small ? raster_fwd_kernel<T, false, 1, 256, FM, true, false>
                                 : raster_fwd_kernel<T, false, 1, 1024, 1, true, false>))
              : ppl4 ? (small ? raster_fwd_kernel<T, false, 4, 256, LIG_RASTER_FWD_MINB>
                              : raster_fwd_kernel<T, false, 4, 1024, 1>)
              : ppl2 ? (small ? raster_fwd_kernel<T, false, 2, 256, LIG_RASTER_FWD_MINB>
                              : raster_fwd_kernel<T, false, 2, 1024, 1>)
                     : (small ? raster_fwd_kernel<T, false, 1, 256, LIG_RASTER_FWD_MINB>
                              : raster_fwd_kernel<T, false, 1, 1024, 1>);
    if (!set_dyn_smem((const void *)fn, sm)) return LIG_ERR_LAUNCH;
    int grid = geo.total_tiles();
    if (walk.work) {
        const int pg = persistent_grid((const void *)fn, nt, sm);
        if (pg <= 0) return LIG_ERR_LAUNCH;
        grid = grid < pg ? grid : pg;
        cudaMemsetAsync(walk.work, 0, sizeof(int), s);
    }
    fn<<<grid, nt, sm, s>>>(geo, walk.cum, walk.work, ids, (const int2 *)bins, d_total,
                            (const Rec<T> *)ws, (T *)img, (T *)wsum, ga ? (T *)dx : nullptr,
                            ga ? (T *)dy : nullptr, ga ? (T *)dxy : nullptr, fin, l2);
    int launches = 1;
    if (l2.target || l2.target_u8) {
        const TileChunks ch = tile_chunks(geo);
        double *chunk_sum = l2.tile_partial + geo.total_tiles();
        if (ch.chunk_off[geo.n_img] > 0)
            l2_tiles_chunk_kernel<<<ch.chunk_off[geo.n_img], 256, 0, s>>>(geo, ch, l2.tile_partial,
                                                                         chunk_sum);
        l2_chunks_final_kernel<T><<<1, 1024, 0, s>>>(geo, ch, chunk_sum, l2o.loss, l2o.per_image);
        launches += 2;
    }
    note_launches(launches);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

// Backward workspace: packed records [N] followed by packed gradients [N][12].
template <typename T>
inline size_t bwd_grad_offset(int n) {
    return (sizeof(Rec<T>) * (size_t)(n > 0 ? n : 1) + 255) & ~(size_t)255;
}

template <typename T>
int raster_bwd(const BatchGeo &geo, TileWalk walk, const int32_t *ids, const int32_t *bins,
               const int32_t *d_total, const void *xys, const void *con, const void *col,
               const void *op, const int32_t *fin, CotSrc<T> cot, const void *v_dx,
               const void *v_dy, const void *v_dxy, double clamp, void *ws, size_t ws_bytes,
               void *v_xy, void *v_abs, void *v_con, void *v_rgb, void *v_op, cudaStream_t s) {
    const int n = geo.total_points();
    const size_t goff = bwd_grad_offset<T>(n);
    if (ws_bytes < goff + sizeof(T) * 12 * (size_t)n) return LIG_ERR_WORKSPACE;
    const bool ga = v_dx != nullptr;
    // the fused-loss backward without opacities needs neither |v_xy| nor an
    // opacity gradient (nor a wsum cotangent)
    const bool lean = !ga && !cot.v_img && !cot.v_wsum && !op && !v_op;
    // an explicit image cotangent without wsum cotangent or opacities (the
    // drop-in API under autograd, LIG's own training loop): the same lean
    // walk plus the per-pixel |v_xy| sums the reference returns (float)
    const bool lean_abs = !ga && cot.v_img && !cot.v_wsum && !op && !v_op &&
                          sizeof(T) == 4 && LIG_RASTER_BWD_F2;
    const int stride = lean ? 8 : 12;
    T *packed = reinterpret_cast<T *>((char *)ws + goff);
    // records, and the packed gradients cleared in the same pass
    int rc = pack<T>(n, xys, con, col, op, ws, goff, s, false, packed, stride);
    if (rc) return rc;
    const T cl = (T)(clamp > 0 ? clamp : (ga ? 0.999 : 0.99));
    const bool large = geo.total_tiles() >= LIG_RASTER_BWD_LARGE_MIN_TILES;
    // the float lean walks of large images: 8x8 regions (tiles up to 16x16)
    const double density = (double)n / (double)geo.total_pixels();
    const int rr_auto = density <= LIG_RASTER_BWD_R16_MAX_DENSITY ? 16 : 8;
    const int rr = (LIG_RASTER_BWD_RROWS != 4 && sizeof(T) == 4 && LIG_RASTER_BWD_F2 &&
                    (lean || lean_abs) && large && geo.B <= 16)
                       ? (LIG_RASTER_BWD_RROWS ? LIG_RASTER_BWD_RROWS : rr_auto)
                       : 4;
    const int nt = 32 * Regions::make(ga ? 2 : (rr == 8 ? 1 : rr == 16 ? 3 : 0), geo.B).count;
    const int nw = nt / 32;
    const size_t pix = ga ? sizeof(PixRec<T, true>) : sizeof(PixRec<T, false>) * (rr == 16 ? 2 : 1);
    const size_t sm = (size_t)nt * pix + (size_t)nt * (sizeof(Rec<T>) + 2 * sizeof(uint32_t)) +
                      (size_t)nw * nt * sizeof(uint16_t);
    using K = void (*)(const BatchGeo, const int32_t *, int *, const int32_t *, const int2 *,
                       const int32_t *, const Rec<T> *, const int32_t *, CotSrc<T>, const T *,
                       const T *, const T *, T, T *);
    const bool small = nt <= 256;
    constexpr bool kAbs = sizeof(T) == 4 && LIG_RASTER_BWD_F2;
    K fn = ga ? (small ? raster_bwd_kernel<T, true, false, 256, LIG_RASTER_BWD_MINB>
                       : raster_bwd_kernel<T, true, false, 1024, 1>)
         : lean_abs ? (small ? (large ? raster_bwd_kernel<T, false, true, 256,
                                                          LIG_RASTER_BWD_LEAN_MINB_LARGE, kAbs>
                                      : raster_bwd_kernel<T, false, true, 256,
                                                          LIG_RASTER_BWD_LEAN_MINB, kAbs>)
                             : raster_bwd_kernel<T, false, true, 1024, 1, kAbs>)
              : lean ? (small ? (geo.total_tiles() >= LIG_RASTER_BWD_LARGE_MIN_TILES
                                     ? raster_bwd_kernel<T, false, true, 256,
                                                         LIG_RASTER_BWD_LEAN_MINB_LARGE>
                                     : raster_bwd_kernel<T, false, true, 256,
                                                         LIG_RASTER_BWD_LEAN_MINB>)
                              : raster_bwd_kernel<T, false, true, 1024, 1>)
                     : (small ? raster_bwd_kernel<T, false, false, 256, LIG_RASTER_BWD_MINB>
                              : raster_bwd_kernel<T, false, false, 1024, 1>);
    if constexpr (kAbs) {
        if (rr == 8)
            fn = lean_abs ? raster_bwd_kernel<T, false, true, 128, LIG_RASTER_BWD_RROWS_MINB, true, 8>
                          : raster_bwd_kernel<T, false, true, 128, LIG_RASTER_BWD_RROWS_MINB, false,
                                              8>;
        else if (rr == 16)
            fn = lean_abs ? raster_bwd_kernel<T, false, true, 64, LIG_RASTER_BWD_R16_MINB, true, 16>
                          : raster_bwd_kernel<T, false, true, 64, LIG_RASTER_BWD_R16_MINB, false,
                                              16>;
    }
    if (!set_dyn_smem((const void *)fn, sm)) return LIG_ERR_LAUNCH;
    int grid = geo.total_tiles();
    if (walk.work) {
        const int pg = persistent_grid((const void *)fn, nt, sm);
        if (pg <= 0) return LIG_ERR_LAUNCH;
        grid = grid < pg ? grid : pg;
        cudaMemsetAsync(walk.work, 0, sizeof(int), s);
    }
    fn<<<grid, nt, sm, s>>>(geo, walk.cum, walk.work, ids, (const int2 *)bins, d_total,
                            (const Rec<T> *)ws, fin, cot, ga ? (const T *)v_dx : nullptr,
                            ga ? (const T *)v_dy : nullptr, ga ? (const T *)v_dxy : nullptr, cl,
                            packed);
    Grads<T> g{(T *)v_xy, (T *)v_abs, (T *)v_con, (T *)v_rgb, (T *)v_op};
    if (n > 0 && lean) unpack_lean_grads_kernel<T><<<(n + 255) / 256, 256, 0, s>>>(n, packed, g);
    else if (n > 0) unpack_grads_kernel<T><<<(n + 255) / 256, 256, 0, s>>>(n, packed, g);
    note_launches(n > 0 ? 2 : 1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

inline bool raster_args_ok(int H, int W, int B, int n) {
    // pixel-channel indices are 32-bit
    return H > 0 && W > 0 && B >= 2 && B <= 32 && n >= 0 &&
           3ll * H * W <= 0x7fffffffll;
}

}  // namespace lig

using namespace lig;

extern "C" size_t lig_raster_workspace_bytes(int dtype, int n) {
    size_t m = (size_t)(n > 0 ? n : 1);
    if (dtype == LIG_F64) return bwd_grad_offset<double>(n) + sizeof(double) * 12 * m;
    return bwd_grad_offset<float>(n) + sizeof(float) * 12 * m;
}

extern "C" int lig_raster_fwd(int dtype, int H, int W, int B, int n, const int32_t *ids,
                              const int32_t *bins, const int32_t *d_total, const void *xys,
                              const void *con, const void *col, const void *op, void *ws,
                              size_t ws_bytes, void *img, void *wsum, void *dx, void *dy,
                              void *dxy, int32_t *fin, void *stream) {
    if (!raster_args_ok(H, W, B, n) || !bins || !d_total || !img || !wsum || !fin || !ws ||
        (n > 0 && (!xys || !con || !col)) || ((dx || dy || dxy) && !(dx && dy && dxy)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return raster_fwd<float>(BatchGeo::single(H, W, B, n), TileWalk{}, ids, bins, d_total,
                                 xys, con, col, op, ws, ws_bytes, img, wsum, dx, dy, dxy, fin, s);
    if (dtype == LIG_F64)
        return raster_fwd<double>(BatchGeo::single(H, W, B, n), TileWalk{}, ids, bins, d_total,
                                  xys, con, col, op, ws, ws_bytes, img, wsum, dx, dy, dxy, fin, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_bwd(int dtype, int H, int W, int B, int n, const int32_t *ids,
                              const int32_t *bins, const int32_t *d_total, const void *xys,
                              const void *con, const void *col, const void *op,
                              const int32_t *fin, const void *v_img, const void *v_wsum,
                              const void *v_dx, const void *v_dy, const void *v_dxy,
                              double clamp, void *ws, size_t ws_bytes, void *v_xy, void *v_abs,
                              void *v_con, void *v_rgb, void *v_op, void *stream) {
    if (!raster_args_ok(H, W, B, n) || !bins || !d_total || !fin || !v_img || !ws ||
        (n > 0 && (!xys || !con || !col || !v_xy || !v_abs || !v_con || !v_rgb)) ||
        ((v_dx || v_dy || v_dxy) && !(v_dx && v_dy && v_dxy)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) return LIG_OK;
    if (dtype == LIG_F32) {
        CotSrc<float> cot{(const float *)v_img, (const float *)v_wsum, nullptr, nullptr, nullptr, 0.f};
        return raster_bwd<float>(BatchGeo::single(H, W, B, n), TileWalk{}, ids, bins, d_total,
                                 xys, con, col, op, fin, cot,
                                 v_dx, v_dy, v_dxy, clamp, ws, ws_bytes, v_xy, v_abs, v_con,
                                 v_rgb, v_op, s);
    }
    if (dtype == LIG_F64) {
        CotSrc<double> cot{(const double *)v_img, (const double *)v_wsum, nullptr, nullptr, nullptr, 0.0};
        return raster_bwd<double>(BatchGeo::single(H, W, B, n), TileWalk{}, ids, bins, d_total,
                                  xys, con, col, op, fin, cot,
                                  v_dx, v_dy, v_dxy, clamp, ws, ws_bytes, v_xy, v_abs, v_con,
                                  v_rgb, v_op, s);
    }
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_bwd_l2(int dtype, int H, int W, int B, int n, const int32_t *ids,
                                 const int32_t *bins, const int32_t *d_total, const void *xys,
                                 const void *con, const void *col, const void *op,
                                 const int32_t *fin, const void *img, const void *target,
                                 const void *grad_loss, double clamp, void *ws, size_t ws_bytes,
                                 void *v_xy, void *v_abs, void *v_con, void *v_rgb, void *v_op,
                                 void *stream) {
    if (!raster_args_ok(H, W, B, n) || !bins || !d_total || !fin || !img || !target ||
        !grad_loss || !ws || (n > 0 && (!xys || !con || !col || !v_xy || !v_abs || !v_con || !v_rgb)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) return LIG_OK;
    const double scale = 2.0 / (3.0 * (double)H * (double)W);
    if (dtype == LIG_F32) {
        CotSrc<float> cot{nullptr, nullptr, (const float *)img, (const float *)target,
                          (const float *)grad_loss, (float)scale};
        return raster_bwd<float>(BatchGeo::single(H, W, B, n), TileWalk{}, ids, bins, d_total,
                                 xys, con, col, op, fin, cot,
                                 nullptr, nullptr, nullptr, clamp, ws, ws_bytes, v_xy, v_abs,
                                 v_con, v_rgb, v_op, s);
    }
    if (dtype == LIG_F64) {
        CotSrc<double> cot{nullptr, nullptr, (const double *)img, (const double *)target,
                           (const double *)grad_loss, scale};
        return raster_bwd<double>(BatchGeo::single(H, W, B, n), TileWalk{}, ids, bins, d_total,
                                  xys, con, col, op, fin, cot,
                                  nullptr, nullptr, nullptr, clamp, ws, ws_bytes, v_xy, v_abs,
                                  v_con, v_rgb, v_op, s);
    }
    return LIG_ERR_INVALID;
}

// Number of bounded device-side waits (mbarrier polls of the bulk-staged
// backward) that gave up on the current device since the library loaded;
// 0 unless a kernel malfunctioned.
extern "C" int lig_wait_timeouts(void) {
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_wait_timeouts, sizeof(v)) != cudaSuccess) return -1;
    return (int)v;
}

// ------------------------------------------------------ alpha cut check
namespace lig {
// out[0] = the warp search's cut; out[1] = first failing, out[2] = last
// passing bit pattern of the scan below (initial values for its atomics).
__global__ void alpha_cut_init_kernel(uint32_t *out) {
    const uint32_t cut = alpha_cut_search();
    if (threadIdx.x == 0) {
        out[0] = cut;
        out[1] = 0xffffffffu;
        out[2] = 0u;
    }
}

// The rasterizers' alpha decision at every non-negative float up to +inf
// (bit patterns 0 .. 0x7f800000): the decision is a step with its edge at the
// cut exactly when out[2] + 1 == out[1] == out[0].
__global__ void alpha_cut_scan_kernel(uint32_t *out) {
    constexpr uint32_t kLast = 0x7f800000u;
    uint32_t first_fail = 0xffffffffu, last_pass = 0u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u <= kLast; u += stride) {
        if (alpha_passes(__uint_as_float(u))) last_pass = max(last_pass, u);
        else first_fail = min(first_fail, u);
    }
    first_fail = __reduce_min_sync(0xffffffffu, first_fail);
    last_pass = __reduce_max_sync(0xffffffffu, last_pass);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(out + 1, first_fail);
        atomicMax(out + 2, last_pass);
    }
}
}  // namespace lig

// Writes the alpha cut and the full scan's step edges into out[0..2] (device
// memory, three uint32) on `stream`.
extern "C" int lig_alpha_cut(uint32_t *out, void *stream) {
    if (!out) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    alpha_cut_init_kernel<<<1, 32, 0, s>>>(out);
    alpha_cut_scan_kernel<<<148 * 8, 256, 0, s>>>(out);
    note_launches(2);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

// ----------------------------------------------------- allocation-free entry
// Some callers cannot allocate device memory at the time they render: a
// plugin inside a framework that has already reserved (nearly) all of the
// GPU's memory for its own pool, or a real-time loop whose host forbids
// driver allocations after start-up.  For them, the sum forward below takes
// its scratch (the packed per-Gaussian records) from a fixed array compiled
// into this library instead of a caller workspace.  Every GPU that loads the
// library keeps this array (LIG_STATIC_MAX_POINTS records, 6 MiB) until the
// process exits.
namespace lig {
__device__ __align__(256) unsigned char g_noalloc_scratch[(size_t)LIG_STATIC_MAX_POINTS *
                                                          sizeof(Rec<float>)];

// Device address of the scratch array, looked up once per device (host code
// cannot use the symbol itself: on the host it names a stand-in, not device
// memory).  The first call on a device does the lookup.  A device reset by
// the host application (cudaDeviceReset) ends the context the address
// belongs to: each call first checks, with a host-side pointer query, that
// the cached address is still this device's memory, and looks it up again
// when it is not.
static void *noalloc_scratch_ptr(int &rc) {
    static std::mutex mu;
    static void *ptrs[128] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) {
        rc = LIG_ERR_LAUNCH;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (ptrs[dev]) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, ptrs[dev]) != cudaSuccess ||
            a.type != cudaMemoryTypeDevice || a.device != dev) {
            (void)cudaGetLastError();  // the failed query must not reach the launch check
            ptrs[dev] = nullptr;
        }
    }
    if (!ptrs[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            rc = LIG_ERR_LAUNCH;
            return nullptr;
        }
        ptrs[dev] = p;
    }
    rc = LIG_OK;
    return ptrs[dev];
}
}  // namespace lig

extern "C" int lig_raster_fwd_noalloc(int H, int W, int B, int n, const int32_t *ids,
                                      const int32_t *bins, const int32_t *d_total,
                                      const float *xys, const float *con, const float *col,
                                      const float *op, float *img, float *wsum, int32_t *fin,
                                      void *stream) {
    if (n > LIG_STATIC_MAX_POINTS) return LIG_ERR_TOO_LARGE;
    if (!raster_args_ok(H, W, B, n) || !bins || !d_total || !img || !wsum || !fin ||
        (n > 0 && (!xys || !con || !col)))
        return LIG_ERR_INVALID;
    int rc = LIG_OK;
    void *scratch = noalloc_scratch_ptr(rc);
    if (rc != LIG_OK) return rc;
    return raster_fwd<float>(BatchGeo::single(H, W, B, n), TileWalk{}, ids, bins, d_total, xys,
                             con, col, op, scratch, sizeof(g_noalloc_scratch), img, wsum, nullptr,
                             nullptr, nullptr, fin, (cudaStream_t)stream);
}

// ------------------------------------------------------------ batched entries
// A batch of images in one launch per stage: image i has heights[i] x
// widths[i] pixels and counts[i] Gaussians; Gaussians, tile lists and the
// HWC buffers are the images' arrays concatenated in batch order.  The
// (image, tile) work list is flattened (image-major, row-major tiles within
// an image); persistent != 0 runs one CTA per resident slot pulling work
// items from `work` (one int of device memory, overwritten).
namespace lig {
inline bool batch_geo(int n_img, const int32_t *h, const int32_t *w, const int32_t *c, int B,
                      BatchGeo &geo) {
    if (!h || !w || !c || B < 2 || B > 32) return false;
    return BatchGeo::make(n_img, h, w, c, B, geo);
}
}  // namespace lig

extern "C" int lig_raster_fwd_batch(int dtype, int n_img, const int32_t *heights,
                                    const int32_t *widths, const int32_t *counts, int B,
                                    const int32_t *ids, const int32_t *bins,
                                    const int32_t *d_total, const int32_t *cum, const void *xys,
                                    const void *con, const void *col, const void *op,
                                    int persistent, int32_t *work, void *ws, size_t ws_bytes,
                                    void *img, void *wsum, void *dx, void *dy, void *dxy,
                                    int32_t *fin, void *stream) {
    BatchGeo geo;
    if (!batch_geo(n_img, heights, widths, counts, B, geo)) return LIG_ERR_INVALID;
    const int n = geo.total_points();
    if (!bins || !d_total || !img || !wsum || !fin || !ws || (persistent && !work) ||
        (n > 0 && (!xys || !con || !col || !cum)) || ((dx || dy || dxy) && !(dx && dy && dxy)))
        return LIG_ERR_INVALID;
    TileWalk walk{n > 0 ? cum : nullptr, persistent ? work : nullptr};
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return raster_fwd<float>(geo, walk, ids, bins, d_total, xys, con, col, op, ws, ws_bytes,
                                 img, wsum, dx, dy, dxy, fin, s);
    if (dtype == LIG_F64)
        return raster_fwd<double>(geo, walk, ids, bins, d_total, xys, con, col, op, ws, ws_bytes,
                                  img, wsum, dx, dy, dxy, fin, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_bwd_l2_batch(int dtype, int n_img, const int32_t *heights,
                                       const int32_t *widths, const int32_t *counts, int B,
                                       const int32_t *ids, const int32_t *bins,
                                       const int32_t *d_total, const int32_t *cum,
                                       const void *xys, const void *con, const void *col,
                                       const void *op, const int32_t *fin, const void *img,
                                       const void *target, const void *grad_loss, double clamp,
                                       int persistent, int32_t *work, void *ws, size_t ws_bytes,
                                       void *v_xy, void *v_abs, void *v_con, void *v_rgb,
                                       void *v_op, void *stream) {
    BatchGeo geo;
    if (!batch_geo(n_img, heights, widths, counts, B, geo)) return LIG_ERR_INVALID;
    const int n = geo.total_points();
    if (!bins || !d_total || !fin || !img || !target || !grad_loss || !ws ||
        (persistent && !work) ||
        (n > 0 && (!xys || !con || !col || !cum || !v_xy || !v_abs || !v_con || !v_rgb)))
        return LIG_ERR_INVALID;
    if (n == 0) return LIG_OK;
    TileWalk walk{cum, persistent ? work : nullptr};
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32) {
        // per-image scale 2 / (3 H_i W_i) is formed in the kernel
        CotSrc<float> cot{nullptr, nullptr, (const float *)img, (const float *)target,
                          (const float *)grad_loss, 0.f};
        return raster_bwd<float>(geo, walk, ids, bins, d_total, xys, con, col, op, fin, cot,
                                 nullptr, nullptr, nullptr, clamp, ws, ws_bytes, v_xy, v_abs,
                                 v_con, v_rgb, v_op, s);
    }
    if (dtype == LIG_F64) {
        CotSrc<double> cot{nullptr, nullptr, (const double *)img, (const double *)target,
                           (const double *)grad_loss, 0.0};
        return raster_bwd<double>(geo, walk, ids, bins, d_total, xys, con, col, op, fin, cot,
                                  nullptr, nullptr, nullptr, clamp, ws, ws_bytes, v_xy, v_abs,
                                  v_con, v_rgb, v_op, s);
    }
    return LIG_ERR_INVALID;
}

// ------------------------------------------------------- fused-L2 forward
// The fit loop's forward: tile lists rendered as lig_raster_fwd, but each
// pixel stores diff = (0 <= x <= 1) ? clamp(x) - target : 0 (not the image)
// and loss = sum_i mean_i((clamp(x) - target)^2) is reduced from per-tile
// fp64 partials; lig_raster_bwd_diff then forms the loss gradient from diff.
extern "C" size_t lig_l2_tile_partials_bytes(int num_tiles) {
    // per-tile partials, then the chunk sums (at most one per kLossChunk
    // tiles plus one per image of a batch)
    const size_t t = (size_t)(num_tiles > 0 ? num_tiles : 0);
    return sizeof(double) * (t + t / kLossChunk + 1 + kMaxBatch);
}

namespace lig {
// target: T values, or bytes when u8
template <typename T>
int fwd_l2(const BatchGeo &geo, TileWalk walk, const int32_t *ids, const int32_t *bins,
           const int32_t *d_total, const void *xys, const void *con, const void *col,
           const void *op, const void *target, void *ws, size_t ws_bytes, double *partials,
           void *diff, int32_t *fin, void *loss, void *per_image, cudaStream_t s,
           bool u8 = false) {
    const L2Fwd<T> l2 = u8 ? L2Fwd<T>{nullptr, partials, (const uint8_t *)target}
                           : L2Fwd<T>{(const T *)target, partials};
    return raster_fwd<T>(geo, walk, ids, bins, d_total, xys, con, col, op, ws, ws_bytes, diff,
                         nullptr, nullptr, nullptr, nullptr, fin, s, l2,
                         L2Out<T>{(T *)loss, (T *)per_image});
}

template <typename T>
int bwd_diff(const BatchGeo &geo, TileWalk walk, const int32_t *ids, const int32_t *bins,
             const int32_t *d_total, const void *xys, const void *con, const void *col,
             const void *op, const int32_t *fin, const void *diff, const void *grad_loss,
             double clamp, void *ws, size_t ws_bytes, void *v_xy, void *v_abs, void *v_con,
             void *v_rgb, void *v_op, cudaStream_t s) {
    // per-image scale 2 / (3 H_i W_i) is formed in the kernel
    CotSrc<T> cot{nullptr, nullptr, nullptr, nullptr, (const T *)grad_loss, (T)0,
                  (const T *)diff};
    return raster_bwd<T>(geo, walk, ids, bins, d_total, xys, con, col, op, fin, cot, nullptr,
                         nullptr, nullptr, clamp, ws, ws_bytes, v_xy, v_abs, v_con, v_rgb, v_op,
                         s);
}
}  // namespace lig

extern "C" int lig_raster_fwd_l2(int dtype, int H, int W, int B, int n, const int32_t *ids,
                                 const int32_t *bins, const int32_t *d_total, const void *xys,
                                 const void *con, const void *col, const void *op,
                                 const void *target, void *ws, size_t ws_bytes,
                                 double *tile_partials, void *diff, int32_t *fin, void *loss,
                                 void *stream) {
    if (!raster_args_ok(H, W, B, n) || !bins || !d_total || !target || !ws || !tile_partials ||
        !diff || !loss || (n > 0 && (!xys || !con || !col)))
        return LIG_ERR_INVALID;
    const BatchGeo geo = BatchGeo::single(H, W, B, n);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return fwd_l2<float>(geo, TileWalk{}, ids, bins, d_total, xys, con, col, op, target, ws,
                             ws_bytes, tile_partials, diff, fin, loss, nullptr, s);
    if (dtype == LIG_F64)
        return fwd_l2<double>(geo, TileWalk{}, ids, bins, d_total, xys, con, col, op, target, ws,
                              ws_bytes, tile_partials, diff, fin, loss, nullptr, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_fwd_l2_u8(int dtype, int H, int W, int B, int n, const int32_t *ids,
                                    const int32_t *bins, const int32_t *d_total, const void *xys,
                                    const void *con, const void *col, const void *op,
                                    const uint8_t *target, void *ws, size_t ws_bytes,
                                    double *tile_partials, void *diff, int32_t *fin, void *loss,
                                    void *stream) {
    if (!raster_args_ok(H, W, B, n) || !bins || !d_total || !target || !ws || !tile_partials ||
        !diff || !loss || (n > 0 && (!xys || !con || !col)))
        return LIG_ERR_INVALID;
    const BatchGeo geo = BatchGeo::single(H, W, B, n);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return fwd_l2<float>(geo, TileWalk{}, ids, bins, d_total, xys, con, col, op, target, ws,
                             ws_bytes, tile_partials, diff, fin, loss, nullptr, s, true);
    if (dtype == LIG_F64)
        return fwd_l2<double>(geo, TileWalk{}, ids, bins, d_total, xys, con, col, op, target, ws,
                              ws_bytes, tile_partials, diff, fin, loss, nullptr, s, true);
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_bwd_diff(int dtype, int H, int W, int B, int n, const int32_t *ids,
                                   const int32_t *bins, const int32_t *d_total, const void *xys,
                                   const void *con, const void *col, const void *op,
                                   const int32_t *fin, const void *diff, const void *grad_loss,
                                   double clamp, void *ws, size_t ws_bytes, void *v_xy,
                                   void *v_abs, void *v_con, void *v_rgb, void *v_op,
                                   void *stream) {
    if (!raster_args_ok(H, W, B, n) || !bins || !d_total || (!fin && op) || !diff ||
        !grad_loss || !ws || (n > 0 && (!xys || !con || !col || !v_xy || !v_abs || !v_con || !v_rgb)))
        return LIG_ERR_INVALID;
    if (n == 0) return LIG_OK;
    const BatchGeo geo = BatchGeo::single(H, W, B, n);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return bwd_diff<float>(geo, TileWalk{}, ids, bins, d_total, xys, con, col, op, fin, diff,
                               grad_loss, clamp, ws, ws_bytes, v_xy, v_abs, v_con, v_rgb, v_op, s);
    if (dtype == LIG_F64)
        return bwd_diff<double>(geo, TileWalk{}, ids, bins, d_total, xys, con, col, op, fin,
                                diff, grad_loss, clamp, ws, ws_bytes, v_xy, v_abs, v_con, v_rgb,
                                v_op, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_fwd_l2_batch(int dtype, int n_img, const int32_t *heights,
                                       const int32_t *widths, const int32_t *counts, int B,
                                       const int32_t *ids, const int32_t *bins,
                                       const int32_t *d_total, const int32_t *cum,
                                       const void *xys, const void *con, const void *col,
                                       const void *op, const void *target, int persistent,
                                       int32_t *work, void *ws, size_t ws_bytes,
                                       double *tile_partials, void *diff, int32_t *fin,
                                       void *loss, void *per_image, void *stream) {
    BatchGeo geo;
    if (!batch_geo(n_img, heights, widths, counts, B, geo)) return LIG_ERR_INVALID;
    const int n = geo.total_points();
    if (!bins || !d_total || !target || !ws || !tile_partials || !diff || !loss ||
        (persistent && !work) || (n > 0 && (!xys || !con || !col || !cum)))
        return LIG_ERR_INVALID;
    TileWalk walk{n > 0 ? cum : nullptr, persistent ? work : nullptr};
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return fwd_l2<float>(geo, walk, ids, bins, d_total, xys, con, col, op, target, ws,
                             ws_bytes, tile_partials, diff, fin, loss, per_image, s);
    if (dtype == LIG_F64)
        return fwd_l2<double>(geo, walk, ids, bins, d_total, xys, con, col, op, target, ws,
                              ws_bytes, tile_partials, diff, fin, loss, per_image, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_fwd_l2_u8_batch(int dtype, int n_img, const int32_t *heights,
                                          const int32_t *widths, const int32_t *counts, int B,
                                          const int32_t *ids, const int32_t *bins,
                                          const int32_t *d_total, const int32_t *cum,
                                          const void *xys, const void *con, const void *col,
                                          const void *op, const uint8_t *target, int persistent,
                                          int32_t *work, void *ws, size_t ws_bytes,
                                          double *tile_partials, void *diff, int32_t *fin,
                                          void *loss, void *per_image, void *stream) {
    BatchGeo geo;
    if (!batch_geo(n_img, heights, widths, counts, B, geo)) return LIG_ERR_INVALID;
    const int n = geo.total_points();
    if (!bins || !d_total || !target || !ws || !tile_partials || !diff || !loss ||
        (persistent && !work) || (n > 0 && (!xys || !con || !col || !cum)))
        return LIG_ERR_INVALID;
    TileWalk walk{n > 0 ? cum : nullptr, persistent ? work : nullptr};
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return fwd_l2<float>(geo, walk, ids, bins, d_total, xys, con, col, op, target, ws,
                             ws_bytes, tile_partials, diff, fin, loss, per_image, s, true);
    if (dtype == LIG_F64)
        return fwd_l2<double>(geo, walk, ids, bins, d_total, xys, con, col, op, target, ws,
                              ws_bytes, tile_partials, diff, fin, loss, per_image, s, true);
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_bwd_diff_batch(int dtype, int n_img, const int32_t *heights,
                                         const int32_t *widths, const int32_t *counts, int B,
                                         const int32_t *ids, const int32_t *bins,
                                         const int32_t *d_total, const int32_t *cum,
                                         const void *xys, const void *con, const void *col,
                                         const void *op, const int32_t *fin, const void *diff,
                                         const void *grad_loss, double clamp, int persistent,
                                         int32_t *work, void *ws, size_t ws_bytes, void *v_xy,
                                         void *v_abs, void *v_con, void *v_rgb, void *v_op,
                                         void *stream) {
    BatchGeo geo;
    if (!batch_geo(n_img, heights, widths, counts, B, geo)) return LIG_ERR_INVALID;
    const int n = geo.total_points();
    if (!bins || !d_total || (!fin && op) || !diff || !grad_loss || !ws || (persistent && !work) ||
        (n > 0 && (!xys || !con || !col || !cum || !v_xy || !v_abs || !v_con || !v_rgb)))
        return LIG_ERR_INVALID;
    if (n == 0) return LIG_OK;
    TileWalk walk{cum, persistent ? work : nullptr};
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return bwd_diff<float>(geo, walk, ids, bins, d_total, xys, con, col, op, fin, diff,
                               grad_loss, clamp, ws, ws_bytes, v_xy, v_abs, v_con, v_rgb, v_op, s);
    if (dtype == LIG_F64)
        return bwd_diff<double>(geo, walk, ids, bins, d_total, xys, con, col, op, fin, diff,
                                grad_loss, clamp, ws, ws_bytes, v_xy, v_abs, v_con, v_rgb, v_op,
                                s);
    return LIG_ERR_INVALID;
}
