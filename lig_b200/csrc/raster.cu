// Weighted-sum rasterizer, forward and backward, plain and gradient-aware.
//
// Work decomposition (B200): one warp owns one (tile, band) work item.  A band
// is up to PPL "pixel blocks" of the tile; a pixel block is 32 pixels, one per
// lane, so a lane holds PPL pixels and keeps their accumulators (forward) or
// cotangents (backward) in registers for the whole tile list.  There is no
// __syncthreads: warps of a CTA work on different tiles.
//
// Pixel blocks are 8x4 pixel rectangles, except in the gradient-aware backward,
// where block b is the reference's warp b (thread ranks 32b..32b+31 of the
// B x B tile, rank = ty*B + tx): its v_xy_abs is |sum over that warp| per
// Gaussian (csrc/gradient_aware_rasterizer.cu:317-341), so the grouping is
// part of the result.
//
// Gaussian data: a pack kernel writes one 16-byte-aligned record per Gaussian
// (mean, conic, opacity, colour, cull half-widths).  A warp streams its tile's
// sorted id list in chunks of 32: lane l fetches record (chunk + l) into
// registers two chunks ahead of use (ids three chunks ahead), then parks it in
// a per-warp shared-memory slot from which all lanes read it by broadcast.
//
// Culling: for each (Gaussian, pixel block) the warp tests the block's pixel
// centres against a conservative box around the Gaussian's alpha >= 1/255
// ellipse and skips the block when it misses.  The box is built with margin
// (see pack_kernel), so every skipped pixel would have failed the reference's
// own `alpha < 1/255` test (csrc/forward.cu:258): results are unchanged.
//
// Per-pixel arithmetic is written exactly as the reference writes it
// (csrc/forward.cu:250-269, csrc/backward.cu:102-150,
// csrc/gradient_aware_rasterizer.cu:201-315, :434-482) so that the float
// roundings, and with them the alpha-threshold decisions, are the same.
#include "common.cuh"

namespace lig {

template <typename T> struct alignas(16) Rec {
    T x, y, a, b;     // mean, conic (a, b)
    T c, o, wx, wy;   // conic c, opacity, cull half-widths (negative: never cull)
    T r, g, bl, pad;  // colour
};

// ------------------------------------------------------------------ pack
// Cull half-widths: the alpha >= 1/255 region of a positive-definite conic is
// the ellipse sigma <= t/2, t = 2 ln(255 o), whose x half-extent is
// sqrt(t Sxx).  We use t_c = max(t, 0.01) and w = 1.001 sqrt(t_c Sxx) + 2 px:
// a pixel centre outside the box has sigma above the threshold by at least
// ~sqrt(t_c/Sxx) + 0.001 t_c, orders of magnitude above float rounding of
// sigma and __expf.  No culling (w < 0) for non-finite inputs, non-positive
// opacity, non-positive-definite or nearly degenerate conics (b^2 > 0.999 ac),
// where the reference's per-pixel tests must run everywhere in the tile.
template <typename T>
__global__ void pack_kernel(int n, const T *__restrict__ xys, const T *__restrict__ conics,
                            const T *__restrict__ colors, const T *__restrict__ opac,
                            Rec<T> *__restrict__ recs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
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
    r.pad = 0;
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
        if (hx < 1e7 && hy < 1e7) {
            wx = (T)hx;
            wy = (T)hy;
        }
    }
    r.wx = wx;
    r.wy = wy;
    recs[i] = r;
}

// ------------------------------------------------------------ pixel maps
// mode 0: 8x4 blocks; mode 1: reference warps (32 consecutive thread ranks).
struct TileMap {
    int B, nbx, nblk;
    __device__ __forceinline__ void pixel(int mode, int bi, int lane, int &lx, int &ly) const {
        if (mode == 0) {
            int bx = bi % nbx, by = bi / nbx;
            lx = bx * 8 + (lane & 7);
            ly = by * 4 + (lane >> 3);
        } else {
            int r = bi * 32 + lane;
            lx = r % B;
            ly = r / B;
            if (r >= B * B) ly = B;  // mark invalid
        }
    }
    // conservative tile-local pixel-index rectangle of block bi
    __device__ __forceinline__ void rect(int mode, int bi, int &x0, int &x1, int &y0,
                                         int &y1) const {
        if (mode == 0) {
            int bx = bi % nbx, by = bi / nbx;
            x0 = bx * 8; x1 = x0 + 7;
            y0 = by * 4; y1 = y0 + 3;
        } else {
            int r0 = bi * 32, r1 = min(r0 + 31, B * B - 1);
            y0 = r0 / B; y1 = r1 / B;
            if (y0 == y1) { x0 = r0 % B; x1 = r1 % B; }
            else { x0 = 0; x1 = B - 1; }
        }
    }
};

// True when the Gaussian's cull box misses the block's pixel centres.  Written
// as "strictly outside" so NaN / infinite values never cause a skip.
template <typename T>
__device__ __forceinline__ bool box_misses(const Rec<T> &g, T bx0, T bx1, T by0, T by1) {
    if (!(g.wx >= (T)0)) return false;
    return (g.x + g.wx < bx0) || (g.x - g.wx > bx1) || (g.y + g.wy < by0) || (g.y - g.wy > by1);
}

// Record streaming state for one warp.
template <typename T>
struct Stream {
    Rec<T> *slots;   // 32 per-warp shared slots
    Rec<T> nxt;      // record of the next chunk (this lane's entry)
    int id_nxt2;     // id of the chunk after next (this lane's entry)
    const Rec<T> *recs;
    const int32_t *ids;
    int end;

    __device__ __forceinline__ void fetch_id(int e, int &id) const {
        id = e < end ? __ldg(ids + e) : -1;
    }
    __device__ __forceinline__ void fetch_rec(int id, Rec<T> &r) const {
        if (id >= 0) r = recs[id];
    }
    // Begin at entry e0: park chunk e0 in smem, prefetch chunk e0+32, ids of e0+64.
    __device__ __forceinline__ void start(int e0, int lane) {
        int id0, id1;
        fetch_id(e0 + lane, id0);
        fetch_id(e0 + 32 + lane, id1);
        fetch_id(e0 + 64 + lane, id_nxt2);
        Rec<T> cur;
        fetch_rec(id0, cur);
        fetch_rec(id1, nxt);
        slots[lane] = cur;
        __syncwarp();
    }
    // After chunk `e` is consumed: park chunk e+32, prefetch e+64, ids of e+96.
    __device__ __forceinline__ void advance(int e, int lane) {
        __syncwarp();
        slots[lane] = nxt;
        int id = id_nxt2;
        fetch_id(e + 96 + lane, id_nxt2);
        fetch_rec(id, nxt);
        __syncwarp();
    }
};

// --------------------------------------------------------------- forward
template <typename T, bool GA, int PPL>
__global__ void __launch_bounds__(128)
raster_fwd_kernel(int H, int W, int B, int tbx, int nbands, int nwork,
                  const int32_t *__restrict__ ids, const int2 *__restrict__ tile_bins,
                  const int32_t *__restrict__ d_total, const Rec<T> *__restrict__ recs,
                  T *__restrict__ img, T *__restrict__ wsum, T *__restrict__ odx,
                  T *__restrict__ ody, T *__restrict__ odxy, int32_t *__restrict__ final_idx) {
    using M = Math<T>;
    __shared__ Rec<T> s_rec[4][32];
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int work = blockIdx.x * 4 + wib;
    if (work >= nwork) return;
    int tile = work / nbands, band = work % nbands;
    int tx0 = (tile % tbx) * B, ty0 = (tile / tbx) * B;
    TileMap map{B, (B + 7) / 8, ((B + 7) / 8) * ((B + 3) / 4)};

    T px[PPL], py[PPL];
    bool in[PPL];
    int pix[PPL];
#pragma unroll
    for (int i = 0; i < PPL; ++i) {
        int bi = band * PPL + i, lx = B, ly = B;
        if (bi < map.nblk) map.pixel(0, bi, lane, lx, ly);
        int gx = tx0 + lx, gy = ty0 + ly;
        in[i] = lx < B && ly < B && gx < W && gy < H;
        px[i] = (T)gx + (T)0.5;
        py[i] = (T)gy + (T)0.5;
        pix[i] = gy * W + gx;
    }

    if (*d_total == 0) {  // reference: white image, zero weights (rasterize.py:80-90)
#pragma unroll
        for (int i = 0; i < PPL; ++i) {
            if (!in[i]) continue;
            int p = pix[i];
            img[3 * p] = (T)1; img[3 * p + 1] = (T)1; img[3 * p + 2] = (T)1;
            wsum[p] = 0;
            final_idx[p] = 0;
            if (GA) {
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) { odx[3 * p + ch] = 0; ody[3 * p + ch] = 0; odxy[3 * p + ch] = 0; }
            }
        }
        return;
    }

    T acc[PPL][3], ws[PPL];
    T adx[GA ? PPL : 1][3], ady[GA ? PPL : 1][3], adxy[GA ? PPL : 1][3];
    int cur[PPL];
#pragma unroll
    for (int i = 0; i < PPL; ++i) {
        acc[i][0] = acc[i][1] = acc[i][2] = 0;
        ws[i] = 0;
        cur[i] = 0;
        if (GA) {
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) adx[i][ch] = ady[i][ch] = adxy[i][ch] = 0;
        }
    }
    // block pixel-centre rectangles (image coordinates), per i
    T bx0[PPL], bx1[PPL], by0[PPL], by1[PPL];
    bool bvalid[PPL];
#pragma unroll
    for (int i = 0; i < PPL; ++i) {
        int bi = band * PPL + i;
        int x0 = 0, x1 = -1, y0 = 0, y1 = -1;
        bvalid[i] = bi < map.nblk;
        if (bvalid[i]) map.rect(0, bi, x0, x1, y0, y1);
        bx0[i] = (T)(tx0 + x0) + (T)0.5; bx1[i] = (T)(tx0 + x1) + (T)0.5;
        by0[i] = (T)(ty0 + y0) + (T)0.5; by1[i] = (T)(ty0 + y1) + (T)0.5;
    }

    int2 range = tile_bins[tile];
    Stream<T> st;
    st.slots = s_rec[wib];
    st.recs = recs;
    st.ids = ids;
    st.end = range.y;
    if (range.x < range.y) st.start(range.x, lane);
    for (int e = range.x; e < range.y; e += 32) {
        int cnt = min(32, range.y - e);
        for (int t = 0; t < cnt; ++t) {
            const Rec<T> g = st.slots[t];
#pragma unroll
            for (int i = 0; i < PPL; ++i) {
                if (!bvalid[i] || box_misses(g, bx0[i], bx1[i], by0[i], by1[i])) continue;
                if (!in[i]) continue;
                if (!GA) {
                    // csrc/forward.cu:250-269
                    const T dx = g.x - px[i];
                    const T dy = g.y - py[i];
                    const T sigma = (T)0.5 * (g.a * dx * dx + g.c * dy * dy) + g.b * dx * dy;
                    const T alpha = M::min_((T)0.999, g.o * M::exp_(-sigma));
                    if (sigma < (T)0 || alpha < (T)1 / (T)255) continue;
                    acc[i][0] += g.r * alpha;
                    acc[i][1] += g.g * alpha;
                    acc[i][2] += g.bl * alpha;
                    ws[i] += alpha;
                    cur[i] = e + t;
                } else {
                    // csrc/gradient_aware_rasterizer.cu:434-482
                    const T dx = px[i] - g.x;
                    const T dy = py[i] - g.y;
                    const T sigma = (T)0.5 * (g.a * dx * dx + g.c * dy * dy) + g.b * dx * dy;
                    const T alpha = M::min_((T)0.999, g.o * M::exp_(-sigma));
                    if (sigma < (T)0 || alpha < (T)1 / (T)255) continue;
                    const T sdx = g.a * dx + g.b * dy;
                    const T sdy = g.b * dx + g.c * dy;
                    const T s2 = g.b;
                    const T adx_ = -alpha * sdx;
                    const T ady_ = -alpha * sdy;
                    const T adxy_ = -alpha * (s2 - sdx * sdy);
                    acc[i][0] += g.r * alpha;
                    acc[i][1] += g.g * alpha;
                    acc[i][2] += g.bl * alpha;
                    adx[i][0] += g.r * adx_; adx[i][1] += g.g * adx_; adx[i][2] += g.bl * adx_;
                    ady[i][0] += g.r * ady_; ady[i][1] += g.g * ady_; ady[i][2] += g.bl * ady_;
                    adxy[i][0] += g.r * adxy_; adxy[i][1] += g.g * adxy_; adxy[i][2] += g.bl * adxy_;
                    ws[i] += alpha;
                    cur[i] = e + t;
                }
            }
        }
        if (e + 32 < range.y) st.advance(e, lane);
    }
#pragma unroll
    for (int i = 0; i < PPL; ++i) {
        if (!in[i]) continue;
        int p = pix[i];
        final_idx[p] = cur[i];
        img[3 * p] = acc[i][0];
        img[3 * p + 1] = acc[i][1];
        img[3 * p + 2] = acc[i][2];
        wsum[p] = ws[i];
        if (GA) {
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                odx[3 * p + ch] = adx[i][ch];
                ody[3 * p + ch] = ady[i][ch];
                odxy[3 * p + ch] = adxy[i][ch];
            }
        }
    }
}

// ------------------------------------------------------------- backward
// Transpose-reduce of 16 per-lane values over the warp in 16 shuffles: after
// the call lane l holds the warp sum of value ((l >> 1) & 15) in v[0].
template <typename T>
__device__ __forceinline__ void transpose_reduce16(T (&v)[16], int lane) {
    const unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        bool up = lane & 16;
        T send = up ? v[k] : v[k + 8];
        T keep = up ? v[k + 8] : v[k];
        v[k] = keep + __shfl_xor_sync(FULL, send, 16);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        bool up = lane & 8;
        T send = up ? v[k] : v[k + 4];
        T keep = up ? v[k + 4] : v[k];
        v[k] = keep + __shfl_xor_sync(FULL, send, 8);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        bool up = lane & 4;
        T send = up ? v[k] : v[k + 2];
        T keep = up ? v[k + 2] : v[k];
        v[k] = keep + __shfl_xor_sync(FULL, send, 4);
    }
    {
        bool up = lane & 2;
        T send = up ? v[0] : v[1];
        T keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(FULL, send, 2);
    }
    v[0] += __shfl_xor_sync(FULL, v[0], 1);
}

template <typename T>
struct Grads {
    T *v_xy, *v_abs, *v_conic, *v_rgb, *v_opac;
    // value index k: 0-1 v_xy, 2-3 v_xy_abs, 4-6 v_conic, 7-9 v_rgb, 10 v_opacity
    __device__ __forceinline__ void add(int k, int g, T val) const {
        T *p = nullptr;
        if (k < 2) p = v_xy + 2 * g + k;
        else if (k < 4) p = v_abs + 2 * g + (k - 2);
        else if (k < 7) p = v_conic + 3 * g + (k - 4);
        else if (k < 10) p = v_rgb + 3 * g + (k - 7);
        else if (k == 10 && v_opac) p = v_opac + g;
        if (p) atomicAdd(p, val);
    }
};

template <typename T, bool GA, int PPL>
__global__ void __launch_bounds__(128)
raster_bwd_kernel(int H, int W, int B, int tbx, int nbands, int nwork,
                  const int32_t *__restrict__ ids, const int2 *__restrict__ tile_bins,
                  const int32_t *__restrict__ d_total, const Rec<T> *__restrict__ recs,
                  const int32_t *__restrict__ final_idx, const T *__restrict__ v_img,
                  const T *__restrict__ v_wsum, const T *__restrict__ v_dx,
                  const T *__restrict__ v_dy, const T *__restrict__ v_dxy, T clamp,
                  Grads<T> out) {
    using M = Math<T>;
    constexpr int MODE = GA ? 1 : 0;
    __shared__ Rec<T> s_rec[4][32];
    const unsigned FULL = 0xffffffffu;
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int work = blockIdx.x * 4 + wib;
    if (work >= nwork) return;
    if (*d_total == 0) return;  // gradients stay zero (rasterize.py:156-161)
    int tile = work / nbands, band = work % nbands;
    int tx0 = (tile % tbx) * B, ty0 = (tile / tbx) * B;
    int nblk = GA ? (B * B + 31) / 32 : ((B + 7) / 8) * ((B + 3) / 4);
    TileMap map{B, (B + 7) / 8, nblk};

    T px[PPL], py[PPL];
    int fin[PPL];
    T vo[PPL][3], vw[PPL];
    T vdx[GA ? PPL : 1][3], vdy[GA ? PPL : 1][3], vdxy[GA ? PPL : 1][3];
    T bx0[PPL], bx1[PPL], by0[PPL], by1[PPL];
    bool bvalid[PPL];
    int band_fin = -1;
#pragma unroll
    for (int i = 0; i < PPL; ++i) {
        int bi = band * PPL + i, lx = B, ly = B;
        bvalid[i] = bi < map.nblk;
        int x0 = 0, x1 = -1, y0 = 0, y1 = -1;
        if (bvalid[i]) {
            map.pixel(MODE, bi, lane, lx, ly);
            map.rect(MODE, bi, x0, x1, y0, y1);
        }
        bx0[i] = (T)(tx0 + x0) + (T)0.5; bx1[i] = (T)(tx0 + x1) + (T)0.5;
        by0[i] = (T)(ty0 + y0) + (T)0.5; by1[i] = (T)(ty0 + y1) + (T)0.5;
        int gx = tx0 + lx, gy = ty0 + ly;
        bool inside = lx < B && ly < B && gx < W && gy < H;
        px[i] = (T)gx + (T)0.5;
        py[i] = (T)gy + (T)0.5;
        int p = inside ? gy * W + gx : 0;
        fin[i] = inside ? final_idx[p] : -1;  // -1: never valid
        vo[i][0] = inside ? v_img[3 * p] : (T)0;
        vo[i][1] = inside ? v_img[3 * p + 1] : (T)0;
        vo[i][2] = inside ? v_img[3 * p + 2] : (T)0;
        vw[i] = inside ? v_wsum[p] : (T)0;
        if (GA) {
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                vdx[i][ch] = inside ? v_dx[3 * p + ch] : (T)0;
                vdy[i][ch] = inside ? v_dy[3 * p + ch] : (T)0;
                vdxy[i][ch] = inside ? v_dxy[3 * p + ch] : (T)0;
            }
        }
        band_fin = max(band_fin, fin[i]);
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) band_fin = max(band_fin, __shfl_xor_sync(FULL, band_fin, o));

    int2 range = tile_bins[tile];
    int end = min(range.y, band_fin + 1);  // entries past every pixel's final index: no work
    Stream<T> st;
    st.slots = s_rec[wib];
    st.recs = recs;
    st.ids = ids;
    st.end = end;
    if (range.x < end) st.start(range.x, lane);
    for (int e = range.x; e < end; e += 32) {
        int cnt = min(32, end - e);
        for (int t = 0; t < cnt; ++t) {
            const Rec<T> g = st.slots[t];
            const int k = e + t;
            T v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = 0;
            bool any = false;
#pragma unroll
            for (int i = 0; i < PPL; ++i) {
                if (!bvalid[i] || box_misses(g, bx0[i], bx1[i], by0[i], by1[i])) continue;
                bool valid = k <= fin[i];
                if (!GA) {
                    if (!__any_sync(FULL, valid)) continue;
                    if (!valid) continue;
                    // csrc/backward.cu:102-150
                    const T dx = g.x - px[i];
                    const T dy = g.y - py[i];
                    const T sigma = (T)0.5 * (g.a * dx * dx + g.c * dy * dy) + g.b * dx * dy;
                    const T vis = M::exp_(-sigma);
                    const T alpha = M::min_(clamp, g.o * vis);
                    if (sigma < (T)0 || alpha < (T)1 / (T)255) continue;
                    any = true;
                    T v_alpha = 0;
                    v[7] += alpha * vo[i][0];
                    v[8] += alpha * vo[i][1];
                    v[9] += alpha * vo[i][2];
                    v_alpha += g.r * vo[i][0];
                    v_alpha += g.g * vo[i][1];
                    v_alpha += g.bl * vo[i][2];
                    v_alpha += vw[i];
                    v[10] += vis * v_alpha;
                    const T v_sigma = -alpha * v_alpha;
                    v[4] += (T)0.5 * v_sigma * dx * dx;
                    v[5] += v_sigma * dx * dy;
                    v[6] += (T)0.5 * v_sigma * dy * dy;
                    const T gx = v_sigma * (g.a * dx + g.b * dy);
                    const T gy = v_sigma * (g.b * dx + g.c * dy);
                    v[0] += gx;
                    v[1] += gy;
                    v[2] += M::abs_(gx);
                    v[3] += M::abs_(gy);
                } else {
                    // csrc/gradient_aware_rasterizer.cu:191-315
                    T gx = 0, gy = 0;
                    bool ok = false;
                    if (valid) {
                        const T dx = px[i] - g.x;
                        const T dy = py[i] - g.y;
                        const T sigma = (T)0.5 * (g.a * dx * dx + g.c * dy * dy) + g.b * dx * dy;
                        const T vis = M::exp_(-sigma);
                        const T alpha = M::min_(clamp, g.o * vis);
                        ok = !(sigma < (T)0 || alpha < (T)1 / (T)255);
                        if (ok) {
                            const T sx = g.a * dx + g.b * dy;
                            const T sy = g.b * dx + g.c * dy;
                            const T a = g.a, b = g.b, cc = g.c;
                            const T ax = -alpha * sx;
                            const T ay = -alpha * sy;
                            const T axy = alpha * (sx * sy - b);
                            v[7] += vo[i][0] * alpha + vdx[i][0] * ax + vdy[i][0] * ay + vdxy[i][0] * axy;
                            v[8] += vo[i][1] * alpha + vdx[i][1] * ax + vdy[i][1] * ay + vdxy[i][1] * axy;
                            v[9] += vo[i][2] * alpha + vdx[i][2] * ax + vdy[i][2] * ay + vdxy[i][2] * axy;
                            const T va = (vo[i][0] * g.r + vo[i][1] * g.g + vo[i][2] * g.bl) + vw[i];
                            const T vax = vdx[i][0] * g.r + vdx[i][1] * g.g + vdx[i][2] * g.bl;
                            const T vay = vdy[i][0] * g.r + vdy[i][1] * g.g + vdy[i][2] * g.bl;
                            const T vaxy = vdxy[i][0] * g.r + vdxy[i][1] * g.g + vdxy[i][2] * g.bl;
                            const T sx2 = sx * sx, sy2 = sy * sy, sxsy = sx * sy;
                            gx = alpha * (va * sx + vax * (a - sx2) + vay * (b - sxsy) +
                                          vaxy * (sx2 * sy - (T)2 * b * sx - a * sy));
                            gy = alpha * (va * sy + vax * (b - sxsy) + vay * (cc - sy2) +
                                          vaxy * (sx * sy2 - (T)2 * b * sy - cc * sx));
                            const T dx2 = dx * dx, dy2 = dy * dy, dxdy = dx * dy;
                            const T P = sxsy - b;
                            v[4] += alpha * (va * (-(T)0.5 * dx2) + vax * ((T)0.5 * dx2 * sx - dx) +
                                             vay * ((T)0.5 * dx2 * sy) +
                                             vaxy * (-(T)0.5 * dx2 * P + dx * sy));
                            v[5] += alpha * (va * (-dxdy) + vax * (dxdy * sx - dy) +
                                             vay * (dxdy * sy - dx) +
                                             vaxy * (-dxdy * P + dy * sy + dx * sx - (T)1));
                            v[6] += alpha * (va * (-(T)0.5 * dy2) + vax * ((T)0.5 * dy2 * sx) +
                                             vay * ((T)0.5 * dy2 * sy - dy) +
                                             vaxy * (-(T)0.5 * dy2 * P + dy * sx));
                            v[10] += vis * va;
                            v[0] += gx;
                            v[1] += gy;
                        }
                    }
                    if (!__any_sync(FULL, ok)) continue;
                    any = true;
                    // v_xy_abs: |sum over this reference warp| (all lanes get the sum)
                    T sx_ = gx, sy_ = gy;
#pragma unroll
                    for (int o = 16; o >= 1; o >>= 1) {
                        sx_ += __shfl_xor_sync(FULL, sx_, o);
                        sy_ += __shfl_xor_sync(FULL, sy_, o);
                    }
                    if (lane == 0) {
                        v[2] += M::abs_(sx_);
                        v[3] += M::abs_(sy_);
                    }
                }
            }
            if (!__any_sync(FULL, any)) continue;
            transpose_reduce16(v, lane);
            int kk = (lane >> 1) & 15;
            if ((lane & 1) == 0 && kk < 11) {
                int gid = __ldg(ids + k);
                out.add(kk, gid, v[0]);
            }
        }
        if (e + 32 < end) st.advance(e, lane);
    }
}

// ------------------------------------------------------------------ host
constexpr int kWarpsPerCta = 4;

template <typename T> struct Cfg;
template <> struct Cfg<float> {
    static constexpr int kFwd = 8, kFwdGA = 4, kBwd = 8, kBwdGA = 4;
};
template <> struct Cfg<double> {
    static constexpr int kFwd = 2, kFwdGA = 2, kBwd = 2, kBwdGA = 2;
};

inline int nblocks_map(int B, bool rank_map) {
    return rank_map ? (B * B + 31) / 32 : ((B + 7) / 8) * ((B + 3) / 4);
}

template <typename T>
int pack(int n, const void *xys, const void *con, const void *col, const void *op, void *ws,
         size_t ws_bytes, cudaStream_t s) {
    if (ws_bytes < sizeof(Rec<T>) * (size_t)n) return LIG_ERR_WORKSPACE;
    if (n > 0)
        pack_kernel<T><<<(n + 255) / 256, 256, 0, s>>>(n, (const T *)xys, (const T *)con,
                                                      (const T *)col, (const T *)op, (Rec<T> *)ws);
    note_launches(n > 0 ? 1 : 0);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

template <typename T>
int raster_fwd(int H, int W, int B, int n, const int32_t *ids, const int32_t *bins,
               const int32_t *d_total, const void *xys, const void *con, const void *col,
               const void *op, void *ws, size_t ws_bytes, void *img, void *wsum, void *dx,
               void *dy, void *dxy, int32_t *fin, cudaStream_t s) {
    int rc = pack<T>(n, xys, con, col, op, ws, ws_bytes, s);
    if (rc) return rc;
    bool ga = dx != nullptr;
    int tbx = (W + B - 1) / B, tby = (H + B - 1) / B;
    int ppl = ga ? Cfg<T>::kFwdGA : Cfg<T>::kFwd;
    int nbands = (nblocks_map(B, false) + ppl - 1) / ppl;
    int nwork = tbx * tby * nbands;
    int grid = (nwork + kWarpsPerCta - 1) / kWarpsPerCta;
    if (ga)
        raster_fwd_kernel<T, true, Cfg<T>::kFwdGA><<<grid, 32 * kWarpsPerCta, 0, s>>>(
            H, W, B, tbx, nbands, nwork, ids, (const int2 *)bins, d_total, (const Rec<T> *)ws,
            (T *)img, (T *)wsum, (T *)dx, (T *)dy, (T *)dxy, fin);
    else
        raster_fwd_kernel<T, false, Cfg<T>::kFwd><<<grid, 32 * kWarpsPerCta, 0, s>>>(
            H, W, B, tbx, nbands, nwork, ids, (const int2 *)bins, d_total, (const Rec<T> *)ws,
            (T *)img, (T *)wsum, nullptr, nullptr, nullptr, fin);
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

template <typename T>
int raster_bwd(int H, int W, int B, int n, const int32_t *ids, const int32_t *bins,
               const int32_t *d_total, const void *xys, const void *con, const void *col,
               const void *op, const int32_t *fin, const void *v_img, const void *v_wsum,
               const void *v_dx, const void *v_dy, const void *v_dxy, double clamp, void *ws,
               size_t ws_bytes, void *v_xy, void *v_abs, void *v_con, void *v_rgb, void *v_op,
               cudaStream_t s) {
    cudaMemsetAsync(v_xy, 0, sizeof(T) * 2 * (size_t)n, s);
    cudaMemsetAsync(v_abs, 0, sizeof(T) * 2 * (size_t)n, s);
    cudaMemsetAsync(v_con, 0, sizeof(T) * 3 * (size_t)n, s);
    cudaMemsetAsync(v_rgb, 0, sizeof(T) * 3 * (size_t)n, s);
    if (v_op) cudaMemsetAsync(v_op, 0, sizeof(T) * (size_t)n, s);
    int rc = pack<T>(n, xys, con, col, op, ws, ws_bytes, s);
    if (rc) return rc;
    bool ga = v_dx != nullptr;
    T cl = (T)(clamp > 0 ? clamp : (ga ? 0.999 : 0.99));
    int tbx = (W + B - 1) / B, tby = (H + B - 1) / B;
    int ppl = ga ? Cfg<T>::kBwdGA : Cfg<T>::kBwd;
    int nbands = (nblocks_map(B, ga) + ppl - 1) / ppl;
    int nwork = tbx * tby * nbands;
    int grid = (nwork + kWarpsPerCta - 1) / kWarpsPerCta;
    Grads<T> g{(T *)v_xy, (T *)v_abs, (T *)v_con, (T *)v_rgb, (T *)v_op};
    if (ga)
        raster_bwd_kernel<T, true, Cfg<T>::kBwdGA><<<grid, 32 * kWarpsPerCta, 0, s>>>(
            H, W, B, tbx, nbands, nwork, ids, (const int2 *)bins, d_total, (const Rec<T> *)ws,
            fin, (const T *)v_img, (const T *)v_wsum, (const T *)v_dx, (const T *)v_dy,
            (const T *)v_dxy, cl, g);
    else
        raster_bwd_kernel<T, false, Cfg<T>::kBwd><<<grid, 32 * kWarpsPerCta, 0, s>>>(
            H, W, B, tbx, nbands, nwork, ids, (const int2 *)bins, d_total, (const Rec<T> *)ws,
            fin, (const T *)v_img, (const T *)v_wsum, nullptr, nullptr, nullptr, cl, g);
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

inline bool raster_args_ok(int H, int W, int B, int n) {
    return H > 0 && W > 0 && B >= 2 && B <= 32 && n >= 0;
}

}  // namespace lig

using namespace lig;

extern "C" size_t lig_raster_workspace_bytes(int dtype, int n) {
    size_t rec = dtype == LIG_F64 ? sizeof(Rec<double>) : sizeof(Rec<float>);
    return rec * (size_t)(n > 0 ? n : 1);
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
        return raster_fwd<float>(H, W, B, n, ids, bins, d_total, xys, con, col, op, ws, ws_bytes,
                                 img, wsum, dx, dy, dxy, fin, s);
    if (dtype == LIG_F64)
        return raster_fwd<double>(H, W, B, n, ids, bins, d_total, xys, con, col, op, ws, ws_bytes,
                                  img, wsum, dx, dy, dxy, fin, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_raster_bwd(int dtype, int H, int W, int B, int n, const int32_t *ids,
                              const int32_t *bins, const int32_t *d_total, const void *xys,
                              const void *con, const void *col, const void *op,
                              const int32_t *fin, const void *v_img, const void *v_wsum,
                              const void *v_dx, const void *v_dy, const void *v_dxy,
                              double clamp, void *ws, size_t ws_bytes, void *v_xy, void *v_abs,
                              void *v_con, void *v_rgb, void *v_op, void *stream) {
    if (!raster_args_ok(H, W, B, n) || !bins || !d_total || !fin || !v_img || !v_wsum || !ws ||
        (n > 0 && (!xys || !con || !col || !v_xy || !v_abs || !v_con || !v_rgb)) ||
        ((v_dx || v_dy || v_dxy) && !(v_dx && v_dy && v_dxy)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) return LIG_OK;
    if (dtype == LIG_F32)
        return raster_bwd<float>(H, W, B, n, ids, bins, d_total, xys, con, col, op, fin, v_img,
                                 v_wsum, v_dx, v_dy, v_dxy, clamp, ws, ws_bytes, v_xy, v_abs,
                                 v_con, v_rgb, v_op, s);
    if (dtype == LIG_F64)
        return raster_bwd<double>(H, W, B, n, ids, bins, d_total, xys, con, col, op, fin, v_img,
                                  v_wsum, v_dx, v_dy, v_dxy, clamp, ws, ws_bytes, v_xy, v_abs,
                                  v_con, v_rgb, v_op, s);
    return LIG_ERR_INVALID;
}
