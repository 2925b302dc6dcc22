// Tile binning: prefix sum of tile counts, key emission, and the ordering
// of the emitted (Gaussian, tile) slots by tile.
//
// The intersection count lives in a device word written by
// lig_cumsum_tiles; every kernel here reads it and bounds its work by the
// caller's capacity, so the whole chain runs without a host round trip (the
// reference reads it back with .item(), gsplat2d/gsplat2d/utils.py:66).
//
// Ordering (default, LIG_BIN_SCATTER): per-tile counters, their exclusive
// scan, an atomic scatter of every slot into its tile's range and a per-tile
// sort by Gaussian index (see "scatter binning" below); workspace: two
// counters per tile.  Alternative kept for comparison: keys are 32-bit tile
// ids (the reference's int64 (tile << 32) | depth keys carry depth 0, so only
// ceil(log2 T) bits hold information) sorted by a stable LSD radix sort over
// exactly those bits with <= 10-bit digits, then tile ranges from the
// boundaries; workspace keys0/vals0/keys1 [capacity], histograms.  Both give
// the order inside a tile of the reference's stable torch.sort: ascending
// Gaussian id (emission order).
#include <algorithm>
#include <atomic>
#include <mutex>

#include "common.cuh"

namespace lig {

// ------------------------------------------------------------------ scan
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096

// Block-wide inclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint32_t block_incl_scan(uint32_t v, uint32_t &total,
                                                    uint32_t *s_warp) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) s_warp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) s_warp[lane] = w;
    }
    __syncthreads();
    total = s_warp[(blockDim.x >> 5) - 1];
    uint32_t add = warp > 0 ? s_warp[warp - 1] : 0;
    __syncthreads();
    return v + add;
}

// Each thread owns kScanItems consecutive elements (loaded warp-striped and
// transposed through registers via shuffles would save little here: the scan
// runs on <= a few MB).  Phase 1: per-block sums.
__global__ void scan_reduce_kernel(const uint32_t *__restrict__ in, int n,
                                   uint32_t *__restrict__ partials) {
    __shared__ uint32_t s_warp[32];
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        if (i < n) acc += in[i];
    }
    uint32_t total;
    block_incl_scan(acc, total, s_warp);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// Phase 2: exclusive scan of the partials by one block (any count).
__global__ void scan_partials_kernel(uint32_t *__restrict__ partials, int nparts) {
    __shared__ uint32_t s_warp[32];
    uint32_t carry = 0;
    for (int base = 0; base < nparts; base += blockDim.x) {
        int i = base + threadIdx.x;
        uint32_t v = i < nparts ? partials[i] : 0;
        uint32_t total;
        uint32_t incl = block_incl_scan(v, total, s_warp);
        if (i < nparts) partials[i] = carry + incl - v;
        carry += total;
    }
}

// Phase 3: rescan each block with its carry-in; inclusive or exclusive output.
// The last element's inclusive value (the grand total) goes to *total_out.
__global__ void scan_final_kernel(const uint32_t *__restrict__ in, int n,
                                  const uint32_t *__restrict__ partials, bool inclusive,
                                  uint32_t *__restrict__ out, int32_t *__restrict__ total_out) {
    __shared__ uint32_t s_warp[32];
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        v[k] = i < n ? in[i] : 0;
        acc += v[k];
    }
    uint32_t total;
    uint32_t incl = block_incl_scan(acc, total, s_warp);
    uint32_t run = partials[blockIdx.x] + incl - acc;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = base + k;
        uint32_t nxt = run + v[k];
        if (i < n) out[i] = inclusive ? nxt : run;
        if (total_out && i == n - 1) *total_out = (int32_t)nxt;
        run = nxt;
    }
}

inline int scan_blocks(int n) { return (n + kScanTile - 1) / kScanTile; }

// Device-wide scan of n u32 values (in may alias out).  partials needs
// scan_blocks(n) words.
inline int device_scan(const uint32_t *in, uint32_t *out, int n, bool inclusive,
                       uint32_t *partials, int32_t *total_out, cudaStream_t s) {
    if (n <= 0) {
        if (total_out) cudaMemsetAsync(total_out, 0, sizeof(int32_t), s);
        return LIG_OK;
    }
    int nb = scan_blocks(n);
    scan_reduce_kernel<<<nb, kScanThreads, 0, s>>>(in, n, partials);
    scan_partials_kernel<<<1, 1024, 0, s>>>(partials, nb);
    scan_final_kernel<<<nb, kScanThreads, 0, s>>>(in, n, partials, inclusive, out, total_out);
    note_launches(3);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

// -------------------------------------------------------------- emission
// One warp per 32 consecutive Gaussians.  The warp flattens their tile slots
// (counts from the inclusive prefix sum) and writes them lane-per-slot, so the
// stores are coalesced and lanes stay busy whatever the per-Gaussian counts.
// Slot j of Gaussian g maps to tile (y0 + j / w, x0 + j % w): row-major over
// the bbox, the emission order of csrc/forward.cu:134-142.  Gaussians whose
// extent is <= 0 but whose count is non-zero get key 0 / id 0 slots — the
// values the reference leaves in its zero-initialised buffers.
template <typename T>
__global__ void emit_kernel(int n, const T *__restrict__ xys, const T *__restrict__ extents,
                            const int32_t *__restrict__ cum, BatchGeo geo, int capacity,
                            uint32_t *__restrict__ keys,
                            int32_t *__restrict__ vals, int64_t *__restrict__ keys64,
                            int32_t *__restrict__ vals_extra, int32_t *__restrict__ status) {
    const unsigned FULL = 0xffffffffu;
    int lane = threadIdx.x & 31;
    int64_t warp_id = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t g0 = warp_id * 32;
    if (g0 >= n) return;
    int g = (int)(g0 + lane);
    int cnt = 0, start = 0, x0 = 0, y0 = 0, bw = 1, bh = 0;
    unsigned tbx = 1, toff = 0, g_first = 0;
    bool valid = false;
    if (g < n) {
        const int im = geo.image_of_gauss(g);
        tbx = geo.tbx[im];
        toff = (unsigned)geo.tile_off[im];
        g_first = (unsigned)geo.g_off[im];
        int prev = g > 0 ? cum[g - 1] : 0;
        start = prev;
        cnt = cum[g] - prev;
        T ex = extents[2 * g], ey = extents[2 * g + 1];
        valid = !(ex <= (T)0 || ey <= (T)0);
        if (valid && cnt > 0) {
            int x1, y1;
            tile_bbox(xys[2 * g], xys[2 * g + 1], ex, ey, tbx, geo.tby(im), geo.B, x0, y0, x1, y1);
            bw = x1 - x0;
            bh = y1 - y0;
            if (bw <= 0 || bw * bh != cnt) {
                // inconsistent inputs: keep emission in range and flag it
                if (status) atomicOr(status, LIG_STATUS_BADBOX);
                valid = false;
                bw = 1;
            }
        }
    }
    // inclusive warp prefix of counts
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    int total = __shfl_sync(FULL, incl, 31);
    bool overflow = false;
    for (int s0 = 0; s0 < total; s0 += 32) {
        int s = s0 + lane;
        // owner = first lane whose inclusive count exceeds s
        int lo = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
            int probe = lo + step - 1;
            int v = __shfl_sync(FULL, incl, probe);
            if (v <= s) lo += step;
        }
        int owner = lo;
        int o_incl = __shfl_sync(FULL, incl, owner);
        int o_cnt = __shfl_sync(FULL, cnt, owner);
        int o_start = __shfl_sync(FULL, start, owner);
        int o_x0 = __shfl_sync(FULL, x0, owner);
        int o_y0 = __shfl_sync(FULL, y0, owner);
        int o_bw = __shfl_sync(FULL, bw, owner);
        int o_valid = __shfl_sync(FULL, (int)valid, owner);
        unsigned o_tbx = __shfl_sync(FULL, tbx, owner);
        unsigned o_toff = __shfl_sync(FULL, toff, owner);
        unsigned o_first = __shfl_sync(FULL, g_first, owner);
        if (s >= total) continue;
        int j = s - (o_incl - o_cnt);
        int slot = o_start + j;
        if (slot >= capacity) {
            overflow = true;
            continue;
        }
        // phantom slots: the image's first tile and first Gaussian (0 / 0 for
        // a single image)
        uint32_t key = o_toff;
        int32_t gid = (int32_t)o_first;
        if (o_valid) {
            int q = j / o_bw;
            int r = j - q * o_bw;
            key = o_toff + (uint32_t)(o_y0 + q) * o_tbx + (uint32_t)(o_x0 + r);
            gid = (int32_t)(g0 + owner);
        }
        if (keys) keys[slot] = key;
        vals[slot] = gid;
        if (keys64) keys64[slot] = (int64_t)key << 32;
        if (vals_extra) vals_extra[slot] = gid;
    }
    if (overflow && status) atomicOr(status, LIG_STATUS_OVERFLOW);
}

// ----------------------------------------------------------------- radix
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;                         // keys per lane
constexpr int kSortTile = kSortThreads * kSortRounds;   // 4096 keys per block
constexpr int kWarpSeg = 32 * kSortRounds;              // 512 keys per warp

__device__ __forceinline__ int bounded_count(const int32_t *d_total, int capacity) {
    int m = *d_total;
    return m < capacity ? m : capacity;
}

// Per-block digit histogram -> hist[d * nblk + blk].
__global__ void radix_upsweep_kernel(const uint32_t *__restrict__ keys, const int32_t *d_total,
                                     int capacity, int shift, int bins,
                                     uint32_t *__restrict__ hist, int nblk) {
    extern __shared__ uint32_t s_hist[];
    for (int i = threadIdx.x; i < bins; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    int m = bounded_count(d_total, capacity);
    int64_t base = (int64_t)blockIdx.x * kSortTile;
    if (base < m) {
#pragma unroll 4
        for (int r = 0; r < kSortRounds; ++r) {
            int64_t i = base + r * kSortThreads + threadIdx.x;
            if (i < m) atomicAdd(&s_hist[(keys[i] >> shift) & (bins - 1)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < bins; i += blockDim.x)
        hist[(int64_t)i * nblk + blockIdx.x] = s_hist[i];
}

// Stable scatter.  Each warp ranks its 512 consecutive keys in 16 rounds of
// 32 with __match_any_sync and per-warp digit counters, so ranks follow input
// order; counters are then prefixed across warps and digits, the block's keys
// are placed in shared memory in sorted order, and written out in runs
// (consecutive threads -> consecutive output positions of one digit).
// Shared layout: wcnt[kSortWarps][bins] | bofs[bins] | gbase[bins] |
//                skeys[4096] | svals[4096].
#ifndef LIG_SORT_MINB
#define LIG_SORT_MINB 4  // resident downsweep blocks per SM asked of the register allocator
#endif
__global__ void __launch_bounds__(kSortThreads, LIG_SORT_MINB)
radix_downsweep_kernel(const uint32_t *__restrict__ keys_in, const int32_t *__restrict__ vals_in,
                       uint32_t *__restrict__ keys_out, int32_t *__restrict__ vals_out,
                       const int32_t *d_total, int capacity, int shift, int bins,
                       const uint32_t *__restrict__ hist_scan, int nblk) {
    extern __shared__ uint32_t smem[];
    uint32_t *wcnt = smem;
    uint32_t *bofs = wcnt + kSortWarps * bins;
    uint32_t *gbase = bofs + bins;
    uint32_t *skeys = gbase + bins;
    int32_t *svals = (int32_t *)(skeys + kSortTile);

    const unsigned FULL = 0xffffffffu;
    int m = bounded_count(d_total, capacity);
    int64_t base = (int64_t)blockIdx.x * kSortTile;
    if (base >= m) return;  // uniform across the block
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * bins; i += blockDim.x) wcnt[i] = 0;
    for (int i = threadIdx.x; i < bins; i += blockDim.x)
        gbase[i] = hist_scan[(int64_t)i * nblk + blockIdx.x];
    __syncthreads();

    // keys in registers; ranks (< 4096) two per register; the values are
    // read again at the scatter (a small register footprint keeps more
    // blocks resident)
    uint32_t k[kSortRounds];
    uint32_t rk2[kSortRounds / 2];
    int64_t wbase = base + warp * kWarpSeg;
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        int64_t i = wbase + r * 32 + lane;
        k[r] = i < m ? keys_in[i] : 0u;
    }
    uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t *my = wcnt + warp * bins;
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        int64_t i = wbase + r * 32 + lane;
        bool ok = i < m;
        uint32_t d = (k[r] >> shift) & (uint32_t)(bins - 1);
        uint32_t peers = __match_any_sync(FULL, ok ? d : 0xffffffffu);
        uint32_t before = __popc(peers & lt_mask);
        uint32_t old = ok ? my[d] : 0u;
        __syncwarp();
        if (ok && before == 0) my[d] = old + __popc(peers);
        __syncwarp();
        const uint32_t rank = old + before;
        if (r & 1) rk2[r >> 1] |= rank << 16;
        else rk2[r >> 1] = rank;
    }
    __syncthreads();
    // exclusive prefix over warps per digit; block digit totals into bofs
    for (int d = threadIdx.x; d < bins; d += blockDim.x) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t t = wcnt[w * bins + d];
            wcnt[w * bins + d] = run;
            run += t;
        }
        bofs[d] = run;
    }
    __syncthreads();
    // exclusive scan of bofs over digits (bins <= 1024 = 4 per thread)
    {
        __shared__ uint32_t s_warp[32];
        int per = (bins + kSortThreads - 1) / kSortThreads;
        int d0 = threadIdx.x * per;
        uint32_t loc[4] = {0, 0, 0, 0};
        uint32_t acc = 0;
        for (int q = 0; q < per; ++q) {
            int d = d0 + q;
            loc[q] = d < bins ? bofs[d] : 0;
            acc += loc[q];
        }
        uint32_t total;
        uint32_t incl = block_incl_scan(acc, total, s_warp);
        uint32_t run = incl - acc;
        for (int q = 0; q < per; ++q) {
            int d = d0 + q;
            if (d < bins) bofs[d] = run;
            run += loc[q];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        int64_t i = wbase + r * 32 + lane;
        if (i < m) {
            uint32_t d = (k[r] >> shift) & (uint32_t)(bins - 1);
            uint32_t pos = bofs[d] + wcnt[warp * bins + d] + ((rk2[r >> 1] >> (16 * (r & 1))) & 0xffffu);
            skeys[pos] = k[r];
            svals[pos] = vals_in[i];
        }
    }
    __syncthreads();
    int nvalid = (int)min((int64_t)kSortTile, (int64_t)m - base);
    for (int i = threadIdx.x; i < nvalid; i += blockDim.x) {
        uint32_t key = skeys[i];
        uint32_t d = (key >> shift) & (uint32_t)(bins - 1);
        uint32_t gpos = gbase[d] + (uint32_t)i - bofs[d];
        keys_out[gpos] = key;
        vals_out[gpos] = svals[i];
    }
}

inline size_t downsweep_smem(int bins) {
    return sizeof(uint32_t) * ((size_t)(kSortWarps + 2) * bins + 2 * kSortTile);
}

// ----------------------------------------------------------- tile ranges
// Boundary detection on sorted keys (csrc/forward.cu:148-170); tile_bins must
// be zeroed first so empty tiles read (0,0).
template <typename K>
__device__ __forceinline__ int32_t key_tile(K k);
template <> __device__ __forceinline__ int32_t key_tile<uint32_t>(uint32_t k) { return (int32_t)k; }
template <> __device__ __forceinline__ int32_t key_tile<int64_t>(int64_t k) { return (int32_t)(k >> 32); }

template <typename K>
__global__ void tile_ranges_kernel(const K *__restrict__ keys, const int32_t *d_total,
                                   int capacity, int m_host, int2 *__restrict__ bins) {
    int m = d_total ? bounded_count(d_total, capacity) : m_host;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    int32_t cur = key_tile<K>(keys[i]);
    if (i == 0) bins[cur].x = 0;
    if (i == m - 1) bins[cur].y = m;
    if (i == 0) return;
    int32_t prev = key_tile<K>(keys[i - 1]);
    if (prev != cur) {
        bins[prev].y = (int)i;
        bins[cur].x = (int)i;
    }
}

// Widen sorted 32-bit tile keys to the reference's int64 layout (tile << 32).
__global__ void widen_keys_kernel(const uint32_t *__restrict__ keys, const int32_t *d_total,
                                  int capacity, int64_t *__restrict__ out) {
    int m = bounded_count(d_total, capacity);
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = (int64_t)keys[i] << 32;
}

__global__ void flag_overflow_kernel(const int32_t *d_total, int capacity, int32_t *status) {
    if (*d_total > capacity) atomicOr(status, LIG_STATUS_OVERFLOW);
}

// ---------------------------------------------------- scatter binning
// Alternative to emission + radix sort + boundary pass (LIG_BIN_SCATTER):
//   1. count: every tile slot of every Gaussian (the emission enumeration
//      above) adds 1 to its tile's counter;
//   2. an exclusive scan of the counters gives each tile's first position;
//   3. scatter: every slot takes the next free position of its tile (an
//      atomic cursor), so a tile's entries are contiguous but in arbitrary
//      order;
//   4. each tile's entries are sorted by Gaussian index, which restores the
//      stable sort's order (ascending Gaussian id within a tile, as the
//      reference's stable torch.sort of (tile << 32) keys in emission
//      order gives), and tile_bins is written from the counts.
// The sort key is twice the Gaussian index; a slot of a Gaussian with
// extent <= 0 (the reference's zero "phantom" slots in the image's first
// tile, which sort at their Gaussian's emission position) adds 1, and is
// written as the image's first Gaussian id after sorting.
#ifndef LIG_BIN_SCATTER
#define LIG_BIN_SCATTER 1
#endif
constexpr uint32_t kPhantom = 1u;  // low bit of the sort key (key = 2 g + phantom)
constexpr int kSegSmem = 4096;     // sorted in shared memory up to this length (long tiles)
constexpr int kSegWarps = 4;       // warps per CTA of the per-tile sort

// The emission enumeration of emit_kernel, calling f(slot, key, sort_value)
// for every slot below `capacity` (slots past it set overflow).
template <typename T, typename F>
__device__ __forceinline__ void for_each_slot(int n, const T *__restrict__ xys,
                                              const T *__restrict__ extents,
                                              const int32_t *__restrict__ cum,
                                              const BatchGeo &geo, int capacity,
                                              int32_t *__restrict__ status, F f) {
    const unsigned FULL = 0xffffffffu;
    int lane = threadIdx.x & 31;
    int64_t warp_id = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t g0 = warp_id * 32;
    if (g0 >= n) return;
    int g = (int)(g0 + lane);
    int cnt = 0, start = 0, x0 = 0, y0 = 0, bw = 1, bh = 0;
    unsigned tbx = 1, toff = 0;
    bool valid = false;
    if (g < n) {
        const int im = geo.image_of_gauss(g);
        tbx = geo.tbx[im];
        toff = (unsigned)geo.tile_off[im];
        int prev = g > 0 ? cum[g - 1] : 0;
        start = prev;
        cnt = cum[g] - prev;
        T ex = extents[2 * g], ey = extents[2 * g + 1];
        valid = !(ex <= (T)0 || ey <= (T)0);
        if (valid && cnt > 0) {
            int x1, y1;
            tile_bbox(xys[2 * g], xys[2 * g + 1], ex, ey, tbx, geo.tby(im), geo.B, x0, y0, x1, y1);
            bw = x1 - x0;
            bh = y1 - y0;
            if (bw <= 0 || bw * bh != cnt) {
                if (status) atomicOr(status, LIG_STATUS_BADBOX);
                valid = false;
                bw = 1;
            }
        }
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    int total = __shfl_sync(FULL, incl, 31);
    bool overflow = false;
    for (int s0 = 0; s0 < total; s0 += 32) {
        int sl = s0 + lane;
        int lo = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
            int probe = lo + step - 1;
            int v = __shfl_sync(FULL, incl, probe);
            if (v <= sl) lo += step;
        }
        int owner = lo;
        int o_incl = __shfl_sync(FULL, incl, owner);
        int o_cnt = __shfl_sync(FULL, cnt, owner);
        int o_start = __shfl_sync(FULL, start, owner);
        int o_x0 = __shfl_sync(FULL, x0, owner);
        int o_y0 = __shfl_sync(FULL, y0, owner);
        int o_bw = __shfl_sync(FULL, bw, owner);
        int o_valid = __shfl_sync(FULL, (int)valid, owner);
        unsigned o_tbx = __shfl_sync(FULL, tbx, owner);
        unsigned o_toff = __shfl_sync(FULL, toff, owner);
        if (sl >= total) continue;
        int j = sl - (o_incl - o_cnt);
        int slot = o_start + j;
        if (slot >= capacity) {
            overflow = true;
            continue;
        }
        uint32_t key = o_toff;
        uint32_t val = ((uint32_t)(g0 + owner) << 1) | kPhantom;
        if (o_valid) {
            int q = j / o_bw;
            int r = j - q * o_bw;
            key = o_toff + (uint32_t)(o_y0 + q) * o_tbx + (uint32_t)(o_x0 + r);
            val = (uint32_t)(g0 + owner) << 1;
        }
        f(slot, key, val);
    }
    if (overflow && status) atomicOr(status, LIG_STATUS_OVERFLOW);
}

// 1. per-tile counts (slots below capacity; the rest is flagged as overflow)
template <typename T>
__global__ void tile_count_kernel(int n, const T *__restrict__ xys, const T *__restrict__ ext,
                                  const int32_t *__restrict__ cum, BatchGeo geo, int capacity,
                                  uint32_t *__restrict__ tcount, int32_t *__restrict__ status) {
    for_each_slot<T>(n, xys, ext, cum, geo, capacity, status,
                     [&](int, uint32_t key, uint32_t) { atomicAdd(&tcount[key], 1u); });
}

// 3. scatter into the tile's range: `cursor` starts as the exclusive scan of
// the counts (each tile's first position) and one atomic per slot returns
// the slot's absolute position; afterwards cursor[t] = start + count.
template <typename T>
__global__ void tile_scatter_kernel(int n, const T *__restrict__ xys, const T *__restrict__ ext,
                                    const int32_t *__restrict__ cum, BatchGeo geo, int capacity,
                                    uint32_t *__restrict__ cursor, uint32_t *__restrict__ out,
                                    int64_t *__restrict__ keys64, int32_t *__restrict__ gids) {
    for_each_slot<T>(n, xys, ext, cum, geo, capacity, nullptr,
                     [&](int slot, uint32_t key, uint32_t val) {
                         out[atomicAdd(&cursor[key], 1u)] = val;
                         if (keys64) {  // the reference's emission-order outputs
                             const bool ph = (val & kPhantom) != 0;
                             const int g = (int)(val >> 1);
                             const int im = geo.image_of_gauss(g);
                             keys64[slot] = ph ? (int64_t)geo.tile_off[im] << 32
                                               : (int64_t)key << 32;
                             gids[slot] = ph ? geo.g_off[im] : g;
                         }
                     });
}

// sort value -> Gaussian id (phantom slots: the image's first Gaussian)
__device__ __forceinline__ int32_t slot_id(uint32_t v, const BatchGeo &geo) {
    const int g = (int)(v >> 1);
    if (!(v & kPhantom)) return (int32_t)g;
    return geo.g_off[geo.image_of_gauss(g)];
}

// Bitonic sort of E * 32 values held E per lane (value k of lane l is
// element k * 32 + l): pairs within a lane are exchanged in registers,
// pairs across lanes with shuffles.
template <int E>
__device__ __forceinline__ void warp_bitonic(uint32_t (&v)[E]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32 * E; size <<= 1) {
#pragma unroll
        for (int j = size >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const int kk = j >> 5;
#pragma unroll
                for (int k = 0; k < E; ++k) {
                    const int k2 = k ^ kk;
                    if (k2 > k) {
                        const bool asc = (((k * 32 + lane) & size) == 0);
                        const uint32_t a = v[k], b = v[k2];
                        const bool sw = asc ? (a > b) : (a < b);
                        v[k] = sw ? b : a;
                        v[k2] = sw ? a : b;
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < E; ++k) {
                    const uint32_t o = __shfl_xor_sync(0xffffffffu, v[k], j);
                    const bool asc = (((k * 32 + lane) & size) == 0);
                    const bool lower = (lane & j) == 0;
                    v[k] = (lower == asc) ? min(v[k], o) : max(v[k], o);
                }
            }
        }
    }
}

template <int E>
__device__ __forceinline__ void sort_segment_regs(uint32_t *seg, int L, int32_t *dst,
                                                  const BatchGeo &geo) {
    const int lane = threadIdx.x & 31;
    uint32_t v[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int i = k * 32 + lane;
        v[k] = i < L ? seg[i] : 0xffffffffu;
    }
    warp_bitonic<E>(v);
    // element k*32+lane of the sorted order
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int i = k * 32 + lane;
        if (i < L) dst[i] = slot_id(v[k], geo);
    }
}

// 4. one warp per tile: sort its entries (from `vals`, written to `ids` as
// Gaussian ids), write tile_bins ((0, 0) for an empty tile, as the
// reference's zero-initialised edges) and, when asked, the sorted 64-bit
// keys.  Tiles of up to 256 entries are sorted in registers; longer ones are
// queued for tile_sort_long_kernel (no shared memory here, so that the
// common short tiles run at full occupancy).
__global__ void __launch_bounds__(32 * kSegWarps)
tile_sort_kernel(BatchGeo geo, const uint32_t *__restrict__ tcount,
                 const uint32_t *__restrict__ tend, int capacity, uint32_t *__restrict__ vals,
                 int32_t *__restrict__ ids, int2 *__restrict__ tile_bins,
                 int64_t *__restrict__ isect_sorted, int32_t *__restrict__ long_list) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int T = geo.total_tiles();
    const int nwarps = gridDim.x * kSegWarps;
    for (int t = blockIdx.x * kSegWarps + w; t < T; t += nwarps) {
        const uint32_t c = tcount[t];
        const uint32_t e = tend[t];  // start + count after the scatter
        const int a = (int)min((uint32_t)capacity, e - c);
        const int b = (int)min((uint32_t)capacity, e);
        if (lane == 0) tile_bins[t] = c ? make_int2(a, b) : make_int2(0, 0);
        const int L = b - a;
        if (L <= 0) continue;
        if (isect_sorted)
            for (int i = lane; i < L; i += 32) isect_sorted[a + i] = (int64_t)t << 32;
        uint32_t *seg = vals + a;
        int32_t *dst = ids + a;
        if (L <= 32) sort_segment_regs<1>(seg, L, dst, geo);
        else if (L <= 64) sort_segment_regs<2>(seg, L, dst, geo);
        else if (L <= 128) sort_segment_regs<4>(seg, L, dst, geo);
        else if (L <= 256) sort_segment_regs<8>(seg, L, dst, geo);
        else if (lane == 0) long_list[1 + atomicAdd(long_list, 1)] = t;
    }
}

// Tiles with more than 256 entries: one CTA per tile.  Up to kSegSmem
// entries are sorted in shared memory (bitonic, padded to a power of two
// with the largest key); longer segments in place in global memory with the
// bitonic sort written with ascending comparators only (each merge starts by
// comparing mirrored positions of its block, then half-cleaners), so the
// padding up to a power of two (conceptually the largest key, always at the
// higher index of a comparator) never moves and is not stored: every
// comparator that reaches past the segment is skipped.
constexpr int kLongThreads = 256;
__global__ void __launch_bounds__(kLongThreads)
tile_sort_long_kernel(BatchGeo geo, const uint32_t *__restrict__ tcount,
                      const uint32_t *__restrict__ tend, int capacity,
                      uint32_t *__restrict__ vals, int32_t *__restrict__ ids,
                      const int32_t *__restrict__ long_list) {
    __shared__ uint32_t s_buf[kSegSmem];
    const int nlong = long_list[0];
    for (int q = blockIdx.x; q < nlong; q += gridDim.x) {
        const int t = long_list[1 + q];
        const int a = (int)min((uint32_t)capacity, tend[t] - tcount[t]);
        const int b = (int)min((uint32_t)capacity, tend[t]);
        const int L = b - a;
        int P = 1;
        while (P < L) P <<= 1;
        const bool smem = P <= kSegSmem;
        uint32_t *seg = smem ? s_buf : vals + a;
        if (smem)
            for (int i = threadIdx.x; i < P; i += blockDim.x)
                s_buf[i] = i < L ? vals[a + i] : 0xffffffffu;
        __syncthreads();
        const int n = smem ? P : L;  // elements that exist
        for (int size = 2; size <= P; size <<= 1) {
            for (int j = size >> 1; j > 0; j >>= 1) {
                for (int p = threadIdx.x; p < P / 2; p += blockDim.x) {
                    int i, k;
                    if (j == size >> 1) {  // mirrored pair of the block
                        const int blk = p / j, o = p - blk * j;
                        i = blk * size + o;
                        k = blk * size + size - 1 - o;
                    } else {  // half-cleaner at distance j
                        i = 2 * p - (p & (j - 1));
                        k = i + j;
                    }
                    if (k >= n) continue;
                    const uint32_t x = seg[i], y = seg[k];
                    if (x > y) {
                        seg[i] = y;
                        seg[k] = x;
                    }
                }
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < L; i += blockDim.x) ids[a + i] = slot_id(seg[i], geo);
        __syncthreads();
    }
}

// ------------------------------------------------------- workspace plan
struct BinPlan {
    int bits, passes, dbits, bins, nblk;
    size_t off_k0, off_v0, off_k1, off_hist, off_part, total;
};

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

inline BinPlan make_plan(int capacity, int num_tiles) {
    BinPlan p{};
    int bits = 0;
    while (bits < 31 && (1ll << bits) < (long long)num_tiles) ++bits;
    p.bits = bits;
    p.passes = (bits + 9) / 10;
    p.dbits = p.passes ? (bits + p.passes - 1) / p.passes : 0;
    p.bins = 1 << p.dbits;
    p.nblk = (capacity + kSortTile - 1) / kSortTile;
    if (p.nblk < 1) p.nblk = 1;
    size_t cap = (size_t)(capacity > 0 ? capacity : 1);
    size_t off = 0;
    p.off_k0 = off; off = align_up(off + 4 * cap);
    p.off_v0 = off; off = align_up(off + 4 * cap);
    p.off_k1 = off; off = align_up(off + 4 * cap);
    size_t hist_n = (size_t)p.bins * p.nblk;
    p.off_hist = off; off = align_up(off + 4 * hist_n);
    size_t nparts = (hist_n + kScanTile - 1) / kScanTile + 1;
    p.off_part = off; off = align_up(off + 4 * nparts);
    p.total = off;
    return p;
}

// Workspace of the scatter path: per-tile counts and cursors (the cursors
// start as the scan of the counts), scan partials, the long-tile list.  The sort keys are scattered
// into gid_sorted itself and sorted in place there.
struct ScatterPlan {
    size_t off_count, off_cursor, off_part, off_long, total;
};

inline ScatterPlan make_scatter_plan(int num_tiles) {
    ScatterPlan p{};
    size_t t = (size_t)(num_tiles > 0 ? num_tiles : 1);
    size_t off = 0;
    p.off_count = off; off = align_up(off + 4 * t);
    p.off_cursor = off; off = align_up(off + 4 * t);
    p.off_part = off; off = align_up(off + 4 * ((t + kScanTile - 1) / kScanTile + 1));
    p.off_long = off; off = align_up(off + 4 * (t + 1));
    p.total = off;
    return p;
}

template <typename T>
int run_bin_scatter(const BatchGeo &geo, const void *xys, const void *ext, const int32_t *cum,
                    const int32_t *d_total, int capacity, void *ws, size_t ws_bytes,
                    int32_t *gid_sorted, int32_t *tile_bins, int64_t *isect, int32_t *gids,
                    int64_t *isect_sorted, int32_t *status, cudaStream_t s) {
    const int n = geo.total_points();
    const int T_ = geo.total_tiles();
    ScatterPlan p = make_scatter_plan(T_);
    if (ws_bytes < p.total) return LIG_ERR_WORKSPACE;
    char *base = (char *)ws;
    uint32_t *tcount = (uint32_t *)(base + p.off_count);
    uint32_t *cursor = (uint32_t *)(base + p.off_cursor);
    uint32_t *part = (uint32_t *)(base + p.off_part);
    int32_t *long_list = (int32_t *)(base + p.off_long);
    cudaMemsetAsync(status, 0, sizeof(int32_t), s);
    if (n == 0 || capacity == 0) {
        cudaMemsetAsync(tile_bins, 0, sizeof(int32_t) * 2 * (size_t)T_, s);
        flag_overflow_kernel<<<1, 1, 0, s>>>(d_total, capacity, status);
        note_launches(1);
        LIG_LAUNCH_CHECK();
        return LIG_OK;
    }
    cudaMemsetAsync(tcount, 0, sizeof(uint32_t) * (size_t)T_, s);
    cudaMemsetAsync(long_list, 0, sizeof(int32_t), s);
    const int warps = (n + 31) / 32;
    const int eblocks = (warps * 32 + 255) / 256;
    tile_count_kernel<T><<<eblocks, 256, 0, s>>>(n, (const T *)xys, (const T *)ext, cum, geo,
                                                 capacity, tcount, status);
    flag_overflow_kernel<<<1, 1, 0, s>>>(d_total, capacity, status);
    note_launches(2);
    LIG_LAUNCH_CHECK();
    int rc = device_scan(tcount, cursor, T_, false, part, nullptr, s);
    if (rc) return rc;
    uint32_t *vals = (uint32_t *)gid_sorted;
    tile_scatter_kernel<T><<<eblocks, 256, 0, s>>>(n, (const T *)xys, (const T *)ext, cum, geo,
                                                   capacity, cursor, vals, isect, gids);
    const int sort_blocks = (int)std::min<int64_t>(((int64_t)T_ + kSegWarps - 1) / kSegWarps,
                                                   148 * 32);
    tile_sort_kernel<<<sort_blocks, 32 * kSegWarps, 0, s>>>(geo, tcount, cursor, capacity, vals,
                                                          gid_sorted, (int2 *)tile_bins,
                                                          isect_sorted, long_list);
    tile_sort_long_kernel<<<148 * 4, kLongThreads, 0, s>>>(geo, tcount, cursor, capacity, vals,
                                                           gid_sorted, long_list);
    note_launches(3);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

template <typename T>
int run_bin(const BatchGeo &geo, const void *xys, const void *ext, const int32_t *cum,
            const int32_t *d_total, int capacity, void *ws, size_t ws_bytes, int32_t *gid_sorted,
            int32_t *tile_bins, int64_t *isect, int32_t *gids, int64_t *isect_sorted,
            int32_t *status, cudaStream_t s) {
    if (LIG_BIN_SCATTER)
        return run_bin_scatter<T>(geo, xys, ext, cum, d_total, capacity, ws, ws_bytes,
                                  gid_sorted, tile_bins, isect, gids, isect_sorted, status, s);
    const int n = geo.total_points();
    const int T_ = geo.total_tiles();
    BinPlan p = make_plan(capacity, T_);
    if (ws_bytes < p.total) return LIG_ERR_WORKSPACE;
    char *base = (char *)ws;
    uint32_t *k0 = (uint32_t *)(base + p.off_k0);
    int32_t *v0 = (int32_t *)(base + p.off_v0);
    uint32_t *k1 = (uint32_t *)(base + p.off_k1);
    uint32_t *hist = (uint32_t *)(base + p.off_hist);
    uint32_t *part = (uint32_t *)(base + p.off_part);

    cudaMemsetAsync(status, 0, sizeof(int32_t), s);
    cudaMemsetAsync(tile_bins, 0, sizeof(int32_t) * 2 * (size_t)T_, s);
    if (n == 0 || capacity == 0) {
        flag_overflow_kernel<<<1, 1, 0, s>>>(d_total, capacity, status);
        note_launches(1);
        LIG_LAUNCH_CHECK();
        return LIG_OK;
    }
    // Ping-pong so that the last pass lands in (k1, gid_sorted).
    uint32_t *ka = (p.passes % 2 == 1) ? k0 : k1;
    int32_t *va = (p.passes % 2 == 1) ? v0 : gid_sorted;
    uint32_t *kb = (p.passes % 2 == 1) ? k1 : k0;
    int32_t *vb = (p.passes % 2 == 1) ? gid_sorted : v0;

    int warps = (n + 31) / 32;
    int eblocks = (warps * 32 + 255) / 256;
    emit_kernel<T><<<eblocks, 256, 0, s>>>(n, (const T *)xys, (const T *)ext, cum, geo, capacity,
                                           ka, va, isect, gids, status);
    flag_overflow_kernel<<<1, 1, 0, s>>>(d_total, capacity, status);
    note_launches(2);
    LIG_LAUNCH_CHECK();

    size_t dsm = downsweep_smem(p.bins);
    if (dsm > 48 * 1024) {
        // opt in once per (device, size): the digit count — and with it the
        // shared memory — depends on the tile count, so a later call may need
        // more than an earlier one; never during a stream capture after the
        // first eager call of that size
        static std::mutex mu;
        static size_t opted[128] = {};
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return LIG_ERR_LAUNCH;
        std::lock_guard<std::mutex> lock(mu);
        if (opted[dev] < dsm) {
            if (cudaFuncSetAttribute(radix_downsweep_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)dsm) != cudaSuccess)
                return LIG_ERR_LAUNCH;
            opted[dev] = dsm;
        }
    }
    int hist_n = p.bins * p.nblk;
    for (int pass = 0; pass < p.passes; ++pass) {
        int shift = pass * p.dbits;
        radix_upsweep_kernel<<<p.nblk, kSortThreads, sizeof(uint32_t) * p.bins, s>>>(
            ka, d_total, capacity, shift, p.bins, hist, p.nblk);
        int rc = device_scan(hist, hist, hist_n, false, part, nullptr, s);
        if (rc) return rc;
        radix_downsweep_kernel<<<p.nblk, kSortThreads, dsm, s>>>(
            ka, va, kb, vb, d_total, capacity, shift, p.bins, hist, p.nblk);
        note_launches(2);
        LIG_LAUNCH_CHECK();
        uint32_t *tk = ka; ka = kb; kb = tk;
        int32_t *tv = va; va = vb; vb = tv;
    }
    // (ka, va) now hold the sorted keys / ids; va == gid_sorted.
    // with zero passes (a single tile) emission already wrote (k1, gid_sorted)
    tile_ranges_kernel<uint32_t><<<(capacity + 255) / 256, 256, 0, s>>>(ka, d_total, capacity, 0,
                                                                      (int2 *)tile_bins);
    if (isect_sorted)
        widen_keys_kernel<<<(capacity + 255) / 256, 256, 0, s>>>(ka, d_total, capacity,
                                                                 isect_sorted);
    note_launches(isect_sorted ? 2 : 1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

}  // namespace lig

using namespace lig;

extern "C" size_t lig_cumsum_workspace_bytes(int n) {
    return sizeof(uint32_t) * ((size_t)scan_blocks(n > 0 ? n : 1) + 1);
}

extern "C" int lig_cumsum_tiles(int n, const int32_t *counts, int32_t *cum, int32_t *total,
                                void *workspace, size_t workspace_bytes, void *stream) {
    if (n < 0 || !total || (n > 0 && (!counts || !cum || !workspace))) return LIG_ERR_INVALID;
    if (workspace_bytes < lig_cumsum_workspace_bytes(n)) return LIG_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        cudaMemsetAsync(total, 0, sizeof(int32_t), s);
        LIG_LAUNCH_CHECK();
        return LIG_OK;
    }
    return device_scan((const uint32_t *)counts, (uint32_t *)cum, n, true, (uint32_t *)workspace,
                       total, s);
}

extern "C" size_t lig_bin_workspace_bytes(int n, int capacity, int num_tiles) {
    (void)n;
    if (LIG_BIN_SCATTER) return make_scatter_plan(num_tiles).total;
    return make_plan(capacity, num_tiles).total;
}

extern "C" int lig_bin(int dtype, int n, const void *xys, const void *ext, const int32_t *cum,
                       const int32_t *d_total, int h, int w, int b, int capacity, void *ws,
                       size_t ws_bytes, int32_t *gid_sorted, int32_t *tile_bins, int64_t *isect,
                       int32_t *gids, int64_t *isect_sorted, int32_t *status, void *stream) {
    if (n < 0 || h <= 0 || w <= 0 || b < 1 || capacity < 0 || !d_total || !tile_bins || !status ||
        (n > 0 && (!xys || !ext || !cum)) || (capacity > 0 && (!gid_sorted || !ws)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const BatchGeo geo = BatchGeo::single(h, w, b, n);
    if (dtype == LIG_F32)
        return run_bin<float>(geo, xys, ext, cum, d_total, capacity, ws, ws_bytes, gid_sorted,
                              tile_bins, isect, gids, isect_sorted, status, s);
    if (dtype == LIG_F64)
        return run_bin<double>(geo, xys, ext, cum, d_total, capacity, ws, ws_bytes, gid_sorted,
                               tile_bins, isect, gids, isect_sorted, status, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_bin_batch(int dtype, int n_img, const int32_t *heights, const int32_t *widths,
                             const int32_t *counts_per_image, int b, const void *xys,
                             const void *ext, const int32_t *cum, const int32_t *d_total,
                             int capacity, void *ws, size_t ws_bytes, int32_t *gid_sorted,
                             int32_t *tile_bins, int32_t *status, void *stream) {
    BatchGeo geo;
    if (!heights || !widths || !counts_per_image ||
        !BatchGeo::make(n_img, heights, widths, counts_per_image, b, geo))
        return LIG_ERR_INVALID;
    const int n = geo.total_points();
    if (capacity < 0 || !d_total || !tile_bins || !status || (n > 0 && (!xys || !ext || !cum)) ||
        (capacity > 0 && (!gid_sorted || !ws)))
        return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == LIG_F32)
        return run_bin<float>(geo, xys, ext, cum, d_total, capacity, ws, ws_bytes, gid_sorted,
                              tile_bins, nullptr, nullptr, nullptr, status, s);
    if (dtype == LIG_F64)
        return run_bin<double>(geo, xys, ext, cum, d_total, capacity, ws, ws_bytes, gid_sorted,
                               tile_bins, nullptr, nullptr, nullptr, status, s);
    return LIG_ERR_INVALID;
}

extern "C" int lig_map_intersects(int dtype, int n, int m, const void *xys, const void *ext,
                                  const int32_t *cum, int tbx, int tby, int b, int64_t *isect,
                                  int32_t *gids, void *stream) {
    if (n < 0 || m < 0 || tbx <= 0 || tby <= 0 || b < 1 || (m > 0 && (!isect || !gids)) ||
        (n > 0 && (!xys || !ext || !cum)))
        return LIG_ERR_INVALID;
    if (n == 0 || m == 0) return LIG_OK;
    cudaStream_t s = (cudaStream_t)stream;
    // reference semantics: slots not written by any Gaussian stay zero
    cudaMemsetAsync(isect, 0, sizeof(int64_t) * (size_t)m, s);
    cudaMemsetAsync(gids, 0, sizeof(int32_t) * (size_t)m, s);
    int warps = (n + 31) / 32;
    int eblocks = (warps * 32 + 255) / 256;
    const BatchGeo geo = BatchGeo::single(tby * b, tbx * b, b, n);
    if (dtype == LIG_F32)
        emit_kernel<float><<<eblocks, 256, 0, s>>>(n, (const float *)xys, (const float *)ext, cum,
                                                   geo, m, nullptr, gids, isect, nullptr, nullptr);
    else if (dtype == LIG_F64)
        emit_kernel<double><<<eblocks, 256, 0, s>>>(n, (const double *)xys, (const double *)ext,
                                                    cum, geo, m, nullptr, gids, isect, nullptr,
                                                    nullptr);
    else
        return LIG_ERR_INVALID;
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

extern "C" int lig_tile_bin_edges(int m, const int64_t *isect_sorted, int num_tiles,
                                  int32_t *tile_bins, void *stream) {
    if (m < 0 || num_tiles <= 0 || !tile_bins || (m > 0 && !isect_sorted)) return LIG_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(tile_bins, 0, sizeof(int32_t) * 2 * (size_t)num_tiles, s);
    if (m > 0)
        tile_ranges_kernel<int64_t><<<(m + 255) / 256, 256, 0, s>>>(isect_sorted, nullptr, m, m,
                                                                    (int2 *)tile_bins);
    note_launches(m > 0 ? 1 : 0);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}
