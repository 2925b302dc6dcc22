// Tile binning: prefix sum of tile counts, key emission, and the ordering
// of the emitted (Gaussian, tile) slots by tile.
//
// The intersection count lives in a device word written by
// lig_cumsum_tiles (one single-pass look-back scan kernel); every kernel here
// reads it and bounds its work by the caller's capacity, so the whole chain
// runs without a host round trip (the reference reads it back with .item(),
// gsplat2d/gsplat2d/utils.py:66).
//
// Ordering (default, LIG_BIN_SCATTER): per-tile counters, their exclusive
// scan, an atomic scatter of every slot into its tile's range and a per-tile
// sort by Gaussian index (see "scatter binning" below); workspace: two
// counters per tile, the scan state and the long-tile list.  Alternative kept for comparison: keys are 32-bit tile
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

// Single-pass scan with decoupled look-back.  Each CTA takes a ticket (the
// order in which CTAs started), scans its kScanTile values and publishes its
// aggregate in a 64-bit state word (flag in the high half: 1 = aggregate,
// 2 = inclusive prefix); warp 0 then reads its predecessors' words 32 at a
// time, nearest first, summing aggregates until it meets an inclusive
// prefix, and publishes its own inclusive prefix.  A CTA only waits on CTAs
// holding earlier tickets, which are already running, and each wait is
// bounded (kScanWaitCycles of SM clock): a CTA that gives up sums its
// predecessors' inputs directly instead, so the result is exact either way.
// state: scan_state_words(n) words, zeroed before the launch (the last word
// holds the ticket counter).
constexpr uint64_t kScanFlagAgg = 1ull << 32;
constexpr uint64_t kScanFlagPre = 2ull << 32;
constexpr long long kScanWaitCycles = 1ll << 20;

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t *p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Exclusive prefix of CTA `tile` from its predecessors' state words (warp 0,
// all lanes; the result is uniform).  false: the wait gave up.
__device__ __forceinline__ bool scan_look_back(const uint64_t *state, int tile,
                                               uint32_t &excl) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    excl = 0;
    int p0 = tile - 1;
    const long long t0 = clock64();
    for (;;) {
        const int p = p0 - lane;
        const uint64_t w = p >= 0 ? ld_relaxed_u64(&state[p]) : kScanFlagPre;
        const uint32_t flag = (uint32_t)(w >> 32);
        const unsigned pre = __ballot_sync(FULL, flag == 2u);
        const unsigned none = __ballot_sync(FULL, flag == 0u);
        // lanes up to and including the nearest inclusive prefix
        const unsigned upto = pre ? ((pre & (0u - pre)) << 1) - 1u : FULL;
        if (none & upto) {
            if (__any_sync(FULL, clock64() - t0 > kScanWaitCycles)) return false;
            continue;
        }
        uint32_t x = ((upto >> lane) & 1u) ? (uint32_t)w : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
        excl += x;
        if (pre) return true;
        p0 -= 32;
    }
}

__global__ void __launch_bounds__(kScanThreads)
scan_kernel(const uint32_t *__restrict__ in, int n, uint32_t *__restrict__ out, bool inclusive,
            int32_t *__restrict__ total_out, uint64_t *__restrict__ state,
            uint32_t *__restrict__ ticket) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_tile, s_prefix;
    __shared__ int s_ok;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const int tile = (int)s_tile;
    const int64_t base = (int64_t)tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
    const bool full = base + kScanItems <= n;
    uint32_t v[kScanItems];
    if (full && (reinterpret_cast<uintptr_t>(in) & 15) == 0) {
        const uint4 *q = reinterpret_cast<const uint4 *>(in + base);
#pragma unroll
        for (int k = 0; k < kScanItems / 4; ++k) {
            const uint4 x = q[k];
            v[4 * k] = x.x;
            v[4 * k + 1] = x.y;
            v[4 * k + 2] = x.z;
            v[4 * k + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = base + k < n ? in[base + k] : 0u;
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) acc += v[k];
    uint32_t total;
    const uint32_t incl = block_incl_scan(acc, total, s_warp);
    if (threadIdx.x < 32) {
        uint32_t excl = 0;
        bool ok = true;
        if (tile == 0) {
            if (threadIdx.x == 0) st_relaxed_u64(&state[0], kScanFlagPre | total);
        } else {
            if (threadIdx.x == 0) st_relaxed_u64(&state[tile], kScanFlagAgg | total);
            ok = scan_look_back(state, tile, excl);
        }
        if (threadIdx.x == 0) {
            s_ok = ok;
            s_prefix = excl;
        }
    }
    __syncthreads();
    if (!s_ok) {  // the wait gave up: sum the predecessors' inputs here
        uint32_t part = 0;
        const int64_t lim = (int64_t)tile * kScanTile;
        for (int64_t i = threadIdx.x; i < lim; i += blockDim.x) part += in[i];
        uint32_t sum;
        block_incl_scan(part, sum, s_warp);
        if (threadIdx.x == 0) s_prefix = sum;
        __syncthreads();
    }
    if (threadIdx.x == 0 && tile > 0) st_relaxed_u64(&state[tile], kScanFlagPre | (s_prefix + total));
    uint32_t run = s_prefix + incl - acc;
    if (full && (reinterpret_cast<uintptr_t>(out) & 15) == 0) {
        uint32_t o[kScanItems];
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const uint32_t nxt = run + v[k];
            o[k] = inclusive ? nxt : run;
            run = nxt;
        }
        uint4 *q = reinterpret_cast<uint4 *>(out + base);
#pragma unroll
        for (int k = 0; k < kScanItems / 4; ++k)
            q[k] = make_uint4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
        if (total_out && base + kScanItems == n) *total_out = (int32_t)run;
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const int64_t i = base + k;
            const uint32_t nxt = run + v[k];
            if (i < n) out[i] = inclusive ? nxt : run;
            if (total_out && i == n - 1) *total_out = (int32_t)nxt;
            run = nxt;
        }
    }
}

inline int scan_blocks(int n) { return (n + kScanTile - 1) / kScanTile; }

// 64-bit state words of a scan of n values (one per CTA + the ticket)
inline size_t scan_state_words(int n) { return (size_t)scan_blocks(n > 0 ? n : 1) + 1; }

// Device-wide scan of n u32 values (in and out must not overlap).  state:
// scan_state_words(n) words; zeroed here unless the caller already did
// (`zeroed`, e.g. with a neighbouring buffer in one memset).
inline int device_scan(const uint32_t *in, uint32_t *out, int n, bool inclusive,
                       uint64_t *state, int32_t *total_out, cudaStream_t s,
                       bool zeroed = false) {
    if (n <= 0) {
        if (total_out) cudaMemsetAsync(total_out, 0, sizeof(int32_t), s);
        return LIG_OK;
    }
    const int nb = scan_blocks(n);
    if (!zeroed) cudaMemsetAsync(state, 0, sizeof(uint64_t) * scan_state_words(n), s);
    scan_kernel<<<nb, kScanThreads, 0, s>>>(in, n, out, inclusive, total_out, state,
                                            reinterpret_cast<uint32_t *>(state + nb));
    note_launches(1);
    LIG_LAUNCH_CHECK();
    return LIG_OK;
}

// -------------------------------------------------------------- emission
// Slot j of Gaussian g (j < num_tiles_hit[g], its slots numbered from
// cum[g - 1]) maps to tile (y0 + j / w, x0 + j % w): row-major over the
// bbox, the emission order of csrc/forward.cu:134-142.  A Gaussian whose
// extent is <= 0 but whose count is non-zero has "phantom" slots: tile 0 of
// its image and the image's first Gaussian id (0 / 0 for a single image),
// the values the reference leaves in its zero-initialised buffers.
//
// Every slot carries a sort value 2 g + phantom (the scatter path sorts by it
// within a tile: ascending Gaussian id, phantoms at their Gaussian's place).
constexpr uint32_t kPhantom = 1u;  // low bit of the sort value

// sort value -> Gaussian id (phantom slots: the image's first Gaussian)
__device__ __forceinline__ int32_t slot_id(uint32_t v, const BatchGeo &geo) {
    const int g = (int)(v >> 1);
    if (!(v & kPhantom)) return (int32_t)g;
    return geo.g_off[geo.image_of_gauss(g)];
}

// One warp per 32 consecutive Gaussians hands out their tile slots
// lane-per-slot: the warp flattens its Gaussians' slots, so lanes stay busy
// whatever the per-Gaussian counts and consecutive lanes touch neighbouring
// tiles.  SlotWarp holds each lane's Gaussian (its first slot in the warp's
// flattened order, slot base, first tile, bbox width, row stride and
// reciprocal); slot_at(sl) finds the owner of flattened slot sl with a
// 5-step search over the inclusive count prefix, takes six broadcasts from
// it, and computes the bbox row as a multiply-high by ceil(2^32 / w) — exact
// while count * w <= 2^32, an integer division beyond.  A phantom slot is a
// bbox of width 1 and row stride -1, so its key stays on the first tile.
struct SlotWarp {
    int64_t g0;
    int incl, excl, slot_base, bw, stride, total;
    uint32_t base, magic;
};

template <typename T>
__device__ __forceinline__ bool slot_warp(int n, const T *__restrict__ xys,
                                          const T *__restrict__ extents,
                                          const int32_t *__restrict__ cum, const BatchGeo &geo,
                                          int32_t *__restrict__ status, SlotWarp &sw) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    sw.g0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
    if (sw.g0 >= n) return false;
    const int g = (int)(sw.g0 + lane);
    int cnt = 0, start = 0;
    sw.bw = 1;
    sw.stride = -1;
    sw.base = 0;
    sw.magic = 0;
    if (g < n) {
        const int im = geo.image_of_gauss(g);
        const int tbx = geo.tbx[im];
        sw.base = (uint32_t)geo.tile_off[im];
        const int prev = g > 0 ? cum[g - 1] : 0;
        start = prev;
        cnt = cum[g] - prev;
        const T ex = extents[2 * g], ey = extents[2 * g + 1];
        if (!(ex <= (T)0 || ey <= (T)0) && cnt > 0) {
            int x0, y0, x1, y1;
            tile_bbox(xys[2 * g], xys[2 * g + 1], ex, ey, tbx, geo.tby(im), geo.B, x0, y0, x1, y1);
            const int w = x1 - x0, h = y1 - y0;
            if (w <= 0 || w * h != cnt) {
                // inconsistent inputs: emit phantoms (in range) and flag it
                if (status) atomicOr(status, LIG_STATUS_BADBOX);
            } else {
                sw.bw = w;
                sw.stride = tbx - w;
                sw.base += (uint32_t)y0 * (uint32_t)tbx + (uint32_t)x0;
                if (w > 1 && (uint64_t)cnt * (uint64_t)w <= 0xffffffffull)
                    sw.magic = 0xffffffffu / (uint32_t)w + 1u;
            }
        }
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    sw.incl = incl;
    sw.total = __shfl_sync(FULL, incl, 31);
    sw.excl = incl - cnt;
    sw.slot_base = start - sw.excl;
    return true;
}

// Flattened slot sl of the warp (all lanes call it together): false when sl
// is past the warp's slots; otherwise the slot number, tile key and sort
// value (2 g + phantom).
__device__ __forceinline__ bool slot_at(const SlotWarp &sw, int sl, int &slot, uint32_t &key,
                                        uint32_t &val) {
    const unsigned FULL = 0xffffffffu;
    int lo = 0;  // owner = first lane whose inclusive count exceeds sl
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        const int v = __shfl_sync(FULL, sw.incl, lo + step - 1);
        if (v <= sl) lo += step;
    }
    const int o_excl = __shfl_sync(FULL, sw.excl, lo);
    const int o_sb = __shfl_sync(FULL, sw.slot_base, lo);
    const uint32_t o_base = __shfl_sync(FULL, sw.base, lo);
    const int o_bw = __shfl_sync(FULL, sw.bw, lo);
    const int o_stride = __shfl_sync(FULL, sw.stride, lo);
    const uint32_t o_magic = __shfl_sync(FULL, sw.magic, lo);
    if (sl >= sw.total) return false;
    slot = sl + o_sb;
    const uint32_t j = (uint32_t)(sl - o_excl);
    uint32_t q;  // bbox row of slot j
    if (o_bw == 1) q = j;
    else if (o_magic) q = __umulhi(j, o_magic);
    else q = j / (uint32_t)o_bw;
    key = o_base + j + q * (uint32_t)o_stride;
    val = ((uint32_t)(sw.g0 + lo) << 1) | (o_stride < 0 ? kPhantom : 0u);
    return true;
}

// f(slot, tile key, sort value) for every slot below `capacity` (slots past
// it set LIG_STATUS_OVERFLOW).
template <typename T, typename F>
__device__ __forceinline__ void for_each_slot(int n, const T *__restrict__ xys,
                                              const T *__restrict__ extents,
                                              const int32_t *__restrict__ cum,
                                              const BatchGeo &geo, int capacity,
                                              int32_t *__restrict__ status, F f) {
    SlotWarp sw;
    if (!slot_warp<T>(n, xys, extents, cum, geo, status, sw)) return;
    const int lane = threadIdx.x & 31;
    bool overflow = false;
    for (int s0 = 0; s0 < sw.total; s0 += 32) {
        int slot;
        uint32_t key, val;
        if (!slot_at(sw, s0 + lane, slot, key, val)) continue;
        if (slot >= capacity) {
            overflow = true;
            continue;
        }
        f(slot, key, val);
    }
    if (overflow && status) atomicOr(status, LIG_STATUS_OVERFLOW);
}

// Emission in slot order: 32-bit tile keys and/or Gaussian ids, optionally
// the reference's int64 keys (tile << 32) and a second copy of the ids.
template <typename T>
__global__ void emit_kernel(int n, const T *__restrict__ xys, const T *__restrict__ extents,
                            const int32_t *__restrict__ cum, BatchGeo geo, int capacity,
                            uint32_t *__restrict__ keys,
                            int32_t *__restrict__ vals, int64_t *__restrict__ keys64,
                            int32_t *__restrict__ vals_extra, int32_t *__restrict__ status) {
    for_each_slot<T>(n, xys, extents, cum, geo, capacity, status,
                     [&](int slot, uint32_t key, uint32_t v) {
                         const int32_t gid = slot_id(v, geo);
                         if (keys) keys[slot] = key;
                         if (vals) vals[slot] = gid;
                         if (keys64) keys64[slot] = (int64_t)key << 32;
                         if (vals_extra) vals_extra[slot] = gid;
                     });
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
#ifndef LIG_SORT_LONG_CTAS_PER_SM
#define LIG_SORT_LONG_CTAS_PER_SM 8  // CTAs per SM of the long-tile sort (one tile per CTA at a time)
#endif
#ifndef LIG_SORT_REG512
#define LIG_SORT_REG512 1  // tiles of 257..512 entries sorted by a warp in registers
#endif
constexpr int kSegSmem = 4096;     // sorted in shared memory up to this length (long tiles)
#ifndef LIG_BIN_SORT_WARPS
#define LIG_BIN_SORT_WARPS 8  // measured: 8 warps per CTA 0.258 ms, 4: 0.260, 2: 0.266 (bin, 8192^2)
#endif
constexpr int kSegWarps = LIG_BIN_SORT_WARPS;  // warps per CTA of the per-tile sort

// 1. per-tile counts (slots below capacity; the rest is flagged as overflow,
// as is a total above the capacity)
template <typename T>
__global__ void tile_count_kernel(int n, const T *__restrict__ xys, const T *__restrict__ ext,
                                  const int32_t *__restrict__ cum, const int32_t *d_total,
                                  BatchGeo geo, int capacity, uint32_t *__restrict__ tcount,
                                  int32_t *__restrict__ status) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && *d_total > capacity)
        atomicOr(status, LIG_STATUS_OVERFLOW);
    for_each_slot<T>(n, xys, ext, cum, geo, capacity, status,
                     [&](int, uint32_t key, uint32_t) { atomicAdd(&tcount[key], 1u); });
}

// 3. scatter into the tile's range: `cursor` starts as the exclusive scan of
// the counts (each tile's first position) and one atomic per slot returns
// the slot's absolute position; afterwards cursor[t] = start + count.
// Each lane takes LIG_BIN_SCATTER_ILP slots per trip (32 apart) and issues
// all their atomics before any store, so that many atomic round trips are in
// flight per lane.
#ifndef LIG_BIN_SCATTER_ILP
#define LIG_BIN_SCATTER_ILP 2  // 3 and 4 measured no faster
#endif
template <typename T>
__global__ void tile_scatter_kernel(int n, const T *__restrict__ xys, const T *__restrict__ ext,
                                    const int32_t *__restrict__ cum, BatchGeo geo, int capacity,
                                    uint32_t *__restrict__ cursor, uint32_t *__restrict__ out,
                                    int64_t *__restrict__ keys64, int32_t *__restrict__ gids) {
    constexpr int K = LIG_BIN_SCATTER_ILP;
    SlotWarp sw;
    if (!slot_warp<T>(n, xys, ext, cum, geo, nullptr, sw)) return;
    const int lane = threadIdx.x & 31;
    for (int s0 = 0; s0 < sw.total; s0 += 32 * K) {
        int sl[K];
        uint32_t key[K], val[K], pos[K];
        bool ok[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            ok[k] = slot_at(sw, s0 + 32 * k + lane, sl[k], key[k], val[k]);
            ok[k] = ok[k] && sl[k] < capacity;
        }
#pragma unroll
        for (int k = 0; k < K; ++k) pos[k] = ok[k] ? atomicAdd(&cursor[key[k]], 1u) : 0u;
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (ok[k]) out[pos[k]] = val[k];
        if (keys64) {  // the reference's emission-order outputs
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (ok[k]) {
                    keys64[sl[k]] = (int64_t)key[k] << 32;
                    gids[sl[k]] = slot_id(val[k], geo);
                }
        }
    }
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
// keys.  Tiles of up to 512 entries are sorted in registers (16 a lane at
// most: 48 registers, no block barriers); longer ones are queued for
// tile_sort_long_kernel (no shared memory here, so that the common short
// tiles run at high occupancy).  At config 1's level-1 density (2048^2, 1M
// Gaussians, about 360 entries a tile) sorting 257..512-entry tiles here
// instead of one CTA per tile took the binning from 0.41 to 0.17 ms.
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
#if LIG_SORT_REG512
        else if (L <= 512) sort_segment_regs<16>(seg, L, dst, geo);
#endif
        else if (lane == 0) long_list[1 + atomicAdd(long_list, 1)] = t;
    }
}

// Tiles with more than 512 entries: one CTA per tile, 8 CTAs per SM (0.58 ->
// 0.41 ms binning at 2048^2 / 1M against 2, when this kernel also took the
// 257..512-entry tiles).  Up to kSegSmem
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
    size_t off_k0, off_v0, off_k1, off_hist, off_hscan, off_part, total;
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
    p.off_hscan = off; off = align_up(off + 4 * hist_n);
    p.off_part = off; off = align_up(off + 8 * scan_state_words((int)hist_n));
    p.total = off;
    return p;
}

// Workspace of the scatter path: per-tile counts, the scan state, the
// long-tile list (its first word is the length) and the per-tile cursors
// (they start as the scan of the counts).  The first three are adjacent so
// that one memset clears the counts, the scan state and the list length.
// The sort keys are scattered into gid_sorted itself and sorted in place.
struct ScatterPlan {
    size_t off_count, off_part, off_long, off_cursor, total;
};

inline ScatterPlan make_scatter_plan(int num_tiles) {
    ScatterPlan p{};
    size_t t = (size_t)(num_tiles > 0 ? num_tiles : 1);
    size_t off = 0;
    p.off_count = off; off = align_up(off + 4 * t);
    p.off_part = off; off = align_up(off + 8 * scan_state_words((int)t));
    p.off_long = off; off = align_up(off + 4 * (t + 1));
    p.off_cursor = off; off = align_up(off + 4 * t);
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
    uint64_t *part = (uint64_t *)(base + p.off_part);
    int32_t *long_list = (int32_t *)(base + p.off_long);
    cudaMemsetAsync(status, 0, sizeof(int32_t), s);
    if (n == 0 || capacity == 0) {
        cudaMemsetAsync(tile_bins, 0, sizeof(int32_t) * 2 * (size_t)T_, s);
        flag_overflow_kernel<<<1, 1, 0, s>>>(d_total, capacity, status);
        note_launches(1);
        LIG_LAUNCH_CHECK();
        return LIG_OK;
    }
    // counts, scan state and the long-list length in one memset
    cudaMemsetAsync(tcount, 0, p.off_long + sizeof(int32_t) - p.off_count, s);
    const int warps = (n + 31) / 32;
    const int eblocks = (warps * 32 + 255) / 256;
    tile_count_kernel<T><<<eblocks, 256, 0, s>>>(n, (const T *)xys, (const T *)ext, cum, d_total,
                                                 geo, capacity, tcount, status);
    note_launches(1);
    LIG_LAUNCH_CHECK();
    int rc = device_scan(tcount, cursor, T_, false, part, nullptr, s, /*zeroed=*/true);
    if (rc) return rc;
    uint32_t *vals = (uint32_t *)gid_sorted;
    tile_scatter_kernel<T><<<eblocks, 256, 0, s>>>(n, (const T *)xys, (const T *)ext, cum, geo,
                                                   capacity, cursor, vals, isect, gids);
    const int sort_blocks = (int)std::min<int64_t>(((int64_t)T_ + kSegWarps - 1) / kSegWarps,
                                                   148 * 32);
    tile_sort_kernel<<<sort_blocks, 32 * kSegWarps, 0, s>>>(geo, tcount, cursor, capacity, vals,
                                                          gid_sorted, (int2 *)tile_bins,
                                                          isect_sorted, long_list);
    tile_sort_long_kernel<<<148 * LIG_SORT_LONG_CTAS_PER_SM, kLongThreads, 0, s>>>(
        geo, tcount, cursor, capacity, vals, gid_sorted, long_list);
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
    uint32_t *hscan = (uint32_t *)(base + p.off_hscan);
    uint64_t *part = (uint64_t *)(base + p.off_part);

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
        int rc = device_scan(hist, hscan, hist_n, false, part, nullptr, s);
        if (rc) return rc;
        radix_downsweep_kernel<<<p.nblk, kSortThreads, dsm, s>>>(
            ka, va, kb, vb, d_total, capacity, shift, p.bins, hscan, p.nblk);
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
    return sizeof(uint64_t) * scan_state_words(n);
}

extern "C" int lig_cumsum_tiles(int n, const int32_t *counts, int32_t *cum, int32_t *total,
                                void *workspace, size_t workspace_bytes, void *stream) {
    if (n < 0 || !total || (n > 0 && (!counts || !cum || !workspace))) return LIG_ERR_INVALID;
    // the scan reads its predecessors' inputs when a wait gives up: no aliasing
    if (n > 0 && (const char *)counts < (const char *)(cum + n) &&
        (const char *)cum < (const char *)(counts + n))
        return LIG_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(workspace) & 7) != 0) return LIG_ERR_INVALID;
    if (workspace_bytes < lig_cumsum_workspace_bytes(n)) return LIG_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        cudaMemsetAsync(total, 0, sizeof(int32_t), s);
        LIG_LAUNCH_CHECK();
        return LIG_OK;
    }
    return device_scan((const uint32_t *)counts, (uint32_t *)cum, n, true, (uint64_t *)workspace,
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
