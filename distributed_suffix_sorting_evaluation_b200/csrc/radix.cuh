// Onesweep LSD radix sort over multi-word keys (KW little-endian uint32 words,
// structure-of-arrays) carrying one uint32 value.  Replaces the reference's
// distributed comparison sorts (lightweight_dcx/src/sorters/sorting_wrapper.hpp:57-94,
// sample_sort.hpp:36-171) for every sort of the DCX pipeline.
//
// One kernel per 8-bit digit:
//   * tiles are claimed in order through an atomic counter;
//   * each warp ranks its items with __match_any_sync against a per-warp
//     digit histogram in shared memory;
//   * the tile's per-digit counts are published to a look-back array and each
//     digit's global offset is found by decoupled look-back; every wait is
//     bounded and, when exhausted, sets an error bit and lets the CTA finish;
//   * keys and values are exchanged through shared memory into digit order so
//     that global writes of one digit run are contiguous.
// Global digit offsets for every pass come from one up-front histogram that the
// key producer fuses into its own pass (no extra read of the keys).
#pragma once

#include "common.cuh"

namespace dcx {

constexpr int RADIX_BITS = 8;
constexpr int RADIX = 1 << RADIX_BITS;
constexpr int SORT_THREADS = 256;  // one thread per digit in the look-back
constexpr int MAX_KEY_WORDS = 12;

// Look-back status word: [63:34] epoch, [33:32] flag (1 aggregate, 2 inclusive), [31:0] count.
__device__ __forceinline__ uint64_t lb_pack(uint32_t epoch, uint32_t flag, uint32_t v) {
    return ((uint64_t)epoch << 34) | ((uint64_t)flag << 32) | v;
}

__device__ __forceinline__ void st_relaxed(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

struct SortPassArgs {
    const uint32_t* keys_in[MAX_KEY_WORDS];
    uint32_t* keys_out[MAX_KEY_WORDS];
    const uint32_t* vals_in;
    uint32_t* vals_out;
    uint32_t kw;                  // key words carried
    uint64_t n;
    uint32_t shift;               // bit position of the digit (multiple of 8)
    const uint32_t* digit_base;   // [RADIX] exclusive global offsets of this pass
    uint64_t* lookback;           // [tiles][RADIX]
    uint32_t* tile_counter;       // zeroed before the pass
    uint32_t epoch;
    uint32_t* err;
    uint32_t spin_limit;
};

template <int ITEMS>
__global__ __launch_bounds__(SORT_THREADS) void k_onesweep(SortPassArgs a) {
    constexpr int THREADS = SORT_THREADS;
    constexpr int WARPS = THREADS / 32;
    constexpr int TILE = THREADS * ITEMS;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_hist[WARPS][RADIX];
    __shared__ uint32_t s_tile_excl[RADIX];
    __shared__ uint32_t s_gbase[RADIX];
    __shared__ uint32_t s_scan[THREADS / 32 + 1];
    __shared__ uint32_t s_exch[TILE];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    for (int i = tid; i < WARPS * RADIX; i += THREADS) (&s_warp_hist[0][0])[i] = 0;
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t tile_base = tile * TILE;
    const uint64_t remain = a.n - tile_base;
    const uint32_t tile_valid = remain < (uint64_t)TILE ? (uint32_t)remain : (uint32_t)TILE;
    const int wd = a.shift >> 5, sh = a.shift & 31;

    // 1. load digits (warp-striped: item it of lane l of warp w is element
    //    w*32*ITEMS + it*32 + l of the tile) and rank inside the warp.
    uint32_t pos[ITEMS];  // first: rank in warp, later: local position in tile
    uint32_t dig[ITEMS];
    const uint32_t* kin = a.keys_in[wd];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        dig[it] = e < tile_valid ? (__ldg(kin + tile_base + e) >> sh) & (RADIX - 1) : RADIX;
    }
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t d = dig[it];
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & lanemask_lt());
        uint32_t cnt = 0;
        if (d < RADIX) cnt = s_warp_hist[warp][d];
        pos[it] = cnt + before;
        __syncwarp();
        if (d < RADIX && before == 0) s_warp_hist[warp][d] = cnt + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // 2. per digit: warp prefix, tile count, tile-local digit offsets.
    uint32_t count = 0;
    {
        const int d = tid;  // THREADS == RADIX
#pragma unroll
        for (int w = 0; w < WARPS; w++) {
            uint32_t t = s_warp_hist[w][d];
            s_warp_hist[w][d] = count;
            count += t;
        }
        uint32_t total;
        uint32_t ex = block_excl_scan<THREADS>(count, s_scan, total);
        s_tile_excl[d] = ex;

        // 3. decoupled look-back for digit d.
        uint64_t* my = a.lookback + tile * RADIX + d;
        uint32_t excl = 0;
        if (tile == 0) {
            st_relaxed(my, lb_pack(a.epoch, 2u, count));
        } else {
            st_relaxed(my, lb_pack(a.epoch, 1u, count));
            int64_t t = (int64_t)tile - 1;
            uint32_t spins = 0;
            while (t >= 0) {
                uint64_t v = ld_relaxed(a.lookback + (uint64_t)t * RADIX + d);
                uint32_t ep = (uint32_t)(v >> 34), fl = (uint32_t)(v >> 32) & 3u;
                if (ep != a.epoch || fl == 0) {
                    if (++spins > a.spin_limit) {  // give up: flag and finish cleanly
                        atomicOr(a.err, DEV_ERR_TIMEOUT);
                        break;
                    }
                    if (spins > 64) __nanosleep(64);
                    continue;
                }
                excl += (uint32_t)v;
                if (fl == 2u) break;
                t--;
            }
            st_relaxed(my, lb_pack(a.epoch, 2u, excl + count));
        }
        s_gbase[d] = a.digit_base[d] + excl - ex;
    }
    __syncthreads();

    // local position of every item in the digit-sorted tile
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t d = dig[it];
        if (d < RADIX) pos[it] += s_tile_excl[d] + s_warp_hist[warp][d];
    }

    // 4. exchange the digit word first to learn every sorted slot's destination.
    uint32_t dst[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++)
        if (dig[it] < RADIX) s_exch[pos[it]] = __ldg(kin + tile_base + warp * 32 * ITEMS + it * 32 + lane);
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        uint32_t j = it * THREADS + tid;
        if (j < tile_valid) {
            uint32_t w = s_exch[j];
            uint32_t d = (w >> sh) & (RADIX - 1);
            dst[it] = s_gbase[d] + j;  // modulo 2^32: s_gbase may wrap, the sum does not
            if (dst[it] < a.n) a.keys_out[wd][dst[it]] = w;
            else atomicOr(a.err, DEV_ERR_RANGE);  // only after a timed-out look-back
        }
    }
    __syncthreads();

    // 5. the remaining key words and the values follow the same permutation.
    const int kw = (int)a.kw;
    for (int w = 0; w <= kw; w++) {
        if (w == wd) continue;
        const uint32_t* src = w < kw ? a.keys_in[w] : a.vals_in;
        uint32_t* out = w < kw ? a.keys_out[w] : a.vals_out;
#pragma unroll
        for (int it = 0; it < ITEMS; it++)
            if (dig[it] < RADIX) s_exch[pos[it]] = __ldg(src + tile_base + warp * 32 * ITEMS + it * 32 + lane);
        __syncthreads();
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            uint32_t j = it * THREADS + tid;
            if (j < tile_valid && dst[it] < a.n) out[dst[it]] = s_exch[j];
        }
        __syncthreads();
    }
}

// Histogram of every pass's digit for keys already in memory (used when the
// producer could not fuse it, e.g. sorts of derived pairs).
// Variant with the key width fixed at compile time: every key word and the value
// of the tile are loaded into registers before ranking (all of the tile's bytes
// in flight at once), and all arrays are exchanged through one shared-memory
// buffer of (KW+1) x TILE words with a single barrier.
template <int KW, int ITEMS>
__global__ __launch_bounds__(SORT_THREADS) void k_onesweep_w(SortPassArgs a) {
    constexpr int THREADS = SORT_THREADS;
    constexpr int WARPS = THREADS / 32;
    constexpr int TILE = THREADS * ITEMS;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_hist[WARPS][RADIX];
    __shared__ uint32_t s_tile_excl[RADIX];
    __shared__ uint32_t s_gbase[RADIX];
    __shared__ uint32_t s_scan[THREADS / 32 + 1];
    extern __shared__ uint32_t s_exch[];  // [(KW + 1) * TILE]

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    for (int i = tid; i < WARPS * RADIX; i += THREADS) (&s_warp_hist[0][0])[i] = 0;
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t tile_base = tile * TILE;
    const uint64_t remain = a.n - tile_base;
    const uint32_t tile_valid = remain < (uint64_t)TILE ? (uint32_t)remain : (uint32_t)TILE;
    const int wd = a.shift >> 5, sh = a.shift & 31;

    // 1. all loads up front (warp-striped)
    uint32_t v[KW + 1][ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        const bool ok = e < tile_valid;
#pragma unroll
        for (int w = 0; w < KW; w++) v[w][it] = ok ? __ldg(a.keys_in[w] + tile_base + e) : 0u;
        v[KW][it] = ok ? __ldg(a.vals_in + tile_base + e) : 0u;
    }
    uint32_t pos[ITEMS];
    uint32_t dig[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        uint32_t kword = v[0][it];
#pragma unroll
        for (int w = 1; w < KW; w++)
            if (w == wd) kword = v[w][it];
        dig[it] = e < tile_valid ? (kword >> sh) & (RADIX - 1) : RADIX;
    }
    // 2. rank inside the warp
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t d = dig[it];
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & lanemask_lt());
        uint32_t cnt = 0;
        if (d < RADIX) cnt = s_warp_hist[warp][d];
        pos[it] = cnt + before;
        __syncwarp();
        if (d < RADIX && before == 0) s_warp_hist[warp][d] = cnt + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // 3. per digit: warp prefix, tile count, tile-local offsets, decoupled look-back
    {
        const int d = tid;
        uint32_t count = 0;
#pragma unroll
        for (int w = 0; w < WARPS; w++) {
            uint32_t t = s_warp_hist[w][d];
            s_warp_hist[w][d] = count;
            count += t;
        }
        uint32_t total;
        const uint32_t ex = block_excl_scan<THREADS>(count, s_scan, total);
        s_tile_excl[d] = ex;
        uint64_t* my = a.lookback + tile * RADIX + d;
        uint32_t excl = 0;
        if (tile == 0) {
            st_relaxed(my, lb_pack(a.epoch, 2u, count));
        } else {
            st_relaxed(my, lb_pack(a.epoch, 1u, count));
            int64_t t = (int64_t)tile - 1;
            uint32_t spins = 0;
            while (t >= 0) {
                const uint64_t lv = ld_relaxed(a.lookback + (uint64_t)t * RADIX + d);
                const uint32_t ep = (uint32_t)(lv >> 34), fl = (uint32_t)(lv >> 32) & 3u;
                if (ep != a.epoch || fl == 0) {
                    if (++spins > a.spin_limit) {
                        atomicOr(a.err, DEV_ERR_TIMEOUT);
                        break;
                    }
                    if (spins > 64) __nanosleep(64);
                    continue;
                }
                excl += (uint32_t)lv;
                if (fl == 2u) break;
                t--;
            }
            st_relaxed(my, lb_pack(a.epoch, 2u, excl + count));
        }
        s_gbase[d] = a.digit_base[d] + excl - ex;
    }
    __syncthreads();

    // 4. one exchange of all arrays into digit order, then coalesced-by-run stores
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t d = dig[it];
        if (d < RADIX) {
            const uint32_t p = pos[it] + s_tile_excl[d] + s_warp_hist[warp][d];
#pragma unroll
            for (int w = 0; w <= KW; w++) s_exch[w * TILE + p] = v[w][it];
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t j = it * THREADS + tid;
        if (j < tile_valid) {
            const uint32_t kword = s_exch[wd * TILE + j];
            const uint32_t dst = s_gbase[(kword >> sh) & (RADIX - 1)] + j;
            if (dst < a.n) {
#pragma unroll
                for (int w = 0; w < KW; w++) a.keys_out[w][dst] = s_exch[w * TILE + j];
                a.vals_out[dst] = s_exch[KW * TILE + j];
            } else {
                atomicOr(a.err, DEV_ERR_RANGE);
            }
        }
    }
}

template <int KW, int ITEMS>
constexpr size_t onesweep_w_smem() {
    return sizeof(uint32_t) * (KW + 1) * SORT_THREADS * ITEMS;
}

// Lanes of the warp holding the same 8-bit digit (plus a validity bit), from
// nine ballots; stable ranking needs only the lanes below this one.
__device__ __forceinline__ uint32_t warp_digit_peers(uint32_t d) {
    uint32_t peers = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < RADIX_BITS + 1; b++) {
        const uint32_t bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bal : ~bal;
    }
    return peers;
}

// Onesweep pass with early counts: the tile's digit counts are gathered with
// shared-memory atomics and published to the look-back array before the stable
// ranking, so successors rarely wait; the look-back reads LB_WINDOW
// predecessor tiles per round trip.
template <int ITEMS, bool PRELOAD>
__global__ __launch_bounds__(SORT_THREADS) void k_onesweep_ec(SortPassArgs a) {
    constexpr int THREADS = SORT_THREADS;
    constexpr int WARPS = THREADS / 32;
    constexpr int TILE = THREADS * ITEMS;
    constexpr int LB_WINDOW = 4;
    constexpr int PRE = PRELOAD ? 3 : 1;  // arrays preloaded: up to 2 extra key words + value
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_hist[WARPS][RADIX];
    __shared__ uint32_t s_tile_excl[RADIX];
    __shared__ uint32_t s_gbase[RADIX];
    __shared__ uint32_t s_scan[THREADS / 32 + 1];
    __shared__ uint32_t s_exch[TILE];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    for (int i = tid; i < WARPS * RADIX; i += THREADS) (&s_warp_hist[0][0])[i] = 0;
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t tile_base = tile * TILE;
    const uint64_t remain = a.n - tile_base;
    const uint32_t tile_valid = remain < (uint64_t)TILE ? (uint32_t)remain : (uint32_t)TILE;
    const int wd = a.shift >> 5, sh = a.shift & 31;
    const int kw = (int)a.kw;

    uint32_t kword[ITEMS];
    uint32_t dig[ITEMS];
    const uint32_t* kin = a.keys_in[wd];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        kword[it] = e < tile_valid ? __ldg(kin + tile_base + e) : 0u;
    }
    // other arrays (key words != wd, then the value), preloaded when asked
    uint32_t pre[PRE][ITEMS];
    if (PRELOAD) {
        int slot = 0;
        for (int w = 0; w <= kw && slot < PRE; w++) {
            if (w == wd) continue;
            const uint32_t* src = w < kw ? a.keys_in[w] : a.vals_in;
#pragma unroll
            for (int it = 0; it < ITEMS; it++) {
                const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
                pre[slot][it] = e < tile_valid ? __ldg(src + tile_base + e) : 0u;
            }
            slot++;
        }
    }
    // 1. early counts per warp
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        dig[it] = e < tile_valid ? (kword[it] >> sh) & (RADIX - 1) : RADIX;
        if (dig[it] < RADIX) atomicAdd(&s_warp_hist[warp][dig[it]], 1u);
    }
    __syncthreads();
    uint32_t count = 0;
    {
        const int d = tid;
#pragma unroll
        for (int w = 0; w < WARPS; w++) {
            const uint32_t t = s_warp_hist[w][d];
            s_warp_hist[w][d] = count;  // exclusive prefix over warps: the warp's running base
            count += t;
        }
        uint64_t* my = a.lookback + tile * RADIX + d;
        st_relaxed(my, lb_pack(a.epoch, tile == 0 ? 2u : 1u, count));
        uint32_t total;
        s_tile_excl[d] = block_excl_scan<THREADS>(count, s_scan, total);
    }
    // 2. stable rank inside the warp (ballot peers), positions in the sorted tile
    uint32_t pos[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t d = dig[it];
        const uint32_t peers = warp_digit_peers(d);
        const uint32_t before = __popc(peers & lanemask_lt());
        uint32_t base = 0;
        if (d < RADIX) base = s_warp_hist[warp][d];
        pos[it] = base + before;
        __syncwarp();
        if (d < RADIX && before == 0) s_warp_hist[warp][d] = base + __popc(peers);
        __syncwarp();
    }
    // 3. look-back for digit tid
    {
        const int d = tid;
        uint32_t excl = 0;
        if (tile > 0) {
            int64_t t = (int64_t)tile - 1;
            uint32_t spins = 0;
            while (t >= 0) {
                uint64_t lv[LB_WINDOW];
#pragma unroll
                for (int k = 0; k < LB_WINDOW; k++)
                    lv[k] = (t - k >= 0) ? ld_relaxed(a.lookback + (uint64_t)(t - k) * RADIX + d) : lb_pack(a.epoch, 2u, 0u);
                // consume the window from the nearest tile backwards while statuses are valid
                int k = 0;
                bool stop = false;
                for (; k < LB_WINDOW; k++) {
                    const uint32_t ep = (uint32_t)(lv[k] >> 34), fl = (uint32_t)(lv[k] >> 32) & 3u;
                    if (ep != a.epoch || fl == 0) break;
                    excl += (uint32_t)lv[k];
                    if (fl == 2u) {
                        stop = true;
                        break;
                    }
                }
                if (stop) break;
                t -= k;
                if (k == 0) {
                    if (++spins > a.spin_limit) {
                        atomicOr(a.err, DEV_ERR_TIMEOUT);
                        break;
                    }
                    if (spins > 32) __nanosleep(32);
                }
            }
            st_relaxed(a.lookback + tile * RADIX + d, lb_pack(a.epoch, 2u, excl + count));
        }
        s_gbase[d] = a.digit_base[d] + excl - s_tile_excl[d];
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITEMS; it++)
        if (dig[it] < RADIX) pos[it] += s_tile_excl[dig[it]];

    // 4. exchange the digit word, compute destinations, then the other arrays
    uint32_t dst[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++)
        if (dig[it] < RADIX) s_exch[pos[it]] = kword[it];
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t j = it * THREADS + tid;
        if (j < tile_valid) {
            const uint32_t w = s_exch[j];
            dst[it] = s_gbase[(w >> sh) & (RADIX - 1)] + j;
            if (dst[it] < a.n) a.keys_out[wd][dst[it]] = w;
            else atomicOr(a.err, DEV_ERR_RANGE);
        }
    }
    int slot = 0;
    for (int w = 0; w <= kw; w++) {
        if (w == wd) continue;
        const uint32_t* src = w < kw ? a.keys_in[w] : a.vals_in;
        uint32_t* out = w < kw ? a.keys_out[w] : a.vals_out;
        __syncthreads();
        if (PRELOAD && slot < PRE) {
#pragma unroll
            for (int it = 0; it < ITEMS; it++)
                if (dig[it] < RADIX) s_exch[pos[it]] = pre[slot][it];
        } else {
#pragma unroll
            for (int it = 0; it < ITEMS; it++)
                if (dig[it] < RADIX) s_exch[pos[it]] = __ldg(src + tile_base + warp * 32 * ITEMS + it * 32 + lane);
        }
        slot++;
        __syncthreads();
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            const uint32_t j = it * THREADS + tid;
            if (j < tile_valid && dst[it] < a.n) out[dst[it]] = s_exch[j];
        }
    }
}

// Onesweep pass with early counts and a compile-time key width: all KW key words
// and the value are loaded into registers up front (static indexing, no local
// memory), counts are published before ranking, and each array is exchanged
// through shared memory in turn.  When vals_in is null the value of element i
// is i itself (first pass after key materialisation: the identity permutation).
template <int KW, int ITEMS>
__global__ __launch_bounds__(SORT_THREADS) void k_onesweep_k(SortPassArgs a) {
    constexpr int THREADS = SORT_THREADS;
    constexpr int WARPS = THREADS / 32;
    constexpr int TILE = THREADS * ITEMS;
    constexpr int LB_WINDOW = 4;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_hist[WARPS][RADIX];
    __shared__ uint32_t s_tile_excl[RADIX];
    __shared__ uint32_t s_gbase[RADIX];
    __shared__ uint32_t s_scan[THREADS / 32 + 1];
    __shared__ uint32_t s_exch[TILE];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    for (int i = tid; i < WARPS * RADIX; i += THREADS) (&s_warp_hist[0][0])[i] = 0;
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t tile_base = tile * TILE;
    const uint64_t remain = a.n - tile_base;
    const uint32_t tile_valid = remain < (uint64_t)TILE ? (uint32_t)remain : (uint32_t)TILE;
    const int wd = a.shift >> 5, sh = a.shift & 31;

    uint32_t v[KW + 1][ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        const bool ok = e < tile_valid;
#pragma unroll
        for (int w = 0; w < KW; w++) v[w][it] = ok ? __ldg(a.keys_in[w] + tile_base + e) : 0u;
        v[KW][it] = a.vals_in ? (ok ? __ldg(a.vals_in + tile_base + e) : 0u) : (uint32_t)(tile_base + e);
    }
    uint32_t dig[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        uint32_t kword = v[0][it];
#pragma unroll
        for (int w = 1; w < KW; w++)
            if (w == wd) kword = v[w][it];
        dig[it] = e < tile_valid ? (kword >> sh) & (RADIX - 1) : RADIX;
        if (dig[it] < RADIX) atomicAdd(&s_warp_hist[warp][dig[it]], 1u);
    }
    __syncthreads();
    uint32_t count = 0;
    {
        const int d = tid;
#pragma unroll
        for (int w = 0; w < WARPS; w++) {
            const uint32_t t = s_warp_hist[w][d];
            s_warp_hist[w][d] = count;
            count += t;
        }
        st_relaxed(a.lookback + tile * RADIX + d, lb_pack(a.epoch, tile == 0 ? 2u : 1u, count));
        uint32_t total;
        s_tile_excl[d] = block_excl_scan<THREADS>(count, s_scan, total);
    }
    uint32_t pos[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t d = dig[it];
        const uint32_t peers = warp_digit_peers(d);
        const uint32_t before = __popc(peers & lanemask_lt());
        uint32_t base = 0;
        if (d < RADIX) base = s_warp_hist[warp][d];
        pos[it] = base + before;
        __syncwarp();
        if (d < RADIX && before == 0) s_warp_hist[warp][d] = base + __popc(peers);
        __syncwarp();
    }
    {
        const int d = tid;
        uint32_t excl = 0;
        if (tile > 0) {
            int64_t t = (int64_t)tile - 1;
            uint32_t spins = 0;
            while (t >= 0) {
                uint64_t lv[LB_WINDOW];
#pragma unroll
                for (int k = 0; k < LB_WINDOW; k++)
                    lv[k] = (t - k >= 0) ? ld_relaxed(a.lookback + (uint64_t)(t - k) * RADIX + d)
                                         : lb_pack(a.epoch, 2u, 0u);
                int k = 0;
                bool stop = false;
                for (; k < LB_WINDOW; k++) {
                    const uint32_t ep = (uint32_t)(lv[k] >> 34), fl = (uint32_t)(lv[k] >> 32) & 3u;
                    if (ep != a.epoch || fl == 0) break;
                    excl += (uint32_t)lv[k];
                    if (fl == 2u) {
                        stop = true;
                        break;
                    }
                }
                if (stop) break;
                t -= k;
                if (k == 0) {
                    if (++spins > a.spin_limit) {
                        atomicOr(a.err, DEV_ERR_TIMEOUT);
                        break;
                    }
                    if (spins > 32) __nanosleep(32);
                }
            }
            st_relaxed(a.lookback + tile * RADIX + d, lb_pack(a.epoch, 2u, excl + count));
        }
        s_gbase[d] = a.digit_base[d] + excl - s_tile_excl[d];
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITEMS; it++)
        if (dig[it] < RADIX) pos[it] += s_tile_excl[dig[it]];

    // digit word first: destinations of the sorted slots
    uint32_t dst[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        uint32_t kword = v[0][it];
#pragma unroll
        for (int w = 1; w < KW; w++)
            if (w == wd) kword = v[w][it];
        if (dig[it] < RADIX) s_exch[pos[it]] = kword;
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t j = it * THREADS + tid;
        dst[it] = 0xffffffffu;
        if (j < tile_valid) {
            const uint32_t w = s_exch[j];
            dst[it] = s_gbase[(w >> sh) & (RADIX - 1)] + j;
            if (dst[it] < a.n) a.keys_out[wd][dst[it]] = w;
            else atomicOr(a.err, DEV_ERR_RANGE);
        }
    }
#pragma unroll
    for (int w = 0; w <= KW; w++) {
        if (w == wd) continue;
        uint32_t* out = w < KW ? a.keys_out[w] : a.vals_out;
        __syncthreads();
#pragma unroll
        for (int it = 0; it < ITEMS; it++)
            if (dig[it] < RADIX) s_exch[pos[it]] = v[w][it];
        __syncthreads();
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            const uint32_t j = it * THREADS + tid;
            if (j < tile_valid && dst[it] < a.n) out[dst[it]] = s_exch[j];
        }
    }
}

// Histogram of every 8-bit digit of keys already in memory (4*kw passes), for
// sorts whose producer is a scan operator rather than a key builder.
__global__ __launch_bounds__(256) void k_digit_hist(SortPassArgs a, uint32_t* hist /* [4*kw][RADIX] */) {
    extern __shared__ uint32_t sh[];
    const uint32_t passes = 4 * a.kw;
    for (uint32_t i = threadIdx.x; i < passes * RADIX; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (uint64_t)gridDim.x * blockDim.x) {
        for (uint32_t w = 0; w < a.kw; w++) {
            const uint32_t k = a.keys_in[w][i];
#pragma unroll
            for (int b = 0; b < 4; b++) atomicAdd(&sh[(4 * w + b) * RADIX + ((k >> (8 * b)) & (RADIX - 1))], 1u);
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < passes * RADIX; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Exclusive scan of each pass's 256-bin histogram (one CTA per pass).
__global__ __launch_bounds__(RADIX) void k_digit_offsets(const uint32_t* hist, uint32_t* base) {
    __shared__ uint32_t sm[RADIX / 32 + 1];
    uint32_t v = hist[blockIdx.x * RADIX + threadIdx.x];
    uint32_t total;
    uint32_t ex = block_excl_scan<RADIX>(v, sm, total);
    base[blockIdx.x * RADIX + threadIdx.x] = ex;
}

}  // namespace dcx
