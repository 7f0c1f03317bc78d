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
