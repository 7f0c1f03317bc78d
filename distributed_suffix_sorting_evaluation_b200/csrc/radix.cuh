// Onesweep LSD radix sort over multi-word keys (KW little-endian uint32 words,
// structure-of-arrays) carrying one uint32 value.  Replaces the reference's
// distributed comparison sorts (lightweight_dcx/src/sorters/sorting_wrapper.hpp:57-94,
// sample_sort.hpp:36-171) for every sort of the DCX pipeline.
//
// One kernel per 8-bit digit (k_onesweep<KW, ITEMS>: 4096-element tiles with three CTAs
// per SM by default, 3072-element tiles with four as the alternative a context
// option or the batch autotuner selects):
//   * tiles are claimed in order through an atomic counter;
//   * the words the pass does not rank on (other key words, the value) are
//     prefetched into shared memory with cp.async as soon as the tile is
//     known, so their loads overlap the ranking without holding registers;
//   * the tile's digit counts are gathered with shared-memory atomics and
//     published to a look-back array before the stable ranking (ballot peers
//     inside each warp), and each digit's global offset is found by decoupled
//     look-back; every wait is bounded and, when exhausted, sets an error bit
//     and lets the CTA finish;
//   * every array is exchanged through shared memory into digit order so that
//     global writes of one digit run are contiguous;
//   * full tiles (all but the last) run a copy of the tile code without
//     per-item bounds tests.
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
    uint32_t hold_tile;           // tile that never publishes its status (0xffffffff: none)
    uint32_t* gave_up;            // count of CTAs whose look-back wait ran out
};

// Lanes of the warp holding the same 8-bit digit, from eight ballots, or nine
// when some lanes hold no element (digit RADIX); stable ranking needs only the
// lanes below this one.
template <bool PARTIAL>
__device__ __forceinline__ uint32_t warp_digit_peers(uint32_t d) {
    uint32_t peers = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < RADIX_BITS + (PARTIAL ? 1 : 0); b++) {
        const uint32_t bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bal : ~bal;
    }
    return peers;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

constexpr int ONESWEEP_ITEMS = 16;      // default: 4096-element tiles
constexpr int ONESWEEP_ITEMS_ALT = 12;  // alternative: 3072-element tiles
constexpr int ONESWEEP_TILE = SORT_THREADS * ONESWEEP_ITEMS;

// Register budget of a tile size: three 256-thread CTAs per SM for 16 items per
// thread, four for 12.
__host__ __device__ constexpr int onesweep_min_ctas(int items) { return items > 12 ? 3 : 4; }

// Dynamic shared memory of k_onesweep<KW, ITEMS>: the exchange buffer plus one
// staging buffer per carried array (KW - 1 other key words and the value).
__host__ __device__ constexpr size_t onesweep_smem(uint32_t kw, uint32_t items = ONESWEEP_ITEMS) {
    return sizeof(uint32_t) * (size_t)SORT_THREADS * items * (1 + kw);
}

// Shared state of one CTA of k_onesweep (static shared memory).
struct OnesweepShared {
    uint32_t warp_hist[SORT_THREADS / 32][RADIX];  // per-warp digit counts, then running bases
    uint32_t tile_excl[RADIX];                     // exclusive digit offsets inside the tile
    uint32_t gbase[RADIX];                         // global destination of the tile's digit runs
    uint32_t scan[SORT_THREADS / 32 + 1];
    uint32_t tile;
    uint32_t gave_up;
};

// One tile of one LSD pass over KW key words and a value.  FULL: the tile holds
// TILE valid elements (every tile but the last), which drops every per-item
// bounds test; the last tile marks missing elements with digit RADIX.
template <int KW, int ITEMS, bool FULL>
__device__ __forceinline__ void onesweep_tile(const SortPassArgs& a, OnesweepShared& sm, uint32_t* s_exch,
                                              uint32_t* s_stage, uint64_t tile, uint32_t tile_valid) {
    constexpr int THREADS = SORT_THREADS;
    constexpr int WARPS = THREADS / 32;
    constexpr int TILE = THREADS * ITEMS;
    constexpr int LB_WINDOW = 4;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t tile_base = tile * TILE;
    const int wd = a.shift >> 5, sh = a.shift & 31;

    // 0. prefetch the carried arrays (slot s: key word s < wd ? s : s + 1, the value last)
#pragma unroll
    for (int s = 0; s < KW; s++) {
        const int w = s < wd ? s : s + 1;
        const uint32_t* src = (w < KW ? a.keys_in[w] : a.vals_in) + tile_base;
        uint32_t* dst = s_stage + s * TILE;
        if (FULL) {
#pragma unroll
            for (int i = 0; i < TILE / 4 / THREADS; i++) {
                const int c = (i * THREADS + tid) * 4;
                cp_async16(dst + c, src + c);
            }
        } else {
            for (uint32_t e = tid; e < tile_valid; e += THREADS) cp_async4(dst + e, src + e);
        }
    }
    cp_async_commit();

    // 1. digit word (warp-blocked: item `it` of lane l in warp w is tile element
    //    w*32*ITEMS + it*32 + l) and early counts per warp
    uint32_t kword[ITEMS], dig[ITEMS], pos[ITEMS];
    const uint32_t* kin = a.keys_in[wd] + tile_base;
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        kword[it] = (FULL || e < tile_valid) ? __ldg(kin + e) : 0u;
    }
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t e = warp * 32 * ITEMS + it * 32 + lane;
        dig[it] = (FULL || e < tile_valid) ? (kword[it] >> sh) & (RADIX - 1) : RADIX;
        if (FULL || dig[it] < RADIX) atomicAdd(&sm.warp_hist[warp][dig[it]], 1u);
    }
    __syncthreads();
    uint32_t count = 0;
    {
        const int d = tid;
#pragma unroll
        for (int w = 0; w < WARPS; w++) {
            const uint32_t t = sm.warp_hist[w][d];
            sm.warp_hist[w][d] = count;  // exclusive prefix over warps: the warp's running base
            count += t;
        }
        if (tile != a.hold_tile)
            st_relaxed(a.lookback + tile * RADIX + d, lb_pack(a.epoch, tile == 0 ? 2u : 1u, count));
        uint32_t total;
        sm.tile_excl[d] = block_excl_scan<THREADS>(count, sm.scan, total);
    }
    // 2. stable rank inside the warp, positions in the sorted tile
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t d = dig[it];
        const uint32_t peers = warp_digit_peers<!FULL>(d);
        const uint32_t before = __popc(peers & lanemask_lt());
        uint32_t base = 0;
        if (FULL || d < RADIX) base = sm.warp_hist[warp][d];
        pos[it] = base + before;
        __syncwarp();
        if ((FULL || d < RADIX) && before == 0) sm.warp_hist[warp][d] = base + __popc(peers);
        __syncwarp();
    }
    // 3. decoupled look-back for digit tid (bounded)
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
                        sm.gave_up = 1;
                        break;
                    }
                    if (spins > 32) __nanosleep(32);
                }
            }
            if (tile != a.hold_tile) st_relaxed(a.lookback + tile * RADIX + d, lb_pack(a.epoch, 2u, excl + count));
        }
        sm.gbase[d] = a.digit_base[d] + excl - sm.tile_excl[d];
    }
    __syncthreads();
    if (tid == 0 && sm.gave_up && a.gave_up) atomicAdd(a.gave_up, 1u);
#pragma unroll
    for (int it = 0; it < ITEMS; it++)
        if (FULL || dig[it] < RADIX) pos[it] += sm.tile_excl[dig[it]];

    // 4. digit word: exchange, destinations, store
    uint32_t dst[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++)
        if (FULL || dig[it] < RADIX) s_exch[pos[it]] = kword[it];
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        const uint32_t j = it * THREADS + tid;
        dst[it] = 0xffffffffu;
        if (FULL || j < tile_valid) {
            const uint32_t w = s_exch[j];
            const uint32_t d = sm.gbase[(w >> sh) & (RADIX - 1)] + j;
            if (d < a.n) {
                dst[it] = d;
                a.keys_out[wd][d] = w;
            } else {
                atomicOr(a.err, DEV_ERR_RANGE);
            }
        }
    }
    // 5. carried arrays from the staging buffers, through the same exchange
    cp_async_wait_all();
#pragma unroll
    for (int s = 0; s < KW; s++) {
        const int w = s < wd ? s : s + 1;
        uint32_t* out = w < KW ? a.keys_out[w] : a.vals_out;
        const uint32_t* stg = s_stage + s * TILE;
        __syncthreads();  // s_exch free, every thread's staged copies complete
#pragma unroll
        for (int it = 0; it < ITEMS; it++)
            if (FULL || dig[it] < RADIX) s_exch[pos[it]] = stg[warp * 32 * ITEMS + it * 32 + lane];
        __syncthreads();
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            const uint32_t j = it * THREADS + tid;
            if ((FULL || j < tile_valid) && dst[it] != 0xffffffffu) out[dst[it]] = s_exch[j];
        }
    }
}

// One LSD pass over KW key words (1..3) carrying one value.  Every array base
// must be 16-byte aligned (full tiles are staged with 16-byte copies; the last,
// partial tile uses 4-byte copies, which never read past the array end).
template <int KW, int ITEMS>
__global__ __launch_bounds__(SORT_THREADS, onesweep_min_ctas(ITEMS)) void k_onesweep(SortPassArgs a) {
    constexpr int TILE = SORT_THREADS * ITEMS;
    __shared__ OnesweepShared sm;
    extern __shared__ __align__(16) uint32_t s_dyn[];
    const int tid = threadIdx.x;
    if (tid == 0) {
        sm.tile = atomicAdd(a.tile_counter, 1u);
        sm.gave_up = 0;
    }
    for (int i = tid; i < (SORT_THREADS / 32) * RADIX; i += SORT_THREADS) (&sm.warp_hist[0][0])[i] = 0;
    __syncthreads();
    const uint64_t tile = sm.tile;
    const uint64_t remain = a.n - tile * TILE;
    const uint32_t tile_valid = remain < (uint64_t)TILE ? (uint32_t)remain : (uint32_t)TILE;
    if (tile_valid == (uint32_t)TILE)
        onesweep_tile<KW, ITEMS, true>(a, sm, s_dyn, s_dyn + TILE, tile, tile_valid);
    else
        onesweep_tile<KW, ITEMS, false>(a, sm, s_dyn, s_dyn + TILE, tile, tile_valid);
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

}  // namespace dcx
