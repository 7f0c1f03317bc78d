// Base case: suffix array of a short string inside one CTA.
//
// The reference solves a level sequentially once it is small
// (compute_sa_on_root, lightweight_dcx/src/pdcx/pdcx.hpp:623-633, with
// slow_suffixarray, util/string_util.hpp:100-106).  On the GPU a string of up to
// SMALL_MAX chars is solved by prefix doubling in shared memory: ranks start as
// the chars, each round sorts (rank[i], rank[i+h]) pairs with a bitonic network
// and renames, until all ranks are distinct.  The suffix array is unique, so
// the result equals the reference's.  One CTA per string, so a batch of short
// texts is one launch.
#pragma once

#include "common.cuh"

namespace dcx {

constexpr int SMALL_MAX = 2048;
constexpr int SMALL_THREADS = 1024;

// String s of the launch is text[start[s] .. start[s+1]-1) (each string is
// followed by its 0); its SA (string-local indices) goes to entries [obase[s], obase[s] + n) of
// out, `width` bits per entry.
// Chars must be >= 1.
template <typename CharT>
__global__ __launch_bounds__(SMALL_THREADS) void k_small_sa(const CharT* __restrict__ text,
                                                            const uint64_t* __restrict__ start,
                                                            const uint64_t* __restrict__ obase, void* __restrict__ out, int width) {
    __shared__ uint64_t key[SMALL_MAX];
    __shared__ uint16_t idx[SMALL_MAX];
    __shared__ uint32_t rank[SMALL_MAX];
    __shared__ uint32_t scan_sm[SMALL_THREADS / 32 + 1];
    __shared__ uint32_t s_done;

    const uint32_t s = blockIdx.x;
    const uint64_t b = start[s];
    const uint32_t n = (uint32_t)(start[s + 1] - b - 1);
    if (n == 0) return;
    const CharT* t = text + b;
    const uint64_t ob = obase[s];
    for (uint32_t i = threadIdx.x; i < n; i += SMALL_THREADS) rank[i] = (uint32_t)t[i];
    __syncthreads();
    if (n == 1) {
        if (threadIdx.x == 0) store_sa_entry(out, ob, 0u, width);
        return;
    }
    uint32_t C = 2;
    while (C < n) C <<= 1;
    for (uint32_t h = 1;; h <<= 1) {
        for (uint32_t i = threadIdx.x; i < C; i += SMALL_THREADS) {
            if (i < n) {
                uint32_t r2 = i + h < n ? rank[i + h] : 0u;
                key[i] = ((uint64_t)rank[i] << 32) | r2;
            } else {
                key[i] = ~0ull;
            }
            idx[i] = (uint16_t)i;
        }
        __syncthreads();
        for (uint32_t k = 2; k <= C; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t p = threadIdx.x; p < C / 2; p += SMALL_THREADS) {
                    const uint32_t i = 2 * j * (p / j) + (p % j);
                    const uint32_t q = i + j;
                    const bool up = (i & k) == 0;
                    const uint64_t a = key[i], c = key[q];
                    // ties only between padding entries, which are equal anyway
                    const bool swap = up ? (c < a || (c == a && idx[q] < idx[i]))
                                         : (a < c || (a == c && idx[i] < idx[q]));
                    if (swap) {
                        key[i] = c;
                        key[q] = a;
                        uint16_t x = idx[i];
                        idx[i] = idx[q];
                        idx[q] = x;
                    }
                }
                __syncthreads();
            }
        }
        // rename: rank = 1 + number of distinct pairs before (blocked layout, 2 per thread)
        uint32_t heads[2];
        uint32_t local = 0;
        for (int e = 0; e < 2; e++) {
            uint32_t k = threadIdx.x * 2 + e;
            heads[e] = (k < n) ? (k == 0 || key[k] != key[k - 1]) : 0u;
            local += heads[e];
        }
        uint32_t total;
        uint32_t ex = block_excl_scan<SMALL_THREADS>(local, scan_sm, total);
        for (int e = 0; e < 2; e++) {
            uint32_t k = threadIdx.x * 2 + e;
            ex += heads[e];
            if (k < n) rank[idx[k]] = ex;
        }
        if (threadIdx.x == 0) s_done = (total == n) || (h >= n);
        __syncthreads();
        if (s_done) break;
    }
    for (uint32_t k = threadIdx.x; k < n; k += SMALL_THREADS) store_sa_entry(out, ob + k, idx[k], width);
}

}  // namespace dcx
