// Key materialisation for the suffix sorts.
//
// The reference packs the first X*ratio characters of a suffix MSB-first into
// 64-bit words, 3/5/8 bits per char (lightweight_dcx/src/strings/char_container.hpp:50-104,
// 483-545; cli.cpp:488-533) and compares the words lexicographically.  The GPU
// build needs the same order but as a radix-sortable integer with as few bits as
// possible, so a window c_0..c_{P-1} of chars in 0..sigma (0 = padding past the
// end of the text) is encoded as the mixed-radix integer
//     key = sum_j c_j * (sigma+1)^(P-1-j)
// which orders exactly like the packed words (same prefix -> same key; first
// difference decides).  DNA (sigma = 4) needs log2(5) = 2.32 bits per char
// instead of 3.  The integer is built in chunks: k chars at a time form a
// 32-bit digit of base (sigma+1)^k, then a multi-word multiply-add folds it in.
//
// Each producer also accumulates the 8-bit digit histograms of every radix pass
// of its keys, so the sort needs no extra read of the keys.
#pragma once

#include "common.cuh"
#include "radix.cuh"

namespace dcx {

constexpr int MAX_CHUNKS = 48;

struct KeyPlan {
    uint32_t base;                   // sigma + 1 (chars are 0..sigma)
    uint32_t chars;                  // chars encoded (window length)
    uint32_t kw;                     // key words holding the chars
    uint32_t nchunks;
    uint32_t chunk_len[MAX_CHUNKS];  // chars per chunk
    uint32_t chunk_mul[MAX_CHUNKS];  // (sigma+1)^chunk_len
};

template <typename CharT>
__device__ __forceinline__ uint32_t ldc(const CharT* p) {
    return (uint32_t)__ldg(p);
}

// Encodes chars text[pos+off .. pos+off+plan.chars) (0 at or past n) into acc[0..KW).
template <int KW, typename CharT>
__device__ __forceinline__ void encode_window(const CharT* text, uint64_t n, uint64_t start,
                                              const KeyPlan& plan, uint32_t* acc) {
#pragma unroll
    for (int w = 0; w < KW; w++) acc[w] = 0;
    uint64_t p = start;
    for (uint32_t c = 0; c < plan.nchunks; c++) {
        const uint32_t len = plan.chunk_len[c];
        const uint32_t base = plan.base;
        uint32_t digit = 0;  // the chunk's chars in base sigma+1 (< chunk_mul[c] <= 2^32-1)
        for (uint32_t j = 0; j < len; j++, p++) {
            uint32_t ch = p < n ? ldc(text + p) : 0u;
            digit = digit * base + ch;
        }
        const uint32_t mul = plan.chunk_mul[c];
        uint64_t carry = digit;
#pragma unroll
        for (int w = 0; w < KW; w++) {
            uint64_t t = (uint64_t)acc[w] * mul + carry;
            acc[w] = (uint32_t)t;
            carry = t >> 32;
        }
    }
}

struct KeyOut {
    uint32_t* w[MAX_KEY_WORDS];
};

template <int KW>
__device__ __forceinline__ void hist_add(uint32_t* sh, const uint32_t* key, uint32_t passes) {
    for (uint32_t p = 0; p < passes; p++) {
        uint32_t s = p * RADIX_BITS;
        uint32_t d = (key[s >> 5] >> (s & 31)) & (RADIX - 1);
        atomicAdd(&sh[p * RADIX + d], 1u);
    }
}

// Level keys: for every position i in [0, N) (N = n + 1: position n is the empty
// suffix / dummy sample, key 0), key = window [i, i+chars), value = i.
template <int KW, typename CharT>
__global__ __launch_bounds__(256) void k_keys_prefix(const CharT* __restrict__ text, uint64_t n, uint64_t N,
                                                     KeyPlan plan, KeyOut ko, uint32_t* __restrict__ vals_out,
                                                     uint32_t* hist) {
    extern __shared__ uint32_t sh[];
    const uint32_t total_passes = 4 * KW;
    for (uint32_t i = threadIdx.x; i < total_passes * RADIX; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t key[KW];
        encode_window<KW>(text, n, i, plan, key);
#pragma unroll
        for (int w = 0; w < KW; w++) ko.w[w][i] = key[w];
        vals_out[i] = (uint32_t)i;
        hist_add<KW>(sh, key, total_passes);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < total_passes * RADIX; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Refinement keys for the elements of tie groups: element j sits at sorted slot
// slot[j]; its text position is sa[slot[j]], its group number grp[j].  The key is
// (group number in the top word, window [pos+off, pos+off+chars) below it);
// value = text position.
template <int KW, typename CharT>
__global__ __launch_bounds__(256) void k_keys_refine(const CharT* __restrict__ text, uint64_t n, uint64_t count,
                                                     const uint32_t* __restrict__ slot,
                                                     const uint32_t* __restrict__ grp,
                                                     const uint32_t* __restrict__ sa, uint32_t off,
                                                     KeyPlan plan, KeyOut ko, uint32_t* __restrict__ vals_out,
                                                     uint32_t* hist) {
    extern __shared__ uint32_t sh[];
    const uint32_t total_passes = 4 * (KW + 1);
    for (uint32_t i = threadIdx.x; i < total_passes * RADIX; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < count;
         j += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t pos = sa[slot[j]];
        uint32_t key[KW + 1];
        encode_window<KW>(text, n, (uint64_t)pos + off, plan, key);
        key[KW] = grp[j];
#pragma unroll
        for (int w = 0; w <= KW; w++) ko.w[w][j] = key[w];
        vals_out[j] = pos;
        hist_add<KW + 1>(sh, key, total_passes);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < total_passes * RADIX; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

}  // namespace dcx
