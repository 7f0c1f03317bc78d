// Generalized suffix array of a string set, in the convention of libsais64_gsa
// (libsais/include/libsais64.h:63-72): T holds the strings, each followed by a
// 0 separator (T[n-1] = 0, no empty string), and all n suffixes are ordered as
// if every separator were its own symbol below every character, the
// separators in string order.
//
// Built from the plain SA of T (0 being the smallest byte, the plain order
// compares across separators).  Two suffixes that differ before or at their
// first separator compare the same way in both orders.  Suffixes that agree
// through their separator (same characters, separator at the same offset) are
// exactly the suffixes sharing that prefix, so they form a contiguous run of
// the plain SA; the GSA orders such a run by position (string order).  A run
// is found from the LCP of plain-SA neighbours capped at the distance to the
// suffix's separator: Kasai's bound PLCP[i+1] >= PLCP[i] - 1 holds for the
// capped LCP too (the distance shrinks by one from i to i+1 inside a string
// and is 1 at a separator), so the chunked PLCP kernel carries over.  Each run
// is then re-sorted by (run number, position) with the radix sort.
#pragma once

#include "lcp.cuh"

namespace dcx {

// zeros_before[i] = separators in T[0, i); the first separator at or after i is
// sep_pos[zeros_before[i]].
struct OpSeparators {
    const uint8_t* text;
    uint32_t* zeros_before;
    uint32_t* sep_pos;
    __device__ uint32_t load(uint64_t k) const { return text[k] == 0; }
    __device__ void store(uint64_t k, uint32_t ex, uint32_t v) const {
        zeros_before[k] = ex;
        if (v) sep_pos[ex] = (uint32_t)k;
    }
};

// bad[0] += 1 for a last byte other than 0, and for every empty string (a 0 at
// position 0 or right after another 0) when n > 1: the inputs libsais64_gsa
// refuses.
__global__ void k_gsa_check(const uint8_t* __restrict__ text, uint64_t n, unsigned long long* __restrict__ bad) {
    unsigned long long b = 0;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint8_t ch = text[k];
        if (k == n - 1 && ch != 0) b++;
        if (n > 1 && ch == 0 && (k == 0 || text[k - 1] == 0)) b++;
    }
    if (b) atomicAdd(bad, b);
}

__device__ __forceinline__ uint64_t to_separator(const uint32_t* __restrict__ zeros_before,
                                                 const uint32_t* __restrict__ sep_pos, uint64_t i) {
    return (uint64_t)sep_pos[zeros_before[i]] - i + 1;  // chars of suffix i through its separator
}

// PLCP[i] = min(lcp(i, Phi[i]), to_separator(i) - 1 + through) for a text
// padded with at least 16 readable bytes past its end (16-byte aligned base):
// through = 1 counts the separator as a match (the runs of the GSA
// construction), through = 0 stops before it (the LCP of a GSA, where
// separators are distinct symbols and never match).
__global__ void k_plcp_to_separator(const uint8_t* __restrict__ text, uint64_t n, const uint32_t* __restrict__ phi,
                                    const uint32_t* __restrict__ zeros_before, const uint32_t* __restrict__ sep_pos,
                                    uint32_t* __restrict__ plcp, uint32_t through) {
    const uint64_t* tw = reinterpret_cast<const uint64_t*>(text);
    const uint64_t runs = (n + LCP_RUN - 1) / LCP_RUN;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = r * LCP_RUN;
        const uint64_t i1 = i0 + LCP_RUN < n ? i0 + LCP_RUN : n;
        uint64_t h = 0;
        for (uint64_t i = i0; i < i1; i++) {
            const uint32_t j = phi[i];
            if (j == PHI_NONE) {
                plcp[i] = 0;
                h = 0;
                continue;
            }
            const uint64_t shorter = n - (i > j ? i : (uint64_t)j);
            const uint64_t cap = to_separator(zeros_before, sep_pos, i) - 1 + through;
            const uint64_t lim = cap < shorter ? cap : shorter;
            if (h > lim) h = lim;
            while (h < lim) {
                const uint64_t d = load8_at(tw, i + h) ^ load8_at(tw, (uint64_t)j + h);
                if (d) {
                    h += (uint64_t)(__ffsll((long long)d) - 1) >> 3;
                    break;
                }
                h += 8;
            }
            if (h > lim) h = lim;
            plcp[i] = (uint32_t)h;
            h = h ? h - 1 : 0;
        }
    }
}

// head[k] = 1 where the plain-SA entry k does not agree with entry k-1 through
// its separator (a new run starts).
__global__ void k_gsa_heads(const uint32_t* __restrict__ sa32, uint64_t n, const uint32_t* __restrict__ plcp,
                            const uint32_t* __restrict__ zeros_before, const uint32_t* __restrict__ sep_pos,
                            uint8_t* __restrict__ head) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        uint8_t h = 1;
        if (k > 0) {
            const uint32_t i = sa32[k];
            h = (uint64_t)plcp[i] < to_separator(zeros_before, sep_pos, i);
        }
        head[k] = h;
    }
}

__global__ void k_gsa_scatter(uint64_t cnt, const uint32_t* __restrict__ slot, const uint32_t* __restrict__ pos,
                              uint32_t* __restrict__ sa32) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += (uint64_t)gridDim.x * blockDim.x)
        sa32[slot[j]] = pos[j];
}

__global__ void k_store_sa(const uint32_t* __restrict__ sa32, uint64_t n, void* __restrict__ out, int width) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        store_sa_entry(out, k, sa32[k], width);
}

}  // namespace dcx
