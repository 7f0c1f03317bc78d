// Burrows-Wheeler transform from a text and its suffix array, in the convention
// of libsais64_bwt (libsais/include/libsais64.h:125-135): the last column of
// the sorted rotations of T$, with the sentinel's row left out,
//   U[0] = T[n-1]
//   U[j] = T[SA[j-1] - 1]   for 1 <= j < p
//   U[j] = T[SA[j] - 1]     for p <= j < n
// where the primary index p = 1 + (the k with SA[k] = 0) is where the sentinel
// row would stand.  One pass over the SA finds p and checks every entry is
// below n with exactly one 0 (so the gather cannot read outside the text); a
// second pass gathers.
#pragma once

#include "lcp.cuh"

namespace dcx {

struct BwtScan {
    unsigned long long first_zero;  // smallest k with SA[k] = 0 (all ones: none)
    unsigned long long zeros;       // entries equal to 0
    unsigned long long out_of_range;  // entries >= n
};

__global__ void k_bwt_primary(const void* __restrict__ sa, int width, uint64_t n, BwtScan* __restrict__ st) {
    unsigned long long zeros = 0, bad = 0;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t s = load_sa_u(sa, k, width);
        if (s == 0) {
            zeros++;
            atomicMin(&st->first_zero, (unsigned long long)k);
        }
        bad += s >= n;
    }
    // a valid SA has one zero and nothing out of range: these atomics are rare
    if (zeros) atomicAdd(&st->zeros, zeros);
    if (bad) atomicAdd(&st->out_of_range, bad);
}

// Requires the checks of k_bwt_primary to have passed: 1 <= p <= n, SA[k] in
// [1, n) for every k != p - 1.
__global__ void k_bwt_gather(const uint8_t* __restrict__ text, uint64_t n, const void* __restrict__ sa, int width,
                             uint64_t p, uint8_t* __restrict__ u) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        uint8_t ch;
        if (j == 0) {
            ch = text[n - 1];
        } else {
            const uint64_t k = j < p ? j - 1 : j;
            ch = __ldg(text + load_sa_u(sa, k, width) - 1);
        }
        u[j] = ch;
    }
}

}  // namespace dcx
