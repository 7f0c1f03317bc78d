// Two-step Phi for long texts (the direct k_phi of lcp.cuh scatters one
// 4-byte store per entry into a 32-byte sector, which makes L2 fetch and write
// back the whole sector once the array outgrows L2).
#pragma once

#include "lcp.cuh"

namespace dcx {

// k_phi_records lays out (SA[k], SA[k-1]) and histograms the digit
// (SA[k] >> shift) & 255, the top 8 bits of the position; one radix pass on that
// digit groups the pairs into 256 contiguous position ranges;
// k_phi_scatter then stores them in that order, so the stores of concurrent
// CTAs land in a few megabytes of phi that L2 fills completely before writing
// back.
__global__ void k_phi_records(const uint32_t* __restrict__ sa32, uint64_t n, uint32_t* __restrict__ dst,
                              uint32_t* __restrict__ val, uint32_t* __restrict__ hist, uint32_t shift) {
    __shared__ uint32_t h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t d = sa32[k];
        dst[k] = d;
        val[k] = k ? sa32[k - 1] : PHI_NONE;
        atomicAdd(&h[(d >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

__global__ void k_phi_scatter(const uint32_t* __restrict__ dst, const uint32_t* __restrict__ val, uint64_t n,
                              uint32_t* __restrict__ phi) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        phi[dst[k]] = val[k];
}

}  // namespace dcx
