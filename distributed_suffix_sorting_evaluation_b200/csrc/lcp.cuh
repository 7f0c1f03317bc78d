// LCP array from a text and its suffix array (the first consumer of an SA; the
// reference's tree offers it through libsais64_plcp / libsais64_lcp,
// libsais/include/libsais64.h:236-263, with the same conventions):
//   PLCP[i] = lcp(suffix i, suffix Phi[i]), Phi[SA[k]] = SA[k-1], PLCP[SA[0]] = 0
//   LCP[k]  = PLCP[SA[k]]
// Phi is one scatter.  PLCP follows Kasai et al.'s bound PLCP[i+1] >= PLCP[i] - 1
// inside runs of LCP_RUN consecutive positions per thread (each run starts from
// 0), comparing 8 chars per step with aligned word loads.  LCP is one gather.
#pragma once

#include "common.cuh"

namespace dcx {

constexpr uint32_t LCP_RUN = 64;
constexpr uint32_t PHI_NONE = 0xffffffffu;

__device__ __forceinline__ uint64_t load_sa_u(const void* sa, uint64_t k, int width) {
    if (width == 32) return reinterpret_cast<const uint32_t*>(sa)[k];
    if (width == 64) return reinterpret_cast<const uint64_t*>(sa)[k];
    const uint8_t* b = reinterpret_cast<const uint8_t*>(sa) + 5 * k;
    return (uint64_t)b[0] | ((uint64_t)b[1] << 8) | ((uint64_t)b[2] << 16) | ((uint64_t)b[3] << 24) |
           ((uint64_t)b[4] << 32);
}

// The SA as uint32 (coalesced: 40-bit entries are read four at a time as five
// aligned words when the buffer is 4-byte aligned).
__global__ void k_sa_to_u32(const void* __restrict__ sa, int width, uint64_t n, uint32_t* __restrict__ sa32) {
    const bool quad40 = width == 40 && ((uintptr_t)sa & 3) == 0;
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q * 4 < n; q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k0 = q * 4;
        if (quad40 && k0 + 4 <= n) {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(sa) + q * 5;  // 20 bytes = 4 entries
            const uint32_t w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
            sa32[k0] = w0;                             // bytes 0-3 (byte 4 is the high byte, 0 here)
            sa32[k0 + 1] = (w1 >> 8) | (w2 << 24);     // bytes 5-8
            sa32[k0 + 2] = (w2 >> 16) | (w3 << 16);    // bytes 10-13
            sa32[k0 + 3] = (w3 >> 24) | (w[4] << 8);   // bytes 15-18
        } else {
            for (uint64_t k = k0; k < k0 + 4 && k < n; k++) sa32[k] = (uint32_t)load_sa_u(sa, k, width);
        }
    }
}

// phi[SA[k]] = SA[k-1] (PHI_NONE for k = 0).
__global__ void k_phi(const uint32_t* __restrict__ sa32, uint64_t n, uint32_t* __restrict__ phi) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        phi[sa32[k]] = k ? sa32[k - 1] : PHI_NONE;
}

// 8 chars starting at p from a text padded with at least 8 readable bytes past
// its end (16-byte aligned base): two aligned words and a funnel shift.
__device__ __forceinline__ uint64_t load8_at(const uint64_t* __restrict__ tw, uint64_t p) {
    const uint64_t a = p >> 3;
    const uint32_t s = (uint32_t)(p & 7) * 8;
    const uint64_t lo = __ldg(tw + a);
    if (!s) return lo;
    return (lo >> s) | (__ldg(tw + a + 1) << (64 - s));
}

__global__ void k_plcp(const uint8_t* __restrict__ text, uint64_t n, const uint32_t* __restrict__ phi,
                       uint32_t* __restrict__ plcp) {
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
            const uint64_t lim = n - (i > j ? i : (uint64_t)j);  // the shorter suffix's length
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

// LCP[k] = PLCP[SA[k]], written with `width` bits per entry.
__global__ void k_lcp_gather(const uint32_t* __restrict__ sa32, const uint32_t* __restrict__ plcp, uint64_t n,
                             void* __restrict__ out, int width, bool permuted) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = permuted ? plcp[k] : plcp[sa32[k]];
        if (width == 64) reinterpret_cast<uint64_t*>(out)[k] = v;
        else reinterpret_cast<uint32_t*>(out)[k] = v;
    }
}

}  // namespace dcx
