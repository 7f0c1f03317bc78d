// dcx_build_sa_noalloc: suffix array of a short device-resident text without
// any device allocation.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they need
// a suffix array -- code running inside CUDA stream capture (allocation calls
// are not capturable), allocators' own callbacks, and hosts whose device memory
// is fully pre-reserved by another framework's pool so that any new allocation
// would fail or fragment it.  They pass the text and the output buffer; every
// other byte of working memory comes from one file-scope device array.
//
// The kernel is a variant of the in-CTA base case (prefix doubling with a
// bitonic sort, small_sa.cuh) whose key/index/rank arrays live in that global
// scratch array instead of shared memory, which lifts the length limit from
// 2048 to NOALLOC_MAX_N chars.  One CTA; every array it reads is initialised by
// the kernel itself, so nothing has to start at zero.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "common.cuh"
#include "dcx_gpu.h"

namespace dcx {
namespace {

constexpr uint32_t NOALLOC_MAX_N = 32768;     // longest text (chars)
constexpr int NOALLOC_THREADS = 1024;
// key (8 B) + index (4 B) + rank (4 B) per char: 512 KiB held by every GPU that
// loads the library, until the process exits.
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)NOALLOC_MAX_N * 16;

static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

__global__ __launch_bounds__(NOALLOC_THREADS) void k_small_sa_scratch(const uint8_t* __restrict__ text, uint32_t n,
                                                                      uint32_t* __restrict__ sa, uint8_t* scratch) {
    __shared__ uint32_t scan_sm[NOALLOC_THREADS / 32 + 1];
    __shared__ uint32_t s_done;
    uint64_t* key = reinterpret_cast<uint64_t*>(scratch);
    uint32_t* idx = reinterpret_cast<uint32_t*>(scratch + (size_t)NOALLOC_MAX_N * 8);
    uint32_t* rank = reinterpret_cast<uint32_t*>(scratch + (size_t)NOALLOC_MAX_N * 12);
    if (n == 0) return;
    if (n == 1) {
        if (threadIdx.x == 0) sa[0] = 0;
        return;
    }
    uint32_t C = 2;
    while (C < n) C <<= 1;
    // ranks start as byte + 1 so that 0 stays below every char (end of text)
    for (uint32_t i = threadIdx.x; i < n; i += NOALLOC_THREADS) rank[i] = (uint32_t)text[i] + 1u;
    __syncthreads();
    const uint32_t per = (C + NOALLOC_THREADS - 1) / NOALLOC_THREADS;  // blocked layout for the rename scan
    for (uint32_t h = 1;; h <<= 1) {
        for (uint32_t i = threadIdx.x; i < C; i += NOALLOC_THREADS) {
            key[i] = i < n ? (((uint64_t)rank[i] << 32) | (i + h < n ? rank[i + h] : 0u)) : ~0ull;
            idx[i] = i;
        }
        __syncthreads();
        for (uint32_t k = 2; k <= C; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t p = threadIdx.x; p < C / 2; p += NOALLOC_THREADS) {
                    const uint32_t i = 2 * j * (p / j) + (p % j);
                    const uint32_t q = i + j;
                    const bool up = (i & k) == 0;
                    const uint64_t a = key[i], c = key[q];
                    const uint32_t ia = idx[i], ic = idx[q];
                    const bool swap = up ? (c < a || (c == a && ic < ia)) : (a < c || (a == c && ia < ic));
                    if (swap) {
                        key[i] = c;
                        key[q] = a;
                        idx[i] = ic;
                        idx[q] = ia;
                    }
                }
                __syncthreads();
            }
        }
        // rename: rank = 1 + number of distinct pairs before
        uint32_t local = 0;
        const uint32_t b0 = threadIdx.x * per;
        for (uint32_t e = 0; e < per; e++) {
            const uint32_t k = b0 + e;
            if (k < n) local += (k == 0 || key[k] != key[k - 1]);
        }
        uint32_t total;
        uint32_t ex = block_excl_scan<NOALLOC_THREADS>(local, scan_sm, total);
        for (uint32_t e = 0; e < per; e++) {
            const uint32_t k = b0 + e;
            if (k < n) {
                ex += (k == 0 || key[k] != key[k - 1]);
                rank[idx[k]] = ex;
            }
        }
        if (threadIdx.x == 0) s_done = (total == n) || (h >= n);
        __syncthreads();
        if (s_done) break;
    }
    for (uint32_t k = threadIdx.x; k < n; k += NOALLOC_THREADS) sa[k] = idx[k];
}

// Device address of g_noalloc_scratch, looked up once per device.
constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[MAX_DEVICES] = {};

}  // namespace
}  // namespace dcx

extern "C" int dcx_build_sa_noalloc(const uint8_t* text_dev, uint64_t n, uint32_t* sa_dev, void* stream) {
    using namespace dcx;
    if (n > NOALLOC_MAX_N) return DCX_ERR_ARG;  // longer texts need dcx_build_sa
    if (n == 0) return DCX_OK;
    if (!text_dev || !sa_dev) return DCX_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return DCX_ERR_CUDA;
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            // host code may not use g_noalloc_scratch's name as a device address:
            // ask the runtime for it, once, with this device current
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DCX_ERR_CUDA;
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    k_small_sa_scratch<<<1, NOALLOC_THREADS, 0, (cudaStream_t)stream>>>(text_dev, (uint32_t)n, sa_dev,
                                                                         (uint8_t*)scratch);
    return cudaGetLastError() == cudaSuccess ? DCX_OK : DCX_ERR_CUDA;
}
