// Shared device/host helpers of the DCX engine: error plumbing, launch
// bookkeeping, warp/block scans and the device-wide three-phase scan used by
// naming, compaction and group detection.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "dcx_gpu.h"

namespace dcx {

// Host-side error carrying a dcx status code; every C-ABI entry converts it.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define DCX_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            if (e_ == cudaErrorMemoryAllocation)                                         \
                throw ::dcx::Error(DCX_ERR_OOM, std::string("out of device memory: ") + #call); \
            throw ::dcx::Error(DCX_ERR_CUDA, std::string(cudaGetErrorString(e_)) + " at " +    \
                                                 __FILE__ + ":" + std::to_string(__LINE__)); \
        }                                                                                \
    } while (0)

#define DCX_CHECK_LAUNCH() DCX_CUDA(cudaGetLastError())

inline uint64_t div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Device error word bits (set by kernels that give up a bounded wait or detect
// an out-of-range index; the host turns a nonzero word into an error code).
enum : uint32_t { DEV_ERR_TIMEOUT = 1u, DEV_ERR_RANGE = 2u };

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Inclusive warp scan of a 32-bit sum.
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane_id() >= (uint32_t)o) v += t;
    }
    return v;
}

__device__ __forceinline__ uint64_t warp_incl_scan64(uint64_t v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane_id() >= (uint32_t)o) v += t;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the exclusive prefix and
// writes the block total.  `smem` needs THREADS/32 + 1 slots.
template <int THREADS, typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* smem, T& total) {
    constexpr int WARPS = THREADS / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < WARPS ? smem[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < WARPS) smem[lane] = wi - w;
        if (lane == WARPS - 1) smem[WARPS] = wi;
    }
    __syncthreads();
    T r = smem[warp] + inc - v;
    total = smem[WARPS];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan in three phases (chunk reduce, scan of chunk sums,
// chunk rescan).  Op supplies   T load(uint64_t i)   and
//   void store(uint64_t i, T exclusive_prefix, T value)   for i < n.
// No inter-CTA waits, so nothing can spin.
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// An operator may also supply   void load16(uint64_t base, uint64_t n, T* v)
// (the 16 values of elements base..base+15, zero past n; base is a multiple of
// 16), which it implements with vector loads; both scan phases then give each
// thread 16 consecutive elements.
template <typename Op, typename = void>
struct ScanVec : std::false_type {};
template <typename Op>
struct ScanVec<Op, std::void_t<decltype(&Op::load16)>> : std::true_type {};

// Every CTA owns a contiguous run of `tpc` tiles (chunk) and walks it in
// order, so a scan of a billion elements runs as a few hundred CTAs rather
// than hundreds of thousands of one-tile CTAs.
//
// Reduce phase: loads are warp-striped (lane l of warp w reads element
// w*32*ITEMS + it*32 + l of the tile in iteration it), so every load
// instruction is coalesced; one sum per chunk.
template <typename T, typename Op>
__global__ __launch_bounds__(SCAN_THREADS) void k_scan_reduce(Op op, uint64_t n, T* chunk_sums, uint64_t tpc) {
    __shared__ T sm[SCAN_THREADS / 32 + 1];
    const uint64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    const uint64_t t0 = (uint64_t)blockIdx.x * tpc;
    const uint64_t t1 = t0 + tpc < ntiles ? t0 + tpc : ntiles;
    T acc = T(0);
    for (uint64_t tile = t0; tile < t1; tile++) {
        if constexpr (ScanVec<Op>::value) {
            static_assert(SCAN_ITEMS == 16, "load16 covers a thread's items");
            const uint64_t base = tile * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
            if (base < n) {
                T v[16];
                op.load16(base, n, v);
#pragma unroll
                for (int it = 0; it < 16; it++) acc += v[it];
            }
        } else {
            const uint64_t base = tile * SCAN_TILE + (uint64_t)(threadIdx.x >> 5) * 32 * SCAN_ITEMS + (threadIdx.x & 31);
#pragma unroll
            for (int it = 0; it < SCAN_ITEMS; it++) {
                const uint64_t i = base + (uint64_t)it * 32;
                if (i < n) acc += op.load(i);
            }
        }
    }
    T total;
    block_excl_scan<SCAN_THREADS>(acc, sm, total);
    if (threadIdx.x == 0) chunk_sums[blockIdx.x] = total;
}

// Single-CTA exclusive scan of the chunk sums (in place); also writes the grand total.
template <typename T>
__global__ __launch_bounds__(1024) void k_scan_tile_sums(T* sums, uint64_t count, T* grand_total) {
    __shared__ T sm[1024 / 32 + 1];
    T carry = T(0);
    for (uint64_t base = 0; base < count; base += 1024) {
        uint64_t i = base + threadIdx.x;
        T v = i < count ? sums[i] : T(0);
        T total;
        T ex = block_excl_scan<1024>(v, sm, total);
        if (i < count) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0 && grand_total) *grand_total = carry;
}

// Apply phase: thread t owns SCAN_ITEMS consecutive elements of each tile
// (each thread's loads walk one contiguous 16-element run, fully used through
// L1); the chunk's running prefix carries from tile to tile.
template <typename T, typename Op>
__global__ __launch_bounds__(SCAN_THREADS) void k_scan_apply(Op op, uint64_t n, const T* chunk_prefix, uint64_t tpc) {
    __shared__ T sm[SCAN_THREADS / 32 + 1];
    const uint64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    const uint64_t t0 = (uint64_t)blockIdx.x * tpc;
    const uint64_t t1 = t0 + tpc < ntiles ? t0 + tpc : ntiles;
    T carry = chunk_prefix[blockIdx.x];
    for (uint64_t tile = t0; tile < t1; tile++) {
        const uint64_t base = tile * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
        T vals[SCAN_ITEMS];
        T acc = T(0);
        if constexpr (ScanVec<Op>::value) {
            if (base < n) {
                op.load16(base, n, vals);
            } else {
#pragma unroll
                for (int it = 0; it < SCAN_ITEMS; it++) vals[it] = T(0);
            }
#pragma unroll
            for (int it = 0; it < SCAN_ITEMS; it++) acc += vals[it];
        } else {
#pragma unroll
            for (int it = 0; it < SCAN_ITEMS; it++) {
                const uint64_t i = base + it;
                vals[it] = i < n ? op.load(i) : T(0);
                acc += vals[it];
            }
        }
        T total;
        const T ex = block_excl_scan<SCAN_THREADS>(acc, sm, total);
        T run = carry + ex;
#pragma unroll
        for (int it = 0; it < SCAN_ITEMS; it++) {
            const uint64_t i = base + it;
            if (i < n) op.store(i, run, vals[it]);
            run += vals[it];
        }
        carry += total;
    }
}

// SA entry k of an output of `width` bits (32, 64, or 40 = 5 little-endian bytes).
__device__ __forceinline__ void store_sa_entry(void* out, uint64_t k, uint32_t v, int width) {
    if (width == 32) reinterpret_cast<uint32_t*>(out)[k] = v;
    else if (width == 64) reinterpret_cast<uint64_t*>(out)[k] = v;
    else {
        uint8_t* o = reinterpret_cast<uint8_t*>(out) + 5 * k;
        o[0] = (uint8_t)v;
        o[1] = (uint8_t)(v >> 8);
        o[2] = (uint8_t)(v >> 16);
        o[3] = (uint8_t)(v >> 24);
        o[4] = 0;
    }
}

// Unsigned 32-bit division by a divisor fixed per launch (Granlund and
// Montgomery's round-up method): with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, q = (umulhi(m, a) + a) >> l for every
// 32-bit a (the sum is formed in 64 bits).  A runtime-divisor '%' or '/' costs
// a few dozen instructions; this costs four.
struct FastDiv {
    uint32_t d, m, l;
};

inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f{d, 0, 0};
    while ((1ull << f.l) < d) f.l++;
    f.m = (uint32_t)((((1ull << 32) * ((1ull << f.l) - d)) / d) + 1);
    return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t a, const FastDiv& f) {
    return (uint32_t)(((uint64_t)__umulhi(f.m, a) + a) >> f.l);
}
__device__ __forceinline__ void fdivmod(uint32_t a, const FastDiv& f, uint32_t& q, uint32_t& r) {
    q = fdiv(a, f);
    r = a - q * f.d;
}

// 16 flag bytes f[base..base+15] plus f[base+16] (`past` when base+16 >= n);
// base is a multiple of 16 and the array is 16-byte aligned.  Bytes at or past
// n read as `past`.
__device__ __forceinline__ void load_flags17(const uint8_t* __restrict__ f, uint64_t base, uint64_t n, uint32_t past,
                                             uint32_t* b) {
    if (base + 16 <= n) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(f + base));
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 16; k++) b[k] = (w[k >> 2] >> (8 * (k & 3))) & 0xffu;
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) b[k] = base + k < n ? f[base + k] : past;
    }
    b[16] = base + 16 < n ? f[base + 16] : past;
}

}  // namespace dcx
