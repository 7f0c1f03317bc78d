// Sequential host emulation of the few CUDA builtins the LCP/BWT/GSA kernels
// use, so their source (csrc/lcp.cuh, bwt.cuh, gsa.cuh, unchanged) compiles as
// host C++ and runs on a CPU.  LAUNCH(kernel, grid, block, args...) runs every
// (block, thread) of a launch one after another: exact for kernels without
// shared memory or barriers whose threads write disjoint elements, which holds
// for the grid-stride kernels tested here.
#pragma once
#include <cstdint>
#include <cstring>
#include <cstddef>
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __restrict__
struct Dim { unsigned x = 1, y = 1, z = 1; };
inline Dim blockIdx, threadIdx, gridDim, blockDim;
template <typename T> inline T __ldg(const T* p) { return *p; }
inline int __ffsll(long long x) { return __builtin_ffsll(x); }
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) { auto o = *p; *p += v; return o; }
inline unsigned long long atomicMin(unsigned long long* p, unsigned long long v) { auto o = *p; if (v < *p) *p = v; return o; }
#define LAUNCH(K, G, B, ...)                                                  \
    for (unsigned _b = 0; _b < (unsigned)(G); _b++)                            \
        for (unsigned _t = 0; _t < (unsigned)(B); _t++) {                      \
            blockIdx.x = _b; threadIdx.x = _t; gridDim.x = (G); blockDim.x = (B); \
            K(__VA_ARGS__);                                                   \
        }
