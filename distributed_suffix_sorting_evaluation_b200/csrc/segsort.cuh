// Phase-4 tie breaking: orders the suffixes inside groups whose first L chars
// are equal, with the difference-cover comparator of the reference
// (DCMergeSamples::operator<, lightweight_dcx/src/pdcx/merge_samples.hpp:87-109,
// and tie_break_ranks, merge_samples.hpp:262-306):
//     (d, r1, r2) = cmpDepthRanks[i mod X][j mod X]
//     i < j  <=>  ranks_i[r1] < ranks_j[r2]
// where ranks_i are the D sample ranks starting at the first sample >= i
// (get_global_ranks_pos, merge_samples.hpp:181-188).  The chars are already equal
// for the whole window (L >= X > d), so only the rank comparison remains.
//
// Groups are binned by size: up to 32 elements are sorted by a bitonic network
// inside W = 2..32 lanes of a warp (several groups per warp); 33..256 by one
// warp each (k_tie_warpsort, warpsort.cuh); up to 2048 by a bitonic network in
// shared memory of one CTA; larger groups are cut into
// 2048-chunks sorted the same way and then merged in rounds where every element
// finds its output slot by binary search in the partner run.
#pragma once

#include "common.cuh"

namespace dcx {

constexpr int MAX_X = 133;
constexpr int MAX_D = 12;
constexpr uint32_t INVALID_POS = 0xffffffffu;

struct DcDev {
    uint32_t X, D;
    FastDiv fx;  // division by X
    uint32_t next_rank[MAX_X];
    uint32_t dc[MAX_D];
    uint16_t cmp[MAX_X * MAX_X];  // r1 | r2 << 8
};

// Texts of the level: a group's elements all belong to one text s (the text id
// is part of the sort key); the comparator works on text-local positions and
// the text's rank slots start at rbase[s].
struct TieSeg {
    const uint32_t* segw;   // text of each sorted element, or null for one text
    const uint64_t* start;  // first position of each text
    const uint64_t* rbase;  // first rank slot of each text
};

__device__ __forceinline__ void tie_bases(const TieSeg& ts, uint64_t sorted_slot, uint64_t& pos0, uint64_t& slot0) {
    const uint32_t s = ts.segw ? ts.segw[sorted_slot] : 0u;
    pos0 = ts.start[s];
    slot0 = ts.rbase[s];
}

template <int D>
struct Rec {
    uint32_t pos;  // text-local position
    uint32_t res;  // pos mod X
    uint32_t r[D];
};

template <int D>
__device__ __forceinline__ Rec<D> load_rec(uint32_t pos, const uint32_t* __restrict__ rank_text, const FastDiv& fx,
                                           const uint32_t* next_rank) {
    Rec<D> r;
    r.pos = pos;
    r.res = 0;
    if (pos == INVALID_POS) {
#pragma unroll
        for (int k = 0; k < D; k++) r.r[k] = 0;
        return r;
    }
    uint32_t q;
    fdivmod(pos, fx, q, r.res);
    const uint64_t rp = (uint64_t)q * D + next_rank[r.res];
#pragma unroll
    for (int k = 0; k < D; k++) r.r[k] = __ldg(rank_text + rp + k);
    return r;
}

template <int D>
__device__ __forceinline__ uint32_t pick(const Rec<D>& a, uint32_t k) {
    uint32_t v = a.r[0];
#pragma unroll
    for (int t = 1; t < D; t++)
        if (k == (uint32_t)t) v = a.r[t];
    return v;
}

// a < b under the difference-cover comparator; invalid records sort last.
template <int D>
__device__ __forceinline__ bool dc_less(const Rec<D>& a, const Rec<D>& b, uint32_t X, const uint16_t* tab) {
    if (a.pos == INVALID_POS) return false;
    if (b.pos == INVALID_POS) return true;
    const uint16_t e = tab[a.res * X + b.res];
    return pick<D>(a, e & 0xffu) < pick<D>(b, e >> 8);
}

template <int D>
__device__ __forceinline__ Rec<D> shfl_xor_rec(const Rec<D>& a, int j) {
    Rec<D> o;
    o.pos = __shfl_xor_sync(0xffffffffu, a.pos, j);
    o.res = __shfl_xor_sync(0xffffffffu, a.res, j);
#pragma unroll
    for (int k = 0; k < D; k++) o.r[k] = __shfl_xor_sync(0xffffffffu, a.r[k], j);
    return o;
}

__device__ __forceinline__ void load_dc_smem(const DcDev& dc, uint16_t* tab, uint32_t* nr) {
    const uint32_t XX = dc.X * dc.X;
    for (uint32_t i = threadIdx.x; i < XX; i += blockDim.x) tab[i] = dc.cmp[i];
    for (uint32_t i = threadIdx.x; i < dc.X; i += blockDim.x) nr[i] = dc.next_rank[i];
    __syncthreads();
}

// Dynamic shared memory of k_tie_pair / k_tie_warp: the X*X comparator table
// and next_rank, sized for the level's X (a static MAX_X table would take 35 KB
// and cut the CTAs per SM for small covers).
__host__ __device__ inline size_t tie_tab_smem(uint32_t X) { return (((size_t)X * X * 2 + 15) & ~(size_t)15) + MAX_X * 4; }

__device__ __forceinline__ void tie_tab_ptrs(uint32_t X, uint16_t*& tab, uint32_t*& nr) {
    extern __shared__ __align__(16) uint8_t s_tab_dyn[];
    tab = reinterpret_cast<uint16_t*>(s_tab_dyn);
    nr = reinterpret_cast<uint32_t*>(s_tab_dyn + (((size_t)X * X * 2 + 15) & ~(size_t)15));
}

// Groups of exactly two elements, one per thread: the comparator needs one
// cover rank of each suffix, so only those two ranks are read.
__global__ __launch_bounds__(256) void k_tie_pair(const uint32_t* __restrict__ gstart, uint64_t ngroups,
                                                  uint32_t* __restrict__ sa, const uint32_t* __restrict__ rank_text,
                                                  const DcDev* __restrict__ dcp, TieSeg ts) {
    uint16_t* tab;
    uint32_t* nr;
    tie_tab_ptrs(dcp->X, tab, nr);
    load_dc_smem(*dcp, tab, nr);
    const uint32_t X = dcp->X, D = dcp->D;
    const FastDiv fx = dcp->fx;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t start = gstart[g];
        uint64_t pos0, slot0;
        tie_bases(ts, start, pos0, slot0);
        const uint32_t a = (uint32_t)(sa[start] - pos0), b = (uint32_t)(sa[start + 1] - pos0);
        uint32_t qa, ma, qb, mb;
        fdivmod(a, fx, qa, ma);
        fdivmod(b, fx, qb, mb);
        const uint16_t e = tab[ma * X + mb];
        const uint32_t ra = __ldg(rank_text + slot0 + (uint64_t)qa * D + nr[ma] + (e & 0xffu));
        const uint32_t rb = __ldg(rank_text + slot0 + (uint64_t)qb * D + nr[mb] + (e >> 8));
        if (!(ra < rb)) {  // a is not before b: the pair is reversed (distinct suffixes are totally ordered)
            sa[start] = (uint32_t)(b + pos0);
            sa[start + 1] = (uint32_t)(a + pos0);
        }
    }
}

// Groups of 2..W elements, 32/W groups per warp.
template <int D, int W>
__global__ __launch_bounds__(256) void k_tie_warp(const uint32_t* __restrict__ gstart, const uint32_t* __restrict__ gsize,
                                                  uint32_t ngroups, uint32_t* __restrict__ sa,
                                                  const uint32_t* __restrict__ rank_text, const DcDev* __restrict__ dcp,
                                                  TieSeg ts) {
    uint16_t* tab;
    uint32_t* nr;
    tie_tab_ptrs(dcp->X, tab, nr);
    load_dc_smem(*dcp, tab, nr);
    const uint32_t X = dcp->X;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp_global = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t g = warp_global * (32 / W) + lane / W;
    const uint32_t l = lane % W;
    bool valid = false;
    uint32_t start = 0;
    uint64_t pos0 = 0, slot0 = 0;
    if (g < ngroups) {
        start = gstart[g];
        valid = l < gsize[g];
        tie_bases(ts, start, pos0, slot0);
    }
    Rec<D> a = load_rec<D>(valid ? (uint32_t)(sa[start + l] - pos0) : INVALID_POS, rank_text + slot0, dcp->fx, nr);
#pragma unroll
    for (int k = 2; k <= W; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            Rec<D> b = shfl_xor_rec<D>(a, j);
            const bool up = (k == W) ? true : ((l & k) == 0);
            const bool lower = (l & j) == 0;
            // lower lane keeps the smaller element when sorting up
            // distinct suffixes are totally ordered, so a < b is !(b < a); for two
            // padding records either answer leaves padding in both lanes
            const bool b_less = dc_less<D>(b, a, X, tab);
            const bool take_b = (lower == up) ? b_less : !b_less;
            if (take_b) a = b;
        }
    }
    if (valid) sa[start + l] = (uint32_t)(a.pos + pos0);
}

// Groups (or chunks) of up to C elements, one at a time per CTA (the CTA loops
// over groups, so the comparator table is loaded once).  The group's records
// stay in place in shared memory as structure of arrays (position, residue mod
// X, D cover ranks); a bitonic network permutes 16-bit indices, and each
// comparison reads just the two ranks it needs.
template <int D, int C, int THREADS>
__global__ __launch_bounds__(THREADS) void k_tie_cta(const uint32_t* __restrict__ gstart, const uint32_t* __restrict__ gsize,
                                                     uint64_t ngroups, uint32_t* __restrict__ sa,
                                                     const uint32_t* __restrict__ rank_text,
                                                     const DcDev* __restrict__ dcp, TieSeg ts) {
    static_assert(C <= 65536, "indices are 16-bit");
    extern __shared__ __align__(16) uint32_t smem[];
    const uint32_t X = dcp->X;
    uint32_t* s_pos = smem;                                         // [C]
    uint32_t* s_rk = s_pos + C;                                     // [C * D]
    uint32_t* nr = s_rk + C * D;                                    // [MAX_X]
    uint16_t* s_idx = reinterpret_cast<uint16_t*>(nr + MAX_X);      // [C]
    uint16_t* tab = s_idx + C;                                      // [X * X]
    uint8_t* s_res = reinterpret_cast<uint8_t*>(tab + X * X);       // [C]
    load_dc_smem(*dcp, tab, nr);
    constexpr uint8_t NO_ELEM = 0xff;  // residue of a padding slot (X <= 133 < 255)
    auto less = [&](uint32_t ia, uint32_t ib) -> bool {
        const uint32_t ra = s_res[ia], rb = s_res[ib];
        if (ra == NO_ELEM) return false;
        if (rb == NO_ELEM) return true;
        const uint16_t e = tab[ra * X + rb];
        return s_rk[ia * D + (e & 0xffu)] < s_rk[ib * D + (e >> 8)];
    };
    for (uint64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const uint32_t start = gstart[g], size = gsize[g];
        uint64_t pos0, slot0;
        tie_bases(ts, start, pos0, slot0);
        // Every thread loads its C / THREADS elements and their D cover ranks with
        // independent loads, so one group costs two memory latencies (positions,
        // then ranks), not one per rank word.
        constexpr int PER = C / THREADS;
        static_assert(PER * THREADS == C, "C is a multiple of THREADS");
        uint32_t p[PER], rk[PER][D];
#pragma unroll
        for (int j = 0; j < PER; j++) {
            const uint32_t i = threadIdx.x + j * THREADS;
            p[j] = i < size ? (uint32_t)(sa[start + i] - pos0) : INVALID_POS;
        }
#pragma unroll
        for (int j = 0; j < PER; j++) {
            const uint32_t i = threadIdx.x + j * THREADS;
            uint32_t q = 0, r = NO_ELEM;
            if (p[j] != INVALID_POS) fdivmod(p[j], dcp->fx, q, r);
            s_pos[i] = p[j];
            s_res[i] = (uint8_t)r;
            s_idx[i] = (uint16_t)i;
            const uint32_t* src = rank_text + slot0 + (uint64_t)q * D + (r == NO_ELEM ? 0u : nr[r]);
#pragma unroll
            for (int k = 0; k < D; k++) rk[j][k] = p[j] != INVALID_POS ? __ldg(src + k) : 0u;
        }
#pragma unroll
        for (int j = 0; j < PER; j++) {
            const uint32_t i = threadIdx.x + j * THREADS;
#pragma unroll
            for (int k = 0; k < D; k++) s_rk[i * D + k] = rk[j][k];
        }
        __syncthreads();
#pragma unroll
        for (uint32_t k = 2; k <= (uint32_t)C; k <<= 1) {
#pragma unroll
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
                for (uint32_t p = threadIdx.x; p < (uint32_t)C / 2; p += THREADS) {
                    const uint32_t i = ((p & ~(j - 1)) << 1) | (p & (j - 1));  // j is a power of two
                    const uint32_t q = i + j;
                    const bool up = (i & k) == 0;
                    const uint32_t a = s_idx[i], b = s_idx[q];
                    const bool swap = up ? less(b, a) : less(a, b);
                    if (swap) {
                        s_idx[i] = (uint16_t)b;
                        s_idx[q] = (uint16_t)a;
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t i = threadIdx.x; i < size; i += THREADS) sa[start + i] = (uint32_t)(s_pos[s_idx[i]] + pos0);
        __syncthreads();  // shared arrays are reused by the next group
    }
}

template <int D, int C>
inline size_t tie_cta_smem(uint32_t X) {
    return sizeof(uint32_t) * ((size_t)C * (1 + D) + MAX_X) + sizeof(uint16_t) * ((size_t)C + (size_t)X * X) + C + 16;
}

// One merge round for groups larger than a chunk.  Flat element f belongs to
// big group g (offsets[g] <= f < offsets[g+1]); runs of width w inside the group
// are sorted; pairs of runs are merged from src into dst.
template <int D>
__global__ __launch_bounds__(256) void k_tie_merge(const uint64_t* __restrict__ offsets, uint32_t ngroups,
                                                   const uint32_t* __restrict__ gstart, uint64_t total, uint32_t w,
                                                   const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                                   const uint32_t* __restrict__ rank_text, const DcDev* __restrict__ dcp,
                                                   TieSeg ts) {
    __shared__ uint16_t tab[MAX_X * MAX_X];
    __shared__ uint32_t nr[MAX_X];
    load_dc_smem(*dcp, tab, nr);
    const uint32_t X = dcp->X;
    for (uint64_t f = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; f < total; f += (uint64_t)gridDim.x * blockDim.x) {
        // group of f
        uint32_t lo = 0, hi = ngroups;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= f) lo = mid; else hi = mid;
        }
        const uint32_t g = lo;
        const uint64_t size = offsets[g + 1] - offsets[g];
        const uint64_t o = f - offsets[g];
        const uint64_t base = gstart[g];
        const uint64_t run = o / w;
        const uint64_t pair_base = (run & ~1ull) * w;
        const bool left = (run & 1ull) == 0;
        const uint64_t own_start = run * w;
        uint64_t p_start, p_end;
        if (left) {
            p_start = own_start + w;
            p_end = p_start + w < size ? p_start + w : size;
        } else {
            p_start = own_start - w;
            p_end = own_start;
        }
        uint64_t pos0, slot0;
        tie_bases(ts, base, pos0, slot0);
        const uint32_t* rt = rank_text + slot0;
        const Rec<D> me = load_rec<D>((uint32_t)(src[base + o] - pos0), rt, dcp->fx, nr);
        uint64_t a = p_start, b = p_end;  // count partner elements < me
        if (p_start < size) {
            while (a < b) {
                uint64_t mid = (a + b) >> 1;
                Rec<D> other = load_rec<D>((uint32_t)(src[base + mid] - pos0), rt, dcp->fx, nr);
                if (dc_less<D>(other, me, X, tab)) a = mid + 1; else b = mid;
            }
        } else {
            a = p_start;
        }
        const uint64_t before = (p_start < size ? a - p_start : 0);
        dst[base + pair_base + (o - own_start) + before] = (uint32_t)(me.pos + pos0);
    }
}

}  // namespace dcx
