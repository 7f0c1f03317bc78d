// Warp-per-group sorts for tie groups of 33..256 elements: the refinement of
// round-0 groups by the rest of their window (one 64-bit window word), and the
// cover-rank tie break.
//
// Repetitive texts (many copies of one sequence) put almost every suffix into
// groups of this size -- one element per copy -- so these two sorts carry most
// of such a build.  One warp owns one group; every lane holds E elements in
// registers in blocked layout (lane l holds sorted slots l*E .. l*E+E-1), and a
// bitonic network orders them: exchanges between slots of one lane are register
// moves, exchanges between lanes shuffles.  The element is small -- (window
// word, position) for the refinement, (slot, residue) for the tie break, whose
// cover ranks stay in the warp's slice of shared memory -- and every comparison
// is branch-free, so lanes of opposite sort direction do not diverge.  No block
// barrier is involved: the groups of one CTA never wait for each other.
#pragma once

#include "keys.cuh"
#include "segsort.cuh"

namespace dcx {

constexpr int WSORT_WARPS = 8;  // warps per CTA

struct KeyPos {  // refinement element: window word, position (0xffffffff = past the group)
    uint64_t key;
    uint32_t pos;
};
__device__ __forceinline__ KeyPos shfl_xor_el(const KeyPos& a, int m) {
    KeyPos o;
    o.key = __shfl_xor_sync(0xffffffffu, a.key, m);
    o.pos = __shfl_xor_sync(0xffffffffu, a.pos, m);
    return o;
}
__device__ __forceinline__ KeyPos sel(bool c, const KeyPos& a, const KeyPos& b) {
    return KeyPos{c ? a.key : b.key, c ? a.pos : b.pos};
}

struct SlotRes {  // tie-break element: offset of its cover ranks (slot * D), residue mod X
    uint32_t rk, res;
};
__device__ __forceinline__ SlotRes shfl_xor_el(const SlotRes& a, int m) {
    return SlotRes{__shfl_xor_sync(0xffffffffu, a.rk, m), __shfl_xor_sync(0xffffffffu, a.res, m)};
}
__device__ __forceinline__ SlotRes sel(bool c, const SlotRes& a, const SlotRes& b) {
    return SlotRes{c ? a.rk : b.rk, c ? a.res : b.res};
}

// One step (k, j) of the network with j < E: both slots in the lane.
template <int E, int J, typename T, typename Less>
__device__ __forceinline__ void wb_in_lane(T (&v)[E], uint32_t lane, uint32_t k, Less less) {
    if constexpr (J < E) {
#pragma unroll
        for (int e = 0; e < E; e++) {
            if (e & J) continue;
            const bool up = ((lane * E + e) & k) == 0;
            const T a = v[e], b = v[e | J];
            // ascending: swap iff b < a; descending: iff a < b
            const bool sw = less(sel(up, b, a), sel(up, a, b));
            v[e] = sel(sw, b, a);
            v[e | J] = sel(sw, a, b);
        }
    }
}

// Ascending bitonic sort of the 32*E elements of a warp (blocked layout) under
// a strict weak order less(x, y).  For a slot pair lo < hi the step swaps iff
// less(hi, lo) (ascending run) or less(lo, hi) (descending run); the two lanes
// of a cross-lane pair evaluate that same comparison, so they agree.  The k and
// j loops stay rolled (k and j are warp-uniform), which keeps the code small.
template <int E, typename T, typename Less>
__device__ __forceinline__ void warp_bitonic(T (&v)[E], uint32_t lane, Less less) {
    constexpr uint32_t N = 32 * E;
#pragma unroll 1
    for (uint32_t k = 2; k <= N; k <<= 1) {
#pragma unroll 1
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= (uint32_t)E) {  // partner slot in lane ^ (j / E)
                const int m = (int)(j / E);
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const T mine = v[e];
                    const T other = shfl_xor_el(mine, m);
                    const uint32_t i = lane * E + e;
                    const bool up = (i & k) == 0;
                    const bool lower = (i & j) == 0;
                    const T lo = sel(lower, mine, other), hi = sel(lower, other, mine);
                    const bool sw = less(sel(up, hi, lo), sel(up, lo, hi));
                    v[e] = sel(sw, other, mine);
                }
            } else if (j == 4) {
                wb_in_lane<E, 4>(v, lane, k, less);
            } else if (j == 2) {
                wb_in_lane<E, 2>(v, lane, k, less);
            } else {
                wb_in_lane<E, 1>(v, lane, k, less);
            }
        }
    }
}

// ---- refinement by the rest of the window (one 64-bit word) --------------------
// Groups of up to 32*E elements (all of one text), sorted by the window word of
// chars [off, L) (a RefineSegPlan with W = 1, as k_refine_seg) and written back
// with head flags where the word changes; equal windows stay tied, in any order.
//
// In a group of copies of one sequence most elements share the word of the
// group's first element ("the majority") and a few differ (a mutation in the
// copy).  When at most 32 differ, those are sorted one per lane and the
// majority is written as one block between the smaller and the larger ones;
// otherwise the whole group goes through the E-per-lane network.  Slots past the
// group hold (max word, 0xffffffff) and sort last: positions are below 2^32 - 1,
// so ordering by (word, position) puts them after every element.
template <int E, typename CharT>
__global__ __launch_bounds__(32 * WSORT_WARPS, 3) void k_refine_warpsort(
    const CharT* __restrict__ text, SegView sv, const uint32_t* __restrict__ segw, const uint32_t* __restrict__ gstart,
    const uint32_t* __restrict__ gsize, uint64_t ngroups, uint32_t* __restrict__ sa, uint8_t* __restrict__ head,
    RefineSegPlan plan) {
    __shared__ KeyPos s_other[WSORT_WARPS][32];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    auto less = [](const KeyPos& x, const KeyPos& y) { return x.key < y.key || (x.key == y.key && x.pos < y.pos); };
    const uint64_t nwarps = (uint64_t)gridDim.x * WSORT_WARPS;
    for (uint64_t g = (uint64_t)blockIdx.x * WSORT_WARPS + warp; g < ngroups; g += nwarps) {
        const uint32_t start = gstart[g], size = gsize[g];
        const uint64_t end = seg_end(sv, segw ? segw[start] : 0u);
        KeyPos v[E];
        // lane l starts with slots e*32 + l (coalesced loads)
#pragma unroll
        for (int e = 0; e < E; e++) {
            const uint32_t i = e * 32 + lane;
            v[e].pos = i < size ? sa[start + i] : 0xffffffffu;
        }
#pragma unroll
        for (int e = 0; e < E; e++)
            v[e].key = v[e].pos != 0xffffffffu
                           ? window_value_t(text, (uint64_t)v[e].pos + plan.off[0], end, plan.rp[0])
                           : ~0ull;
        const uint64_t ref = __shfl_sync(0xffffffffu, v[0].key, 0);  // slot 0 (a group has >= 2 elements)
        uint32_t eqm[E], n_other = 0;
#pragma unroll
        for (int e = 0; e < E; e++) {
            const bool valid = v[e].pos != 0xffffffffu;
            eqm[e] = __ballot_sync(0xffffffffu, valid && v[e].key == ref);
            n_other += __popc(__ballot_sync(0xffffffffu, valid && v[e].key != ref));
        }
        if (n_other <= 32) {
            // the differing elements, one per lane, sorted; the majority block goes
            // after the `below` of them whose word is smaller than the majority's
            uint32_t base_o = 0, base_m = 0;
#pragma unroll
            for (int e = 0; e < E; e++) {
                const bool valid = v[e].pos != 0xffffffffu;
                const bool other = valid && !((eqm[e] >> lane) & 1u);
                const uint32_t om = __ballot_sync(0xffffffffu, other);
                if (other) s_other[warp][base_o + __popc(om & lt)] = v[e];
                base_o += __popc(om);
            }
            __syncwarp();
            KeyPos o[1];
            o[0] = lane < n_other ? s_other[warp][lane] : KeyPos{~0ull, 0xffffffffu};
            warp_bitonic<1>(o, lane, less);
            const uint32_t below = __popc(__ballot_sync(0xffffffffu, lane < n_other && o[0].key < ref));
            const uint32_t n_eq = size - n_other;
            const uint64_t prev = __shfl_up_sync(0xffffffffu, o[0].key, 1);
            if (lane < n_other) {
                const uint32_t slot = lane < below ? lane : lane + n_eq;
                sa[start + slot] = o[0].pos;
                if (slot > 0) head[start + slot] = (lane == below ? ref : prev) != o[0].key ? 1 : 0;
            }
#pragma unroll
            for (int e = 0; e < E; e++) {
                if ((eqm[e] >> lane) & 1u) {
                    const uint32_t slot = below + base_m + __popc(eqm[e] & lt);
                    sa[start + slot] = v[e].pos;
                    if (slot > 0) head[start + slot] = slot == below ? 1 : 0;
                }
                base_m += __popc(eqm[e]);
            }
            __syncwarp();  // s_other is reused by the warp's next group
            continue;
        }
        warp_bitonic<E>(v, lane, less);
        const uint64_t prev_lane_last = __shfl_up_sync(0xffffffffu, v[E - 1].key, 1);
#pragma unroll
        for (int e = 0; e < E; e++) {
            const uint32_t i = lane * E + e;
            if (i < size) {
                sa[start + i] = v[e].pos;
                if (i > 0)  // the group's first element keeps its head flag
                    head[start + i] = v[e].key != (e ? v[e - 1].key : prev_lane_last) ? 1 : 0;
            }
        }
    }
}

// ---- cover-rank tie break -----------------------------------------------------
// Shared memory: the X*X comparator table and next_rank once per CTA, then per
// warp the D cover ranks and the position of every slot of the group.
template <int D, int E>
__host__ __device__ constexpr size_t tie_warpsort_warp_bytes() {
    return ((size_t)32 * E * (4 * D + 4) + 15) & ~(size_t)15;
}
template <int D, int E>
inline size_t tie_warpsort_smem(uint32_t X) {
    return tie_tab_smem(X) + WSORT_WARPS * tie_warpsort_warp_bytes<D, E>();
}

// Groups of up to 32*E elements with equal L-char windows, ordered by the
// difference-cover comparator (as k_tie_cta).  A lane sorts (rank offset,
// residue) pairs; a comparison reads the comparator entry of the two residues
// and the two cover ranks it names from shared memory.  Slots past the group
// hold residue 0 and ranks 0xffffffff, above every rank (ranks are below 2^31),
// so they sort last without a test of their own.
template <int D, int E>
__global__ __launch_bounds__(32 * WSORT_WARPS, 2) void k_tie_warpsort(
    const uint32_t* __restrict__ gstart, const uint32_t* __restrict__ gsize, uint64_t ngroups,
    uint32_t* __restrict__ sa, const uint32_t* __restrict__ rank_text, const DcDev* __restrict__ dcp, TieSeg ts) {
    constexpr int N = 32 * E;
    // rank loads in flight per lane: a batch of elements whose D words fit 32 registers
    constexpr int BATCH = E * D <= 32 ? E : (32 / D > 0 ? 32 / D : 1);
    uint16_t* tab;
    uint32_t* nr;
    const uint32_t X = dcp->X;
    tie_tab_ptrs(X, tab, nr);
    load_dc_smem(*dcp, tab, nr);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t* wbase = reinterpret_cast<uint8_t*>(tab) + tie_tab_smem(X) + warp * tie_warpsort_warp_bytes<D, E>();
    uint32_t* s_rk = reinterpret_cast<uint32_t*>(wbase);  // [N * D]
    uint32_t* s_pos = s_rk + N * D;                       // [N]
    const uint64_t nwarps = (uint64_t)gridDim.x * WSORT_WARPS;
    for (uint64_t g = (uint64_t)blockIdx.x * WSORT_WARPS + warp; g < ngroups; g += nwarps) {
        const uint32_t start = gstart[g], size = gsize[g];
        uint64_t pos0, slot0;
        tie_bases(ts, start, pos0, slot0);
        // lane l loads slots e*32 + l (coalesced); those are its starting elements
        uint32_t p[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
            const uint32_t i = e * 32 + lane;
            p[e] = i < size ? (uint32_t)(sa[start + i] - pos0) : INVALID_POS;
        }
        SlotRes v[E];
#pragma unroll
        for (int e0 = 0; e0 < E; e0 += BATCH) {
            uint32_t rk[BATCH][D];
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                const int e = e0 + b;
                if (e >= E) break;
                const uint32_t i = e * 32 + lane;
                uint32_t q = 0, r = 0;
                if (p[e] != INVALID_POS) fdivmod(p[e], dcp->fx, q, r);
                v[e] = SlotRes{i * D, r};
                s_pos[i] = p[e];
                const uint32_t* src = rank_text + slot0 + (uint64_t)q * D + nr[r];
#pragma unroll
                for (int k = 0; k < D; k++) rk[b][k] = p[e] != INVALID_POS ? __ldg(src + k) : 0xffffffffu;
            }
#pragma unroll
            for (int b = 0; b < BATCH; b++) {
                const int e = e0 + b;
                if (e >= E) break;
                const uint32_t i = e * 32 + lane;
#pragma unroll
                for (int k = 0; k < D; k++) s_rk[i * D + k] = rk[b][k];
            }
        }
        __syncwarp();
        warp_bitonic<E>(v, lane, [&](const SlotRes& x, const SlotRes& y) {
            const uint32_t t = tab[x.res * X + y.res];
            return s_rk[x.rk + (t & 0xffu)] < s_rk[y.rk + (t >> 8)];
        });
#pragma unroll
        for (int e = 0; e < E; e++) {
            const uint32_t i = lane * E + e;
            if (i < size) sa[start + i] = (uint32_t)(s_pos[v[e].rk / D] + pos0);
        }
        __syncwarp();  // the slice is reused by the warp's next group
    }
}

}  // namespace dcx
