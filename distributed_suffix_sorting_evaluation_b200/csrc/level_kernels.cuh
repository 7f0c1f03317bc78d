// Per-level kernels of the DCX pipeline other than the sorts: alphabet remap,
// head flags, the scan operators of naming / compaction / group detection, the
// recursion string in (mod X, div X) order with discarding, and SA emission.
#pragma once

#include "common.cuh"
#include "segsort.cuh"

namespace dcx {

struct DcFlags {
    uint32_t X, D;
    uint8_t in_dc[MAX_X];
    uint32_t next_rank[MAX_X];
    uint32_t dc[MAX_D];
    uint64_t samples_before[MAX_D + 1];
};

__device__ __forceinline__ uint64_t rank_pos_of(uint32_t pos, const DcFlags& f) {
    return (uint64_t)(pos / f.X) * f.D + f.next_rank[pos % f.X];
}

// ---- alphabet (cli.cpp:417-463) ---------------------------------------------
__global__ void k_hist256(const uint8_t* __restrict__ t, uint64_t n, unsigned long long* __restrict__ hist) {
    __shared__ uint32_t h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint64_t n16 = n / 16;
    const uint4* t16 = reinterpret_cast<const uint4*>(t);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x) {
        uint4 v = __ldg(t16 + i);
        uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int b = 0; b < 4; b++) atomicAdd(&h[(w[k] >> (8 * b)) & 255u], 1u);
    }
    for (uint64_t i = n16 * 16 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&h[t[i]], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

struct ByteMap {
    uint8_t m[256];
};

__global__ void k_remap(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, uint64_t n, ByteMap map) {
    __shared__ uint8_t m[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) m[i] = map.m[i];
    __syncthreads();
    const uint64_t n16 = n / 16;
    const uint4* in16 = reinterpret_cast<const uint4*>(in);
    uint4* out16 = reinterpret_cast<uint4*>(out);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x) {
        uint4 v = __ldg(in16 + i);
        uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            uint32_t x = w[k], y = 0;
#pragma unroll
            for (int b = 0; b < 4; b++) y |= (uint32_t)m[(x >> (8 * b)) & 255u] << (8 * b);
            w[k] = y;
        }
        out16[i] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    for (uint64_t i = n16 * 16 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = m[in[i]];
}

__global__ void k_widen_text(const uint8_t* __restrict__ in, uint64_t n, uint32_t* __restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)in[i] + 1u;
}

// ---- head flags --------------------------------------------------------------
struct KeyWords {
    const uint32_t* w[12];
};

__global__ void k_heads(KeyWords k, uint32_t kw, uint64_t N, uint8_t* __restrict__ head) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
        uint8_t h = 1;
        if (i > 0) {
            h = 0;
            for (uint32_t w = 0; w < kw; w++) h |= k.w[w][i] != k.w[w][i - 1];
        }
        head[i] = h;
    }
}

// ---- scan operators (two 32-bit counters packed in a uint64) ------------------
// Tie groups of a partially sorted array: element k is tied when its group
// (run between head flags) has two or more elements.  Emits the tied elements'
// slots and dense group numbers.
struct OpTied {
    const uint8_t* head;
    uint64_t N;
    const uint32_t* sa;
    uint32_t* slot;
    uint32_t* grp;
    uint32_t* tpos;
    __device__ uint64_t load(uint64_t k) const {
        const uint32_t h = head[k];
        const uint32_t nh = (k + 1 < N) ? head[k + 1] : 1u;
        const uint32_t tied = !(h && nh);
        return (uint64_t)h | ((uint64_t)tied << 32);
    }
    __device__ void store(uint64_t k, uint64_t ex, uint64_t v) const {
        if (v >> 32) {
            const uint32_t j = (uint32_t)(ex >> 32);
            slot[j] = (uint32_t)k;
            grp[j] = (uint32_t)ex + (uint32_t)v;  // inclusive group number
            tpos[j] = sa[k];
        }
    }
};

// After a refinement sort: write the refined order back and recompute heads.
__global__ void k_refine_scatter(uint64_t count, const uint32_t* __restrict__ slot, KeyWords k, uint32_t kw,
                                 const uint32_t* __restrict__ vals, uint32_t* __restrict__ sa,
                                 uint8_t* __restrict__ head) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < count; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = slot[j];
        sa[s] = vals[j];
        uint8_t h = 1;
        if (j > 0) {
            h = 0;
            for (uint32_t w = 0; w < kw; w++) h |= k.w[w][j] != k.w[w][j - 1];
        }
        head[s] = h;
    }
}

// Phase 2 step 1: samples in sorted order with the group number of their window
// (compute_lexicographic_ranks, compute_ranks.hpp:89-111).
struct OpSamples {
    const uint8_t* head;
    const uint32_t* sa;
    const DcFlags* f;
    uint32_t* s_pos;
    uint32_t* s_grp;
    uint64_t cap;
    __device__ uint64_t load(uint64_t k) const {
        const uint32_t pos = sa[k];
        const uint32_t smp = f->in_dc[pos % f->X];
        return (uint64_t)head[k] | ((uint64_t)smp << 32);
    }
    __device__ void store(uint64_t k, uint64_t ex, uint64_t v) const {
        if (v >> 32) {
            const uint32_t j = (uint32_t)(ex >> 32);
            if (j >= cap) return;
            s_pos[j] = sa[k];
            s_grp[j] = (uint32_t)ex + (uint32_t)v;
        }
    }
};

// Phase 2 step 2: names = 1 + number of changes before; unique = differs from
// both neighbours (flag_unique_ranks, compute_ranks.hpp:113-134).
struct OpNames {
    const uint32_t* s_grp;
    uint64_t m;
    uint32_t* name;
    uint8_t* uniq;
    __device__ uint32_t load(uint64_t j) const { return j == 0 || s_grp[j] != s_grp[j - 1]; }
    __device__ void store(uint64_t j, uint32_t ex, uint32_t v) const {
        name[j] = ex + v;
        const uint32_t next_changed = (j + 1 == m) || s_grp[j + 1] != s_grp[j];
        uniq[j] = (uint8_t)(v && next_changed);
    }
};

// Sample records in sample text order (slot k = (p/X)*D + NEXT_RANK[p%X] of
// sample p): bits [0,32) name, bit 32 unique flag, bits [33,64) index j of the
// sample in window order.  One random 8-byte write per sample; every later step
// of phase 3 reads these records with coalesced passes.
__device__ __forceinline__ uint32_t srec_name(uint64_t r) { return (uint32_t)r; }
__device__ __forceinline__ uint32_t srec_uniq(uint64_t r) { return (uint32_t)(r >> 32) & 1u; }
__device__ __forceinline__ uint32_t srec_j(uint64_t r) { return (uint32_t)(r >> 33); }

__global__ void k_scatter_samples(uint64_t m, const uint32_t* __restrict__ s_pos, const uint32_t* __restrict__ name,
                                  const uint8_t* __restrict__ uniq, const DcFlags* __restrict__ f,
                                  uint64_t* __restrict__ srec) {
    const DcFlags& F = *f;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = rank_pos_of(s_pos[j], F);
        srec[k] = (uint64_t)name[j] | ((uint64_t)uniq[j] << 32) | ((uint64_t)j << 33);
    }
}

// Distinct names: the rank of every sample is its name.
__global__ void k_ranks_from_names(uint64_t m, const uint64_t* __restrict__ srec, uint32_t* __restrict__ rank_text,
                                   uint32_t* trace_names, uint8_t* trace_uniq) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = srec[k];
        if (rank_text) rank_text[k] = srec_name(r);
        if (trace_names) {
            trace_names[k] = srec_name(r);
            trace_uniq[k] = (uint8_t)srec_uniq(r);
        }
    }
}

// Recursion string in (mod X, div X) order: position q = samples_before[c] + b
// holds the name of sample slot k = b*D + c (a transpose of the D-column layout).
__global__ void k_rec_from_samples(uint64_t m, const uint64_t* __restrict__ srec, const DcFlags* __restrict__ f,
                                   uint32_t* __restrict__ rec, uint8_t* __restrict__ rec_uniq) {
    const DcFlags& F = *f;
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < m; q += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = 0;
        while (c + 1 < F.D && q >= F.samples_before[c + 1]) c++;
        const uint64_t b = q - F.samples_before[c];
        const uint64_t r = srec[b * F.D + c];
        rec[q] = srec_name(r);
        rec_uniq[q] = (uint8_t)srec_uniq(r);
    }
}

// After discarding, unique samples keep their window order: rank = j + 1.
__global__ void k_ranks_unique_text(uint64_t m, const uint64_t* __restrict__ srec, uint32_t* __restrict__ rank_text) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = srec[k];
        if (srec_uniq(r)) rank_text[k] = srec_j(r) + 1;
    }
}

// Non-unique samples (text order) keyed by (name, rank of their position in the
// reduced string); value = sample slot k.
struct OpNonUniqueText {
    const uint64_t* srec;
    const DcFlags* f;
    const uint32_t* kidx;
    const uint32_t* rank_of;
    uint32_t* key_lo;
    uint32_t* key_hi;
    uint32_t* val;
    __device__ uint32_t load(uint64_t k) const { return !srec_uniq(srec[k]); }
    __device__ void store(uint64_t k, uint32_t ex, uint32_t v) const {
        if (v && key_lo) {  // null outputs: counting pass only
            const uint64_t b = k / f->D, c = k % f->D;
            const uint64_t q = f->samples_before[c] + b;
            key_lo[ex] = rank_of[kidx[q]];
            key_hi[ex] = srec_name(srec[k]);
            val[ex] = (uint32_t)k;
        }
    }
};

__global__ void k_ranks_nonunique(uint64_t mu, const uint32_t* __restrict__ key_hi, const uint32_t* __restrict__ val,
                                  const uint32_t* __restrict__ start_s, const uint32_t* __restrict__ start_l,
                                  uint32_t* __restrict__ rank_text) {
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < mu; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t nm = key_hi[t];
        rank_text[val[t]] = start_s[nm] + (uint32_t)(t - start_l[nm]) + 1;
    }
}

// Final SA of a level: sa_full slot 0 is position n (the empty suffix); the
// n remaining slots are written in 32-, 40- (little endian, high byte 0 since
// indices are < 2^32) or 64-bit form.  Four entries per thread so the 40-bit
// form is written as five aligned 32-bit words.
__global__ void k_emit(const uint32_t* __restrict__ sa_full, uint64_t n, void* __restrict__ out, int width) {
    const uint64_t groups = n / 4;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t e0 = sa_full[4 * g + 1], e1 = sa_full[4 * g + 2], e2 = sa_full[4 * g + 3], e3 = sa_full[4 * g + 4];
        if (width == 32) {
            reinterpret_cast<uint4*>(out)[g] = make_uint4(e0, e1, e2, e3);
        } else if (width == 64) {
            ulonglong2* o = reinterpret_cast<ulonglong2*>(out) + 2 * g;
            o[0] = make_ulonglong2(e0, e1);
            o[1] = make_ulonglong2(e2, e3);
        } else {
            uint32_t* o = reinterpret_cast<uint32_t*>(out) + 5 * g;
            o[0] = e0;
            o[1] = e1 << 8;
            o[2] = (e1 >> 24) | (e2 << 16);
            o[3] = (e2 >> 16) | (e3 << 24);
            o[4] = e3 >> 8;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
        const uint64_t k = groups * 4 + threadIdx.x;
        const uint32_t v = sa_full[k + 1];
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
}

// Phase 3 distinct case: ranks = names, scattered to sample text order.
__global__ void k_scatter_names(uint64_t m, const uint32_t* __restrict__ s_pos, const uint32_t* __restrict__ name,
                                const DcFlags* __restrict__ f, uint32_t* __restrict__ rank_text,
                                uint32_t* trace_names, uint8_t* trace_uniq, const uint8_t* uniq) {
    const DcFlags& F = *f;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t rp = rank_pos_of(s_pos[j], F);
        if (rank_text) rank_text[rp] = name[j];
        if (trace_names) {
            trace_names[rp] = name[j];
            trace_uniq[rp] = uniq[j];
        }
    }
}

// Recursion string in (mod X, div X) order (DCRankIndex::cmp_mod_div,
// compute_ranks.hpp:49-56): sample p = b*X + DC[c] goes to samples_before[c] + b.
__global__ void k_build_rec(uint64_t m, const uint32_t* __restrict__ s_pos, const uint32_t* __restrict__ name,
                            const uint8_t* __restrict__ uniq, const DcFlags* __restrict__ f, uint32_t* __restrict__ rec,
                            uint8_t* __restrict__ rec_uniq, uint32_t* __restrict__ q_of_j) {
    const DcFlags& F = *f;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t pos = s_pos[j];
        const uint32_t c = F.next_rank[pos % F.X];
        const uint64_t q = F.samples_before[c] + pos / F.X;
        rec[q] = name[j];
        rec_uniq[q] = uniq[j];
        if (q_of_j) q_of_j[j] = (uint32_t)q;
    }
}

// Direct recursion result: sample at recursion index SA_R[k] has rank k+1
// (recursive_call_direct + map_back, pdcx.hpp:83-94,183-212).
__global__ void k_ranks_from_rec(uint64_t m, const uint32_t* __restrict__ sa_r, const DcFlags* __restrict__ f,
                                 uint32_t* __restrict__ rank_text) {
    const DcFlags& F = *f;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t q = sa_r[k];
        uint32_t c = 0;
        while (c + 1 < F.D && q >= F.samples_before[c + 1]) c++;
        const uint64_t b = q - F.samples_before[c];
        rank_text[b * F.D + c] = (uint32_t)(k + 1);
    }
}

// Discarding (num_ranks_after_discarding / recursive_call_with_discarding,
// pdcx.hpp:215-252): keep element q unless it and its predecessor are unique.
struct OpKeep {
    const uint8_t* rec_uniq;
    const uint32_t* rec;
    uint32_t* rec2;
    uint32_t* kidx;
    __device__ uint32_t load(uint64_t q) const { return q == 0 || !(rec_uniq[q] && rec_uniq[q - 1]); }
    __device__ void store(uint64_t q, uint32_t ex, uint32_t v) const {
        if (rec2 && v) rec2[ex] = rec[q];
        if (kidx) kidx[q] = ex;
    }
};

__global__ void k_inverse(uint64_t m, const uint32_t* __restrict__ sa, uint32_t* __restrict__ inv) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (uint64_t)gridDim.x * blockDim.x)
        inv[sa[k]] = (uint32_t)(k + 1);
}

// Non-unique samples with (name, rank2) keys for the rank recovery after
// discarding (pdcx.hpp:296-346).  rank2 = rank of the sample's position in the
// reduced string.
struct OpNonUnique {
    const uint8_t* uniq;
    const uint32_t* name;
    const uint32_t* q_of_j;
    const uint32_t* kidx;
    const uint32_t* rank_of;
    uint32_t* key_lo;
    uint32_t* key_hi;
    uint32_t* val;
    __device__ uint32_t load(uint64_t j) const { return !uniq[j]; }
    __device__ void store(uint64_t j, uint32_t ex, uint32_t v) const {
        if (v) {
            key_lo[ex] = rank_of[kidx[q_of_j[j]]];
            key_hi[ex] = name[j];
            val[ex] = (uint32_t)j;
        }
    }
};

__global__ void k_name_starts(uint64_t m, const uint32_t* __restrict__ name, uint32_t* __restrict__ start_of) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x)
        if (j == 0 || name[j] != name[j - 1]) start_of[name[j]] = (uint32_t)j;
}

__global__ void k_ranks_after_discarding(uint64_t mu, const uint32_t* __restrict__ key_hi,
                                         const uint32_t* __restrict__ val, const uint32_t* __restrict__ start_s,
                                         const uint32_t* __restrict__ start_l, const uint32_t* __restrict__ s_pos,
                                         const DcFlags* __restrict__ f, uint32_t* __restrict__ rank_text) {
    const DcFlags& F = *f;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < mu; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t nm = key_hi[t];
        const uint32_t j = val[t];
        const uint32_t r = start_s[nm] + (uint32_t)(t - start_l[nm]) + 1;
        rank_text[rank_pos_of(s_pos[j], F)] = r;
    }
}

__global__ void k_ranks_unique(uint64_t m, const uint8_t* __restrict__ uniq, const uint32_t* __restrict__ s_pos,
                               const DcFlags* __restrict__ f, uint32_t* __restrict__ rank_text) {
    const DcFlags& F = *f;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x)
        if (uniq[j]) rank_text[rank_pos_of(s_pos[j], F)] = (uint32_t)(j + 1);
}

// ---- phase 4 tie groups --------------------------------------------------------
struct OpGroups {
    const uint8_t* head;
    uint64_t N;
    uint32_t* starts;
    uint32_t* ends;
    __device__ uint64_t load(uint64_t k) const {
        const uint32_t h = head[k];
        const uint32_t nh = (k + 1 < N) ? head[k + 1] : 1u;
        const uint32_t s = h && !nh;
        const uint32_t e = !h && nh;
        return (uint64_t)s | ((uint64_t)e << 32);
    }
    __device__ void store(uint64_t k, uint64_t ex, uint64_t v) const {
        if (v & 0xffffffffull) starts[(uint32_t)ex] = (uint32_t)k;
        if (v >> 32) ends[(uint32_t)(ex >> 32)] = (uint32_t)k;
    }
};

constexpr int TIE_CLASSES = 12;  // 2,4,8,16,32 (warp) | 64..2048 (CTA) | big
__device__ __forceinline__ int tie_class(uint32_t size) {
    if (size > 2048) return 11;
    int c = 0;
    uint32_t cap = 2;
    while (cap < size) {
        cap <<= 1;
        c++;
    }
    return c;  // size 2 -> 0, <=4 -> 1, ..., <=2048 -> 10
}

__global__ void k_tie_classify(uint64_t G, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ ends,
                               uint32_t* __restrict__ counts) {
    __shared__ uint32_t c[TIE_CLASSES];
    if (threadIdx.x < TIE_CLASSES) c[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G; g += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&c[tie_class(ends[g] - starts[g] + 1)], 1u);
    __syncthreads();
    if (threadIdx.x < TIE_CLASSES && c[threadIdx.x]) atomicAdd(&counts[threadIdx.x], c[threadIdx.x]);
}

// Bins tie groups by size class.  Cursor updates are aggregated per warp: the
// lanes holding the same class elect one lane that reserves their slots.
__global__ void k_tie_bin(uint64_t G, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ ends,
                          uint32_t* __restrict__ cursor, uint32_t* __restrict__ out_start, uint32_t* __restrict__ out_size) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t first = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t rounds = (G + stride - 1) / stride;
    for (uint64_t r = 0; r < rounds; r++) {  // every lane runs the same rounds (warp-wide ballots)
        const uint64_t g = first + r * stride;
        const bool ok = g < G;
        uint32_t sz = 0, cls = 31;
        if (ok) {
            sz = ends[g] - starts[g] + 1;
            cls = (uint32_t)tie_class(sz);
        }
        uint32_t peers = 0xffffffffu;
#pragma unroll
        for (int b = 0; b < 5; b++) {
            const uint32_t bit = (cls >> b) & 1u;
            const uint32_t bal = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? bal : ~bal;
        }
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (ok && lane_id() == leader) base = atomicAdd(&cursor[cls], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (ok) {
            const uint32_t slot = base + __popc(peers & lanemask_lt());
            out_start[slot] = starts[g];
            out_size[slot] = sz;
        }
    }
}

__global__ void k_copy_ranges(const uint64_t* __restrict__ offsets, uint32_t ngroups, const uint32_t* __restrict__ gstart,
                              uint64_t total, const uint32_t* __restrict__ src, uint32_t* __restrict__ dst) {
    for (uint64_t f = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; f < total; f += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = ngroups;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= f) lo = mid; else hi = mid;
        }
        const uint64_t i = (uint64_t)gstart[lo] + (f - offsets[lo]);
        dst[i] = src[i];
    }
}

// ---- SA emission --------------------------------------------------------------
// sa_full holds N = n + 1 slots; slot 0 is position n (the empty suffix).
__global__ void k_emit32(const uint32_t* __restrict__ sa_full, uint64_t n, uint32_t* __restrict__ out) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = sa_full[k + 1];
}

__global__ void k_widen(const uint32_t* __restrict__ sa, uint64_t n, uint8_t* __restrict__ out, int width) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = sa[k];
        if (width == 64) {
            reinterpret_cast<uint64_t*>(out)[k] = v;
        } else {  // 40-bit little endian: low uint32 then high uint8 (util/uint_types.hpp:49-269)
            uint8_t* o = out + 5 * k;
            o[0] = (uint8_t)v;
            o[1] = (uint8_t)(v >> 8);
            o[2] = (uint8_t)(v >> 16);
            o[3] = (uint8_t)(v >> 24);
            o[4] = 0;
        }
    }
}

}  // namespace dcx
