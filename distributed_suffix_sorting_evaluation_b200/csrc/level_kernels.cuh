// Per-level kernels of the DCX pipeline other than the sorts: alphabet remap,
// head flags, the scan operators of naming / compaction / group detection, the
// recursion string in (mod X, div X) order with discarding, SA emission and the
// suffix-array checker.
//
// A level holds K >= 1 texts back to back (text s occupies [start[s],
// start[s+1]-1) and is followed by one 0 which is its empty suffix).  Every
// position-dependent rule of the reference -- which positions are samples, the
// dummy sample, samples_before, the rank slot (i/X)*D + NEXT_RANK[i%X] -- is
// applied per text with local positions; K = 1 is the single-text build.
#pragma once

#include "common.cuh"
#include "segsort.cuh"

namespace dcx {

struct DcFlags {
    uint32_t X, D;
    FastDiv fx;  // division by X
    uint8_t in_dc[MAX_X];
    uint32_t next_rank[MAX_X];
    uint32_t dc[MAX_D];
};

// Recursion modes per text.
enum : uint8_t { REC_NONE = 0, REC_DIRECT = 1, REC_DISCARD = 2 };

// Per-level segment tables (device arrays).
struct LevelSeg {
    uint32_t K;
    const uint64_t* start;  // [K+1] first position of text s; start[K] = N
    const uint64_t* rbase;  // [K+1] first sample slot of text s (texts are padded by D zero slots)
    const uint64_t* qbase;  // [K+1] first position of text s in the (mod X, div X) string
    const uint64_t* sb;     // [K*(D+1)] samples_before of text s (pdcx.hpp:503-508)
    const uint64_t* obase;  // [K+1] first output slot of text s (sum of text lengths)
    const uint8_t* mode;    // [K] recursion mode
    const uint64_t* kbase;  // [K+1] first kept index of text s (scan of keep flags)
    const uint64_t* start2; // [K] first position of text s in the recursion input
};

__device__ __forceinline__ uint32_t bsearch_le(const uint64_t* a, uint32_t K, uint64_t v) {
    uint32_t lo = 0, hi = K;  // largest s < K with a[s] <= v
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= v) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint64_t slot_of_local(uint64_t i, const DcFlags& f) {
    uint32_t q, r;
    fdivmod((uint32_t)i, f.fx, q, r);  // positions are < 2^32
    return (uint64_t)q * f.D + f.next_rank[r];
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

// byte b -> b + 1 in 32-bit chars (all 256 byte values present)
__global__ void k_widen_text(const uint8_t* __restrict__ in, uint64_t n, uint32_t* __restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)in[i] + 1u;
}

// Batch layout: text k of a group (src_off[k] in the round input, length
// goff[k+1] - goff[k]) moves to goff[k] + k of the level buffer, leaving one 0
// after every text.  Texts are cut into chunks of TEXT_CHUNK chars (at least
// one per text, so empty texts still get their 0): text k owns chunks
// [cbase[k], cbase[k+1]), and a thread block handles one chunk at a time, so
// one long text does not serialise the launch.  `widen` maps byte b to the
// 32-bit char b + 1, otherwise the round's alphabet map applies.
constexpr uint32_t TEXT_CHUNK = 16384;

__device__ __forceinline__ uint32_t chunk_text(const uint64_t* cbase, uint32_t K, uint64_t chunk) {
    uint32_t lo = 0, hi = K;  // largest k with cbase[k] <= chunk
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (cbase[mid] <= chunk) lo = mid; else hi = mid;
    }
    return lo;
}

template <typename CharT>
__global__ void k_spread_texts(const uint8_t* __restrict__ in, const uint64_t* __restrict__ src_off,
                               const uint64_t* __restrict__ goff, const uint64_t* __restrict__ cbase, uint32_t K,
                               uint64_t chunks, CharT* __restrict__ out, const ByteMap* __restrict__ map,
                               bool widen) {
    __shared__ uint8_t m[256];
    if (!widen)
        for (int i = threadIdx.x; i < 256; i += blockDim.x) m[i] = map->m[i];
    __syncthreads();
    for (uint64_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        const uint32_t k = chunk_text(cbase, K, c);
        const uint64_t len = goff[k + 1] - goff[k];
        const uint64_t lo = (c - cbase[k]) * TEXT_CHUNK;
        const uint64_t hi = lo + TEXT_CHUNK < len ? lo + TEXT_CHUNK : len;
        const uint8_t* src = in + src_off[k];
        CharT* o = out + goff[k] + k;
        for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
            o[i] = widen ? (CharT)((uint32_t)src[i] + 1u) : (CharT)m[src[i]];
        if (hi == len && threadIdx.x == 0) o[len] = CharT(0);
    }
}

// ---- head flags --------------------------------------------------------------
struct KeyWords {
    const uint32_t* w[12];
};

// Head flags of a sorted key array of KW words; *ties (zeroed by the caller)
// receives the number of elements equal to their predecessor.  Each thread
// takes 16 consecutive elements: 16-byte loads of every key word (arrays and
// head 16-byte aligned), one more load for the predecessor of the first, and
// one 16-byte store of the 16 flags; the tail past the last full 16 is scalar.
template <int KW>
__global__ __launch_bounds__(256) void k_heads16(KeyWords k, uint64_t N, uint8_t* __restrict__ head,
                                                 unsigned long long* __restrict__ ties) {
    uint32_t t = 0;
    const uint64_t groups = N / 16;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = g * 16;
        uint32_t diff[16];
#pragma unroll
        for (int e = 0; e < 16; e++) diff[e] = 0;
#pragma unroll
        for (int w = 0; w < KW; w++) {
            const uint4* p = reinterpret_cast<const uint4*>(k.w[w] + i0);
            uint32_t v[17];
            v[0] = i0 ? __ldg(k.w[w] + i0 - 1) : ~__ldg(k.w[w]);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint4 x = __ldg(p + q);
                v[1 + 4 * q] = x.x;
                v[2 + 4 * q] = x.y;
                v[3 + 4 * q] = x.z;
                v[4 + 4 * q] = x.w;
            }
#pragma unroll
            for (int e = 0; e < 16; e++) diff[e] |= v[e + 1] ^ v[e];
        }
        uint32_t out[4] = {0, 0, 0, 0};
#pragma unroll
        for (int e = 0; e < 16; e++) {
            const uint32_t h = diff[e] != 0;
            out[e >> 2] |= h << (8 * (e & 3));
            t += h ^ 1u;
        }
        reinterpret_cast<uint4*>(head + i0)[0] = make_uint4(out[0], out[1], out[2], out[3]);
    }
    for (uint64_t i = groups * 16 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t h = 1;
        if (i > 0) {
            h = 0;
#pragma unroll
            for (int w = 0; w < KW; w++) h |= k.w[w][i] != k.w[w][i - 1];
        }
        head[i] = (uint8_t)h;
        t += h ^ 1u;
    }
    t = __reduce_add_sync(0xffffffffu, t);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(ties, (unsigned long long)t);
}

// ---- scan operators (two 32-bit counters packed in a uint64) ------------------
// Tie groups of a partially sorted array: element k is tied when its group
// (run between head flags) has two or more elements.  Emits the tied elements'
// slots, dense group numbers, positions and texts.
struct OpTied {
    const uint8_t* head;
    uint64_t N;
    const uint32_t* sa;
    const uint32_t* segw;  // text of each sorted element, or null for one text
    uint32_t* slot;
    uint32_t* grp;
    uint32_t* tpos;
    uint32_t* tseg;
    __device__ uint64_t load(uint64_t k) const {
        const uint32_t h = head[k];
        const uint32_t nh = (k + 1 < N) ? head[k + 1] : 1u;
        const uint32_t tied = !(h && nh);
        return (uint64_t)h | ((uint64_t)tied << 32);
    }
    __device__ void load16(uint64_t base, uint64_t n, uint64_t* v) const {
        uint32_t b[17];
        load_flags17(head, base, N, 1u, b);
#pragma unroll
        for (int k = 0; k < 16; k++)
            v[k] = base + k < n ? ((uint64_t)b[k] | ((uint64_t)!(b[k] && b[k + 1]) << 32)) : 0ull;
    }
    __device__ void store(uint64_t k, uint64_t ex, uint64_t v) const {
        if (v >> 32) {
            const uint32_t j = (uint32_t)(ex >> 32);
            slot[j] = (uint32_t)k;
            grp[j] = (uint32_t)ex + (uint32_t)v;  // inclusive group number
            tpos[j] = sa[k];
            if (tseg) tseg[j] = segw[k];
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

// Phase 2 step 1: samples in window order with the group number of their window
// (compute_lexicographic_ranks, compute_ranks.hpp:89-111).  A position is a
// sample when its local index mod X is in the cover; the text's empty suffix
// (local index n_s) is then the dummy sample of pdcx.hpp:482-501.
struct OpSamples {
    const uint8_t* head;
    const uint32_t* sa;
    const uint32_t* segw;
    const DcFlags* f;
    LevelSeg ls;
    uint32_t* s_pos;  // local index
    uint32_t* s_seg;
    uint32_t* s_grp;
    uint64_t cap;
    __device__ uint64_t load(uint64_t k) const {
        const uint32_t sg = segw ? segw[k] : 0u;
        const uint64_t i = sa[k] - ls.start[sg];
        uint32_t q, r;
        fdivmod((uint32_t)i, f->fx, q, r);
        const uint32_t smp = f->in_dc[r];
        return (uint64_t)head[k] | ((uint64_t)smp << 32);
    }
    __device__ void load16(uint64_t base, uint64_t n, uint64_t* v) const {
        uint32_t b[17];
        load_flags17(head, base, n, 0u, b);
        uint32_t p[16];
        if (base + 16 <= n) {  // sa (and segw) are 16-byte aligned device arrays
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint4 q4 = __ldg(reinterpret_cast<const uint4*>(sa + base) + k);
                p[4 * k] = q4.x; p[4 * k + 1] = q4.y; p[4 * k + 2] = q4.z; p[4 * k + 3] = q4.w;
            }
            if (segw) {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const uint4 s4 = __ldg(reinterpret_cast<const uint4*>(segw + base) + k);
                    p[4 * k] -= (uint32_t)ls.start[s4.x]; p[4 * k + 1] -= (uint32_t)ls.start[s4.y];
                    p[4 * k + 2] -= (uint32_t)ls.start[s4.z]; p[4 * k + 3] -= (uint32_t)ls.start[s4.w];
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < 16; k++)
                p[k] = base + k < n ? (uint32_t)(sa[base + k] - ls.start[segw ? segw[base + k] : 0u]) : 0u;
        }
        const FastDiv fx = f->fx;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            uint32_t q, r;
            fdivmod(p[k], fx, q, r);
            v[k] = base + k < n ? ((uint64_t)b[k] | ((uint64_t)f->in_dc[r] << 32)) : 0ull;
        }
    }
    __device__ void store(uint64_t k, uint64_t ex, uint64_t v) const {
        if (v >> 32) {
            const uint32_t j = (uint32_t)(ex >> 32);
            if (j >= cap) return;
            const uint32_t sg = segw ? segw[k] : 0u;
            s_pos[j] = (uint32_t)(sa[k] - ls.start[sg]);
            if (s_seg) s_seg[j] = sg;
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

// Sample records in sample text order (slot rbase[s] + (i/X)*D + NEXT_RANK[i%X]
// of sample i of text s): bits [0,32) name, bit 32 unique flag, bits [33,64)
// index j of the sample in window order.  The D padding slots after each text
// keep the all-ones pattern (SREC_EMPTY).  One random 8-byte write per sample;
// every later step of phase 3 reads these records with coalesced passes.
constexpr uint64_t SREC_EMPTY = ~0ull;
__device__ __forceinline__ uint32_t srec_name(uint64_t r) { return (uint32_t)r; }
__device__ __forceinline__ uint32_t srec_uniq(uint64_t r) { return (uint32_t)(r >> 32) & 1u; }
__device__ __forceinline__ uint32_t srec_j(uint64_t r) { return (uint32_t)(r >> 33); }

__global__ void k_scatter_samples(uint64_t m, const uint32_t* __restrict__ s_pos, const uint32_t* __restrict__ s_seg,
                                  const uint32_t* __restrict__ name, const uint8_t* __restrict__ uniq,
                                  const DcFlags* __restrict__ f, LevelSeg ls, uint64_t* __restrict__ srec) {
    const DcFlags& F = *f;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = ls.rbase[s_seg ? s_seg[j] : 0u] + slot_of_local(s_pos[j], F);
        srec[k] = (uint64_t)name[j] | ((uint64_t)uniq[j] << 32) | ((uint64_t)j << 33);
    }
}

// The same records in two steps for large levels, so that no store is a lone
// 8-byte write into a 32-byte sector: k_sample_records lays each sample out as
// (slot, name, unique | j << 1) and histograms the top 8 bits of the slot
// ((slot >> shift) & 255); one radix pass on that digit groups the samples into
// 256 contiguous slot ranges; then
// k_scatter_records stores them in that order, so the stores of concurrent
// CTAs land in a few megabytes that L2 fills completely before writing back.
__global__ void k_sample_records(uint64_t m, const uint32_t* __restrict__ s_pos, const uint32_t* __restrict__ s_seg,
                                 const uint32_t* __restrict__ name, const uint8_t* __restrict__ uniq,
                                 const DcFlags* __restrict__ f, LevelSeg ls, uint32_t* __restrict__ slot_out,
                                 uint32_t* __restrict__ name_out, uint32_t* __restrict__ hi_out,
                                 uint32_t* __restrict__ hist, uint32_t shift) {
    __shared__ uint32_t h[RADIX];
    for (int i = threadIdx.x; i < RADIX; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const DcFlags& F = *f;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = (uint32_t)(ls.rbase[s_seg ? s_seg[j] : 0u] + slot_of_local(s_pos[j], F));
        slot_out[j] = k;
        name_out[j] = name[j];
        hi_out[j] = (uint32_t)uniq[j] | ((uint32_t)j << 1);
        atomicAdd(&h[(k >> shift) & (RADIX - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < RADIX; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

__global__ void k_scatter_records(uint64_t m, const uint32_t* __restrict__ slot, const uint32_t* __restrict__ lo,
                                  const uint32_t* __restrict__ hi, uint64_t* __restrict__ srec) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x)
        srec[slot[j]] = (uint64_t)lo[j] | ((uint64_t)hi[j] << 32);
}

// Distinct names: the rank of every sample is its name (padding slots stay 0).
__global__ void k_ranks_from_names(uint64_t slots, const uint64_t* __restrict__ srec, uint32_t* __restrict__ rank_text,
                                   uint32_t* trace_names, uint8_t* trace_uniq) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < slots; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = srec[k];
        if (r == SREC_EMPTY) continue;
        if (rank_text) rank_text[k] = srec_name(r);
        if (trace_names) {
            trace_names[k] = srec_name(r);
            trace_uniq[k] = (uint8_t)srec_uniq(r);
        }
    }
}

// Recursion string in (mod X, div X) order per text (DCRankIndex::cmp_mod_div,
// compute_ranks.hpp:49-56): position qbase[s] + samples_before_s[c] + b holds
// the name of the text's sample slot b*D + c.  rec_flag bit 0 = unique, bit 1 =
// first element of its text's string.  The kernel walks the sample slots in
// order (empty slots, past the last sample of their class, are skipped): the
// records are read once, front to back, and the writes form D sequential
// streams, where walking the string positions would read every record sector
// once per class.  It is launched with one slot per thread, so the blocks in
// flight fill the streams' sectors together.
__global__ void k_rec_from_slots(uint64_t slots, const uint64_t* __restrict__ srec, const DcFlags* __restrict__ f,
                                 LevelSeg ls, uint32_t* __restrict__ rec, uint8_t* __restrict__ rec_flag) {
    const uint32_t D = f->D;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < slots; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = srec[k];
        if (r == SREC_EMPTY) continue;
        const uint32_t s = ls.K > 1 ? bsearch_le(ls.rbase, ls.K, k) : 0u;
        const uint64_t kl = k - ls.rbase[s];
        const uint64_t b = kl / D;
        const uint32_t c = (uint32_t)(kl - b * D);
        const uint64_t q = ls.qbase[s] + ls.sb[(uint64_t)s * (D + 1) + c] + b;
        rec[q] = srec_name(r);
        rec_flag[q] = (uint8_t)(srec_uniq(r) | (kl == 0 ? 2u : 0u));
    }
}

// Discarding rule (num_ranks_after_discarding, pdcx.hpp:215-228): keep q unless it
// and its predecessor in the same text's string are both unique; the first
// element of each text's string is always kept.
__device__ __forceinline__ uint32_t discard_keep(const uint8_t* rec_flag, uint64_t q) {
    const uint32_t fl = rec_flag[q];
    if (fl & 2u) return 1u;
    return !((fl & 1u) && (rec_flag[q - 1] & 1u));
}

// Counting pass: exclusive prefix of the discarding rule over all texts.
struct OpKeepCount {
    const uint8_t* rec_flag;
    uint32_t* kidx;
    __device__ uint32_t load(uint64_t q) const { return discard_keep(rec_flag, q); }
    __device__ void store(uint64_t q, uint32_t ex, uint32_t) const { kidx[q] = ex; }
};

// Compaction into the recursion input: per text, nothing (names distinct), all
// (direct recursion) or the discarding rule.  Text s's kept elements land at
// start2[s] + (kept index - kbase[s]); separators stay 0 (buffer zeroed).
struct OpCompact {
    const uint8_t* rec_flag;
    const uint32_t* rec;
    LevelSeg ls;
    uint32_t* rec2;
    uint32_t* kidx;
    __device__ uint32_t load(uint64_t q) const {
        const uint32_t s = ls.K > 1 ? bsearch_le(ls.qbase, ls.K, q) : 0u;
        const uint8_t md = ls.mode[s];
        if (md == REC_NONE) return 0u;
        if (md == REC_DIRECT) return 1u;
        return discard_keep(rec_flag, q);
    }
    __device__ void store(uint64_t q, uint32_t ex, uint32_t v) const {
        if (!v) return;
        const uint32_t s = ls.K > 1 ? bsearch_le(ls.qbase, ls.K, q) : 0u;
        rec2[ls.start2[s] + (ex - ls.kbase[s])] = rec[q];
        kidx[q] = ex;
    }
};

// OpCompact for a single text (K = 1) without a scan: a direct text keeps every
// position q (kept index q), a discarding text the positions the discarding
// rule keeps, whose kept indices the keep-count scan (OpKeepCount) already
// wrote to kidx.
__global__ void k_compact_one(uint64_t m, const uint8_t* __restrict__ rec_flag, const uint32_t* __restrict__ rec,
                              uint8_t mode, uint64_t start2, uint32_t* __restrict__ rec2,
                              uint32_t* __restrict__ kidx) {
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < m; q += (uint64_t)gridDim.x * blockDim.x) {
        if (mode == REC_DIRECT) {
            rec2[start2 + q] = rec[q];
            kidx[q] = (uint32_t)q;
        } else if (mode == REC_DISCARD && discard_keep(rec_flag, q)) {
            rec2[start2 + kidx[q]] = rec[q];
        }
    }
}

// Results of the recursive call.  sa2 holds, for each recursing text r (in
// order), the suffix array of its reduced string at o2[r].  Direct texts: the
// sample at string position q gets rank k + 1 (pdcx.hpp:183-212, map_back 83-94).
// Discarding texts: rank_of[kept index] = k + 1 (pdcx.hpp:264-291).
__global__ void k_after_recursion(uint64_t total2, const uint32_t* __restrict__ sa2, const uint64_t* __restrict__ o2,
                                  uint32_t R, const uint32_t* __restrict__ rec_text, const DcFlags* __restrict__ f,
                                  LevelSeg ls, uint32_t* __restrict__ rank_text, uint32_t* __restrict__ rank_of) {
    const uint32_t D = f->D;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total2;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = R > 1 ? bsearch_le(o2, R, x) : 0u;
        const uint32_t s = rec_text[r];
        const uint64_t k = x - o2[r];
        const uint64_t ql = sa2[x];
        if (ls.mode[s] == REC_DIRECT) {
            const uint64_t* sb = ls.sb + (uint64_t)s * (D + 1);
            uint32_t c = 0;
            while (c + 1 < D && ql >= sb[c + 1]) c++;
            rank_text[ls.rbase[s] + (ql - sb[c]) * D + c] = (uint32_t)(k + 1);
        } else {
            rank_of[ls.kbase[s] + ql] = (uint32_t)(k + 1);
        }
    }
}

// Two-step form of k_after_recursion for large levels (the same idea as
// k_sample_records): every rank store becomes a record (destination, rank |
// target << 31), target 1 = rank_of, and the top 8 bits of the destination are
// histogrammed; one radix pass on that digit groups the records into 256
// contiguous destination ranges, and k_scatter_ranks stores them in that order.  Ranks are
// below 2^31 (a level has fewer than 2^31 samples), so bit 31 is free.
// dst_out may be sa2 itself (each element is read, then overwritten, by one thread).
__global__ void k_after_records(uint64_t total2, const uint32_t* sa2, const uint64_t* __restrict__ o2,
                                uint32_t R, const uint32_t* __restrict__ rec_text, const DcFlags* __restrict__ f,
                                LevelSeg ls, uint32_t* dst_out, uint32_t* __restrict__ val_out,
                                uint32_t* __restrict__ hist, uint32_t shift) {
    __shared__ uint32_t h[RADIX];
    for (int i = threadIdx.x; i < RADIX; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint32_t D = f->D;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total2;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = R > 1 ? bsearch_le(o2, R, x) : 0u;
        const uint32_t s = rec_text[r];
        const uint64_t k = x - o2[r];
        const uint64_t ql = sa2[x];
        uint32_t dst, v = (uint32_t)(k + 1);
        if (ls.mode[s] == REC_DIRECT) {
            const uint64_t* sb = ls.sb + (uint64_t)s * (D + 1);
            uint32_t c = 0;
            while (c + 1 < D && ql >= sb[c + 1]) c++;
            dst = (uint32_t)(ls.rbase[s] + (ql - sb[c]) * D + c);
        } else {
            dst = (uint32_t)(ls.kbase[s] + ql);
            v |= 0x80000000u;
        }
        dst_out[x] = dst;
        val_out[x] = v;
        atomicAdd(&h[(dst >> shift) & (RADIX - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < RADIX; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

__global__ void k_scatter_ranks(uint64_t n, const uint32_t* __restrict__ dst, const uint32_t* __restrict__ val,
                                uint32_t* __restrict__ rank_text, uint32_t* __restrict__ rank_of) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = val[j];
        if (v >> 31) rank_of[dst[j]] = v & 0x7fffffffu;
        else rank_text[dst[j]] = v;
    }
}

// Non-unique samples of discarding texts keyed by (name, rank of their position
// in the reduced string); value = sample slot (pdcx.hpp:296-346).
struct OpNonUniqueSeg {
    const uint64_t* srec;
    const DcFlags* f;
    LevelSeg ls;
    const uint32_t* kidx;
    const uint32_t* rank_of;
    uint32_t* key_lo;
    uint32_t* key_hi;
    uint32_t* val;
    __device__ uint32_t load(uint64_t k) const {
        const uint64_t r = srec[k];
        if (r == SREC_EMPTY || srec_uniq(r)) return 0u;
        const uint32_t s = ls.K > 1 ? bsearch_le(ls.rbase, ls.K, k) : 0u;
        return ls.mode[s] == REC_DISCARD;
    }
    __device__ void store(uint64_t k, uint32_t ex, uint32_t v) const {
        if (!v || !key_lo) return;  // null outputs: counting pass only
        const uint32_t s = ls.K > 1 ? bsearch_le(ls.rbase, ls.K, k) : 0u;
        const uint64_t kl = k - ls.rbase[s];
        const uint64_t q = ls.qbase[s] + ls.sb[(uint64_t)s * (f->D + 1) + kl % f->D] + kl / f->D;
        key_lo[ex] = rank_of[kidx[q]];
        key_hi[ex] = srec_name(srec[k]);
        val[ex] = (uint32_t)k;
    }
};

__global__ void k_name_starts(uint64_t m, const uint32_t* __restrict__ name, uint32_t* __restrict__ start_of) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x)
        if (j == 0 || name[j] != name[j - 1]) start_of[name[j]] = (uint32_t)j;
}

__global__ void k_ranks_nonunique(uint64_t mu, const uint32_t* __restrict__ key_hi, const uint32_t* __restrict__ val,
                                  const uint32_t* __restrict__ start_s, const uint32_t* __restrict__ start_l,
                                  uint32_t* __restrict__ rank_text) {
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < mu; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t nm = key_hi[t];
        rank_text[val[t]] = start_s[nm] + (uint32_t)(t - start_l[nm]) + 1;
    }
}

// Ranks that need no recursion result: texts with distinct names keep their
// names; unique samples of discarding texts keep their window order (j + 1).
__global__ void k_ranks_rest(uint64_t slots, const uint64_t* __restrict__ srec, LevelSeg ls,
                             uint32_t* __restrict__ rank_text) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < slots; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = srec[k];
        if (r == SREC_EMPTY) continue;
        const uint32_t s = ls.K > 1 ? bsearch_le(ls.rbase, ls.K, k) : 0u;
        const uint8_t md = ls.mode[s];
        if (md == REC_NONE) rank_text[k] = srec_name(r);
        else if (md == REC_DISCARD && srec_uniq(r)) rank_text[k] = srec_j(r) + 1;
    }
}

// out[i] = src[idx[i]] (idx[i] == total_idx reads total_val instead)
__global__ void k_gather_u32(const uint32_t* __restrict__ src, const uint64_t* __restrict__ idx, uint32_t count,
                             uint64_t total_idx, uint32_t total_val, uint32_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        out[i] = idx[i] < total_idx ? src[idx[i]] : total_val;
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
    __device__ void load16(uint64_t base, uint64_t n, uint64_t* v) const {
        uint32_t b[17];
        load_flags17(head, base, N, 1u, b);
#pragma unroll
        for (int k = 0; k < 16; k++)
            v[k] = base + k < n ? ((uint64_t)(b[k] && !b[k + 1]) | ((uint64_t)(!b[k] && b[k + 1]) << 32)) : 0ull;
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

// Tie groups (runs of two or more equal windows) inside parent groups that
// hold every tie: one thread per parent group walks its head flags twice
// (count, then emit); the runs are appended as (start, end) in any order, one
// atomic reservation per warp.  Every lane runs the same number of rounds.
__global__ void k_subgroups(uint64_t Gp, const uint32_t* __restrict__ pstart, const uint32_t* __restrict__ psize,
                            const uint8_t* __restrict__ head, uint32_t* __restrict__ out_start,
                            uint32_t* __restrict__ out_end, uint32_t* __restrict__ count) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t first = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t rounds = (Gp + stride - 1) / stride;
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t r = 0; r < rounds; r++) {
        const uint64_t g = first + r * stride;
        uint32_t st = 0, sz = 0, nsub = 0;
        if (g < Gp) {
            st = pstart[g];
            sz = psize[g];
            uint32_t run = 1;
            for (uint32_t k = 1; k < sz; k++) {
                if (head[st + k]) {
                    nsub += run > 1;
                    run = 1;
                } else {
                    run++;
                }
            }
            nsub += run > 1;
        }
        uint32_t incl = nsub;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        uint32_t base = 0;
        if (lane == 31 && total) base = atomicAdd(count, total);
        base = __shfl_sync(0xffffffffu, base, 31) + incl - nsub;
        if (nsub) {
            uint32_t a = st;
            for (uint32_t k = 1; k <= sz; k++) {
                if (k == sz || head[st + k]) {
                    if (st + k - 1 > a) {
                        out_start[base] = a;
                        out_end[base] = st + k - 1;
                        base++;
                    }
                    a = st + k;
                }
            }
        }
    }
}

// Tie groups of a whole head-flag array (flags 16-byte aligned) without a scan:
// thread t reads flags [16t, 16t + 16) with one 16-byte load plus the flag after
// them, finds the group starts among them (a flag 1 followed by a 0; position N
// counts as a 1), and walks each group to its end: inside its own 16 flags from
// registers, past them byte by byte, at most `limit` flags.  A longer group
// sets *overflow (its entry is then incomplete and the caller scans instead).
// Groups are appended as (start, end) in any order, one atomic reservation per
// warp; every lane runs the same number of rounds.
__global__ void k_groups_walk(uint64_t N, const uint8_t* __restrict__ head, uint32_t limit,
                              uint32_t* __restrict__ out_start, uint32_t* __restrict__ out_end,
                              uint32_t* __restrict__ count, uint32_t* __restrict__ overflow) {
    const uint64_t blocks = (N + 15) / 16;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t first = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t rounds = (blocks + stride - 1) / stride;
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t r = 0; r < rounds; r++) {
        const uint64_t t = first + r * stride;
        const uint64_t i0 = t * 16;
        uint32_t f = 0;  // bit k: flag of i0 + k (k = 0..16); positions >= N count as 1
        if (t < blocks) {
            if (i0 + 16 <= N) {
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(head + i0));
                const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int q = 0; q < 4; q++)
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        if ((w[q] >> (8 * b)) & 0xffu) f |= 1u << (4 * q + b);
            } else {
                for (uint32_t k = 0; k < 16; k++) f |= (i0 + k >= N || head[i0 + k]) ? 1u << k : 0u;
            }
            f |= (i0 + 16 >= N || head[i0 + 16]) ? 1u << 16 : 0u;
        }
        // starts: flag 1 at k, flag 0 at k + 1 (k = 0..15)
        const uint32_t st = t < blocks ? (f & ~(f >> 1)) & 0xffffu : 0u;
        const uint32_t nsub = __popc(st);
        uint32_t incl = nsub;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += x;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        uint32_t base = 0;
        if (lane == 31 && total) base = atomicAdd(count, total);
        base = __shfl_sync(0xffffffffu, base, 31) + incl - nsub;
        uint32_t s = st;
        while (s) {
            const uint32_t k = __ffs(s) - 1;
            s &= s - 1;
            // the group runs from i0 + k to the position before the next flag 1
            const uint32_t later = (f >> (k + 1)) & 0x1ffffu;  // flags of i0 + k + 1 .. i0 + 16
            uint64_t end;
            if (later) {
                end = i0 + k + __ffs(later) - 1;  // next 1 within the 17 flags
            } else {
                uint64_t p = i0 + 17;
                const uint64_t stop = i0 + k + 1 + (uint64_t)limit;
                while (p < N && p < stop && !head[p]) p++;
                if (p < N && p >= stop) atomicOr(overflow, 1u);
                end = p - 1;
            }
            out_start[base] = (uint32_t)(i0 + k);
            out_end[base] = (uint32_t)end;
            base++;
        }
    }
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
// One text: sa_full slot 0 is position n (the empty suffix); the n remaining
// slots are written in 32-, 40- (little endian, high byte 0 since indices are
// < 2^32) or 64-bit form.  Four entries per thread so the 40-bit form is
// written as five aligned 32-bit words.
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


// 40-bit output through shared memory: each thread packs four entries into
// five words (conflict-free: thread t writes words 5t..5t+4), then the CTA
// writes its 1024 entries (5120 bytes) with coalesced 16-byte stores.  The
// output must be 16-byte aligned; entries past the last full tile are written
// by k_emit's byte path (`tail_from` = first entry not written here).
constexpr uint32_t EMIT40_TILE = 1024;
__global__ __launch_bounds__(256) void k_emit40(const uint32_t* __restrict__ sa_full, uint64_t n,
                                                uint8_t* __restrict__ out) {
    __shared__ __align__(16) uint32_t sw[EMIT40_TILE * 5 / 4];
    const uint64_t tiles = n / EMIT40_TILE;
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t k0 = t * EMIT40_TILE + 4 * threadIdx.x;
        const uint32_t e0 = sa_full[k0 + 1], e1 = sa_full[k0 + 2], e2 = sa_full[k0 + 3], e3 = sa_full[k0 + 4];
        uint32_t* o = sw + 5 * threadIdx.x;
        o[0] = e0;
        o[1] = e1 << 8;
        o[2] = (e1 >> 24) | (e2 << 16);
        o[3] = (e2 >> 16) | (e3 << 24);
        o[4] = e3 >> 8;
        __syncthreads();
        uint4* dst = reinterpret_cast<uint4*>(out + t * EMIT40_TILE * 5);
        const uint4* src = reinterpret_cast<const uint4*>(sw);
        for (uint32_t q = threadIdx.x; q < EMIT40_TILE * 5 / 16; q += blockDim.x) dst[q] = src[q];
        __syncthreads();
    }
}

// Several texts: sorted element k belongs to text s = segw[k]; text s's elements
// occupy sorted slots [start[s], start[s+1]) with its empty suffix first, so
// slot start[s] + 1 + r holds the text's r-th suffix; indices are text-local.
__global__ void k_emit_seg(const uint32_t* __restrict__ sa_full, const uint32_t* __restrict__ segw, uint64_t N,
                           LevelSeg ls, void* __restrict__ out, int width) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < N; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = segw ? segw[k] : 0u;  // no segw: a single text
        const uint64_t r = k - ls.start[s];
        if (r == 0) continue;
        store_sa_entry(out, ls.obase[s] + r - 1, (uint32_t)(sa_full[k] - ls.start[s]), width);
    }
}

// ---- suffix-array checker (the conditions of check_suffixarray,
// lightweight_dcx/src/sa_check.hpp:56-184, without its sorts) ------------------
__device__ __forceinline__ uint64_t load_sa_entry(const void* sa, uint64_t k, int width) {
    if (width == 32) return reinterpret_cast<const uint32_t*>(sa)[k];
    if (width == 64) return reinterpret_cast<const uint64_t*>(sa)[k];
    const uint8_t* b = reinterpret_cast<const uint8_t*>(sa) + 5 * k;
    return (uint64_t)b[0] | ((uint64_t)b[1] << 8) | ((uint64_t)b[2] << 16) | ((uint64_t)b[3] << 24) |
           ((uint64_t)b[4] << 32);
}

// Permutation: every position occurs once; isa[p] = 1 + rank of suffix p.
__global__ void k_check_isa(const void* __restrict__ sa, int width, uint64_t n, uint32_t* __restrict__ isa,
                            unsigned long long* __restrict__ bad) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p = load_sa_entry(sa, k, width);
        if (p >= n) {
            atomicAdd(bad, 1ull);
            continue;
        }
        if (atomicExch(&isa[p], (uint32_t)(k + 1)) != 0u) atomicAdd(bad, 1ull);
    }
}

// Order: for adjacent SA entries i, j: (T[i], isa[i+1]) < (T[j], isa[j+1]) with
// isa[n] = 0 (the empty suffix is smallest).
__global__ void k_check_order(const void* __restrict__ sa, int width, uint64_t n, const uint8_t* __restrict__ t,
                              const uint32_t* __restrict__ isa, unsigned long long* __restrict__ bad) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; k < n;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = load_sa_entry(sa, k - 1, width), j = load_sa_entry(sa, k, width);
        if (i >= n || j >= n) continue;  // reported by k_check_isa
        const uint32_t ti = t[i], tj = t[j];
        bool ok = ti < tj;
        if (ti == tj) {
            const uint32_t ri = i + 1 < n ? isa[i + 1] : 0u, rj = j + 1 < n ? isa[j + 1] : 0u;
            ok = ri < rj;
        }
        if (!ok) atomicAdd(bad, 1ull);
    }
}

}  // namespace dcx
