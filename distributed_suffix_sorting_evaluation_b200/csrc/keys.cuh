// Key materialisation for the suffix sorts.
//
// The reference packs the first X*ratio characters of a suffix MSB-first into
// 64-bit words, 3/5/8 bits per char (lightweight_dcx/src/strings/char_container.hpp:50-104,
// 483-545; cli.cpp:488-533) and compares the words lexicographically.  The GPU
// build needs the same order but as a radix-sortable integer with as few bits as
// possible, so a window c_0..c_{P-1} of chars in 0..sigma (0 = padding past the
// end of the text) is encoded as the mixed-radix integer
//     key = sum_j c_j * (sigma+1)^(P-1-j)
// which orders exactly like the packed words (same prefix -> same key; first
// difference decides).  DNA (sigma = 4) needs log2(5) = 2.32 bits per char
// instead of 3.  The integer is built in chunks: k chars at a time form a
// 32-bit digit of base (sigma+1)^k, then a multi-word multiply-add folds it in.
//
// Each producer also accumulates the 8-bit digit histograms of every radix pass
// of its keys, so the sort needs no extra read of the keys.
#pragma once

#include "common.cuh"
#include "radix.cuh"

namespace dcx {

constexpr int MAX_CHUNKS = 48;

struct KeyPlan {
    uint32_t base;                   // sigma + 1 (chars are 0..sigma)
    uint32_t chars;                  // chars encoded (window length)
    uint32_t kw;                     // key words holding the chars
    uint32_t nchunks;
    uint32_t chunk_len[MAX_CHUNKS];  // chars per chunk
    uint32_t chunk_mul[MAX_CHUNKS];  // (sigma+1)^chunk_len
};

template <typename CharT>
__device__ __forceinline__ uint32_t ldc(const CharT* p) {
    return (uint32_t)__ldg(p);
}

// Encodes chars text[start .. start+plan.chars) (0 at or past `end`) into acc[0..KW).
template <int KW, typename CharT>
__device__ __forceinline__ void encode_window(const CharT* text, uint64_t end, uint64_t start,
                                              const KeyPlan& plan, uint32_t* acc, uint32_t top = 0) {
#pragma unroll
    for (int w = 0; w < KW; w++) acc[w] = 0;
    acc[0] = top;  // most significant digit (text id), scaled up by the chunk multiplies
    uint64_t p = start;
    for (uint32_t c = 0; c < plan.nchunks; c++) {
        const uint32_t len = plan.chunk_len[c];
        const uint32_t base = plan.base;
        uint32_t digit = 0;  // the chunk's chars in base sigma+1 (< chunk_mul[c] <= 2^32-1)
        for (uint32_t j = 0; j < len; j++, p++) {
            uint32_t ch = p < end ? ldc(text + p) : 0u;
            digit = digit * base + ch;
        }
        const uint32_t mul = plan.chunk_mul[c];
        uint64_t carry = digit;
#pragma unroll
        for (int w = 0; w < KW; w++) {
            uint64_t t = (uint64_t)acc[w] * mul + carry;
            acc[w] = (uint32_t)t;
            carry = t >> 32;
        }
    }
}

struct KeyOut {
    uint32_t* w[MAX_KEY_WORDS];
};

// Adds one key's 8-bit digits of all 4*KW passes to the block histograms
// (static word/byte indexing keeps the key in registers).
// Each pair of warps owns a private copy of the histograms (HIST_COPIES copies
// per block), so near-constant top digits contend only within two warps.
constexpr int HIST_COPIES = 4;

template <int KW>
__device__ __forceinline__ void hist_add(uint32_t* sh, const uint32_t* key, uint32_t nbytes = 4 * KW) {
    uint32_t* h = sh + (threadIdx.x >> 6) * (4 * KW * RADIX);
#pragma unroll
    for (int w = 0; w < KW; w++)
#pragma unroll
        for (int b = 0; b < 4; b++)
            if ((uint32_t)(4 * w + b) < nbytes)  // higher digit bytes are zero by construction
                atomicAdd(&h[(4 * w + b) * RADIX + ((key[w] >> (8 * b)) & (RADIX - 1))], 1u);
}

// Zero the private copies / fold them into the global histogram.
__device__ __forceinline__ void hist_zero(uint32_t* sh, uint32_t bins) {
    for (uint32_t i = threadIdx.x; i < HIST_COPIES * bins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
}
__device__ __forceinline__ void hist_flush(const uint32_t* sh, uint32_t bins, uint32_t* hist) {
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < bins; i += blockDim.x) {
        uint32_t v = 0;
#pragma unroll
        for (int c = 0; c < HIST_COPIES; c++) v += sh[c * bins + i];
        if (v) atomicAdd(&hist[i], v);
    }
}

// Segments: a level holds K texts back to back, text s at [start[s], start[s+1]-1)
// followed by one 0 at start[s+1]-1 (its empty suffix).  A window reads 0 from
// its own text's end on, so windows never see the next text.  With K = 1 this
// is the single text of length n = start[1] - 1.
struct SegView {
    uint32_t K;
    const uint64_t* start;  // [K + 1]
};

__device__ __forceinline__ uint32_t seg_of(const SegView& sv, uint64_t p) {
    uint32_t lo = 0, hi = sv.K;  // largest s with start[s] <= p
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sv.start[mid] <= p) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ uint64_t seg_end(const SegView& sv, uint32_t s) { return sv.start[s + 1] - 1; }

// Level keys: for every position i in [0, N), key = text * B^chars + window
// [i, i+chars) of i's text (the text id is the most significant mixed-radix
// digit), value = i.
template <int KW, bool SEG, typename CharT>
__global__ __launch_bounds__(256) void k_keys_prefix(const CharT* __restrict__ text, uint64_t N, SegView sv,
                                                     KeyPlan plan, KeyOut ko, uint32_t* __restrict__ vals_out,
                                                     uint32_t* hist) {
    extern __shared__ uint32_t sh[];  // HIST_COPIES * 4*KW * RADIX
    hist_zero(sh, 4 * KW * RADIX);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sg = SEG ? seg_of(sv, i) : 0u;
        uint32_t key[KW];
        encode_window<KW>(text, seg_end(sv, sg), i, plan, key, sg);  // key = text * B^P + window
#pragma unroll
        for (int w = 0; w < KW; w++) ko.w[w][i] = key[w];
        vals_out[i] = (uint32_t)i;
        hist_add<KW>(sh, key);
    }
    hist_flush(sh, 4 * KW * RADIX, hist);
}

// Level keys for windows of at most 64 bits, built with a sliding window: a CTA
// stages SLIDE_TILE + chars of text in shared memory, thread t encodes the
// SLIDE_R consecutive positions [t*R, t*R + R) of the tile (one full encode,
// then key' = (key - c_i * B^(P-1)) * B + c_{i+P} per step, restarting at the
// first position of each text), and the keys are written back through shared
// memory so global stores stay coalesced.
constexpr int SLIDE_THREADS = 256;
constexpr int SLIDE_R = 16;
constexpr int SLIDE_TILE = SLIDE_THREADS * SLIDE_R;
constexpr int SLIDE_MAX_CHARS = 64;

// Padded shared-memory indices: thread t works on positions [16t, 16t+16), so
// unpadded rows of 16 keys (128 B) or 16 chars (16 B) would put a warp's lanes
// on the same banks.  One spare key per 16 keys and 4 spare bytes per 16 chars
// spread the lanes over the banks.
__device__ __forceinline__ uint32_t slide_kidx(uint32_t i) { return i + (i >> 4); }
__device__ __forceinline__ uint32_t slide_cidx(uint32_t i) { return i + ((i >> 4) << 2); }

template <bool SEG, typename CharT>
__global__ __launch_bounds__(SLIDE_THREADS) void k_keys_slide(const CharT* __restrict__ text, uint64_t N, SegView sv,
                                                              KeyPlan plan, uint64_t pow_top, uint64_t seg_mul,
                                                              KeyOut ko, uint32_t* __restrict__ vals_out,
                                                              uint32_t* hist, uint32_t nbytes) {
    extern __shared__ uint32_t sh[];  // HIST_COPIES * 8 * RADIX histogram words, then the staging area
    uint32_t* hst = sh;
    uint64_t* s_keys = reinterpret_cast<uint64_t*>(sh + HIST_COPIES * 8 * RADIX);  // SLIDE_TILE keys, padded
    CharT* s_chars = reinterpret_cast<CharT*>(s_keys + SLIDE_TILE + SLIDE_TILE / 16);  // SLIDE_TILE + P, padded
    const uint32_t W = plan.kw;
    hist_zero(hst, 4 * W * RADIX);
    const uint32_t P = plan.chars;
    const uint64_t B = plan.base;
    for (uint64_t base = (uint64_t)blockIdx.x * SLIDE_TILE; base < N; base += (uint64_t)gridDim.x * SLIDE_TILE) {
        for (uint32_t i = threadIdx.x; i < SLIDE_TILE + P; i += SLIDE_THREADS) {
            const uint64_t p = base + i;
            s_chars[slide_cidx(i)] = p < N ? text[p] : CharT(0);
        }
        __syncthreads();
        const uint32_t r0 = threadIdx.x * SLIDE_R;
        uint32_t sg = SEG ? seg_of(sv, base + r0) : 0u;
        uint64_t end = seg_end(sv, sg);  // position of the text's 0
        auto full = [&](uint32_t r) {     // window of tile position r, cut at `end`
            uint64_t k = 0;
            for (uint32_t j = 0; j < P; j++)
                k = k * B + ((base + r + j < end) ? (uint32_t)s_chars[slide_cidx(r + j)] : 0u);
            return k;
        };
        uint64_t key = full(r0);
#pragma unroll
        for (int r = 0; r < SLIDE_R; r++) {
            const uint64_t i = base + r0 + r;
            s_keys[slide_kidx(r0 + r)] = SEG ? key + (uint64_t)sg * seg_mul : key;  // text * B^P + window
            if (i == end) {  // next position starts the next text
                if (SEG && sg + 1 < sv.K) {
                    sg++;
                    end = seg_end(sv, sg);
                }
                key = full(r0 + r + 1);
            } else {
                const uint32_t out = (uint32_t)s_chars[slide_cidx(r0 + r)];
                const uint32_t in = (i + P < end) ? (uint32_t)s_chars[slide_cidx(r0 + r + P)] : 0u;
                key = (key - (uint64_t)out * pow_top) * B + in;
            }
        }
        __syncthreads();
        const uint32_t tile_n = (uint32_t)((N - base) < SLIDE_TILE ? (N - base) : SLIDE_TILE);
        for (uint32_t i = threadIdx.x; i < tile_n; i += SLIDE_THREADS) {
            const uint64_t k = s_keys[slide_kidx(i)];
            uint32_t kk[2] = {(uint32_t)k, (uint32_t)(k >> 32)};
            ko.w[0][base + i] = kk[0];
            if (W > 1) ko.w[1][base + i] = kk[1];
            vals_out[base + i] = (uint32_t)(base + i);
            if (W == 2) hist_add<2>(hst, kk, nbytes);
            else hist_add<1>(hst, kk, nbytes);
        }
        __syncthreads();
    }
    hist_flush(hst, 4 * W * RADIX, hist);
}

template <typename CharT>
constexpr size_t keys_slide_smem() {
    return sizeof(uint32_t) * HIST_COPIES * 8 * RADIX + sizeof(uint64_t) * (SLIDE_TILE + SLIDE_TILE / 16) +
           sizeof(CharT) * (SLIDE_TILE + SLIDE_MAX_CHARS) * 5 / 4 + 64;
}

// Text id of every sorted element: the key is text-major and text s has
// start[s+1] - start[s] elements, so it owns sorted slots [start[s], start[s+1]).
// A block covers FILL_TILE consecutive slots: two binary searches bound the
// texts of the tile, and each slot searches only inside that range (zero steps
// when the tile lies in one text); stores are coalesced.
constexpr uint32_t FILL_TILE = 2048;

__global__ __launch_bounds__(256) void k_fill_segw(SegView sv, uint64_t N, uint32_t* __restrict__ segw) {
    __shared__ uint32_t s_lo, s_hi;
    for (uint64_t t = (uint64_t)blockIdx.x * FILL_TILE; t < N; t += (uint64_t)gridDim.x * FILL_TILE) {
        const uint64_t e = t + FILL_TILE < N ? t + FILL_TILE : N;
        if (threadIdx.x == 0) {
            s_lo = seg_of(sv, t);
            s_hi = seg_of(sv, e - 1);
        }
        __syncthreads();
        const uint32_t lo0 = s_lo, hi0 = s_hi;
        for (uint64_t k = t + threadIdx.x; k < e; k += blockDim.x) {
            uint32_t lo = lo0, hi = hi0 + 1;  // largest s in [lo0, hi0] with start[s] <= k
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (sv.start[mid] <= k) lo = mid; else hi = mid;
            }
            segw[k] = lo;
        }
        __syncthreads();
    }
}

// Refinement keys for the elements of tie groups: element j has text position
// tpos[j], text tseg[j] and group number grp[j].  The key is (group number in
// the top word, window [pos+off, pos+off+chars) of its text below it); value =
// text position.
template <int KW, typename CharT>
__global__ __launch_bounds__(256) void k_keys_refine(const CharT* __restrict__ text, SegView sv, uint64_t count,
                                                     const uint32_t* __restrict__ tpos,
                                                     const uint32_t* __restrict__ tseg,
                                                     const uint32_t* __restrict__ grp, uint32_t off,
                                                     KeyPlan plan, KeyOut ko, uint32_t* __restrict__ vals_out,
                                                     uint32_t* hist) {
    extern __shared__ uint32_t sh[];  // HIST_COPIES * 4*(KW+1) * RADIX
    hist_zero(sh, 4 * (KW + 1) * RADIX);
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < count;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t pos = tpos[j];
        const uint64_t end = seg_end(sv, tseg ? tseg[j] : 0u);
        uint32_t key[KW + 1];
        encode_window<KW>(text, end, (uint64_t)pos + off, plan, key);
        key[KW] = grp[j];
#pragma unroll
        for (int w = 0; w <= KW; w++) ko.w[w][j] = key[w];
        vals_out[j] = pos;
        hist_add<KW + 1>(sh, key);
    }
    hist_flush(sh, 4 * (KW + 1) * RADIX, hist);
}

// Refinement keys of byte texts (base B <= 256, window P <= 64 chars, key < 2^64).
// The window [s, s+P) is read as aligned 8-byte words (independent loads, at
// most 9), funnel-shifted so that word k holds window chars 8k..8k+7, and each
// word is folded into its base-B value with three SWAR multiply-adds (pairs,
// quads, octets; no lane overflows for B <= 256).  Chars at or past the text's
// end count as 0.  The integer equals the one encode_window builds.
struct RefinePlan8 {
    uint32_t P, m, r;          // chars, words (ceil(P/8)), chars in the last word
    uint64_t B, B2, B4;        // B, B^2, B^4
    uint64_t pow8, powr;       // B^8, B^r
};

__device__ __forceinline__ uint64_t swar_digits8(uint64_t w, const RefinePlan8& rp) {
    // byte 0 is the most significant digit
    const uint64_t t16 = (w & 0x00ff00ff00ff00ffull) * rp.B + ((w >> 8) & 0x00ff00ff00ff00ffull);
    const uint64_t t32 = (t16 & 0x0000ffff0000ffffull) * rp.B2 + ((t16 >> 16) & 0x0000ffff0000ffffull);
    return (t32 & 0xffffffffull) * rp.B4 + (t32 >> 32);
}

// Base-B value of the rp.P chars at s (chars at or past `end` count as 0).
__device__ __forceinline__ uint64_t window_value8(const uint64_t* __restrict__ tw0, uint64_t s, uint64_t end,
                                                  const RefinePlan8& rp) {
    const uint64_t a0 = s & ~7ull;
    const uint32_t shb = (uint32_t)(s - a0) * 8u;
    uint64_t w[9];
#pragma unroll
    for (int k = 0; k < 9; k++)  // words at or past the end hold only zero chars: not read
        w[k] = ((uint32_t)k <= rp.m && a0 + 8ull * k < end) ? __ldg(tw0 + (a0 >> 3) + k) : 0ull;
    const uint64_t v = end > s ? end - s : 0;  // window chars inside the text
    uint64_t key = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if ((uint32_t)k >= rp.m) break;
        uint64_t cw = shb ? (w[k] >> shb) | (w[k + 1] << (64u - shb)) : w[k];
        const int64_t vk = (int64_t)v - 8 * k;
        if (vk < 8) cw = vk <= 0 ? 0ull : cw & ((1ull << (8 * vk)) - 1ull);
        const bool last = (uint32_t)k == rp.m - 1;
        if (last && rp.r < 8) cw <<= 8u * (8u - rp.r);  // drop chars past the window; keep r low digits
        key = key * (last ? rp.powr : rp.pow8) + swar_digits8(cw, rp);
    }
    return key;
}

// Window value for the segmented refinement: byte texts use the SWAR word
// loader, 32-bit texts (alphabet of 256 symbols) fold rp.P chars directly.
__device__ __forceinline__ uint64_t window_value_t(const uint8_t* t, uint64_t s, uint64_t end, const RefinePlan8& rp) {
    return window_value8(reinterpret_cast<const uint64_t*>(t), s, end, rp);
}
__device__ __forceinline__ uint64_t window_value_t(const uint32_t* t, uint64_t s, uint64_t end, const RefinePlan8& rp) {
    uint64_t k = 0;
    for (uint32_t j = 0; j < rp.P; j++) {
        const uint64_t p = s + j;
        k = k * rp.B + (p < end ? __ldg(t + p) : 0u);
    }
    return k;
}

template <int KW>
__global__ __launch_bounds__(256) void k_keys_refine8(const uint8_t* __restrict__ text, SegView sv, uint64_t count,
                                                      const uint32_t* __restrict__ tpos,
                                                      const uint32_t* __restrict__ tseg,
                                                      const uint32_t* __restrict__ grp, uint32_t off, RefinePlan8 rp,
                                                      KeyOut ko, uint32_t* __restrict__ vals_out, uint32_t* hist) {
    extern __shared__ uint32_t sh[];  // HIST_COPIES * 4*(KW+1) * RADIX
    hist_zero(sh, 4 * (KW + 1) * RADIX);
    const uint64_t* tw0 = reinterpret_cast<const uint64_t*>(text);
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < count;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t pos = tpos[j];
        const uint64_t end = seg_end(sv, tseg ? tseg[j] : 0u);
        const uint64_t key = window_value8(tw0, (uint64_t)pos + off, end, rp);
        uint32_t kk[KW + 1];
        kk[0] = (uint32_t)key;
        if (KW > 1) kk[1] = (uint32_t)(key >> 32);
        kk[KW] = grp[j];
#pragma unroll
        for (int w2 = 0; w2 <= KW; w2++) ko.w[w2][j] = kk[w2];
        vals_out[j] = pos;
        hist_add<KW + 1>(sh, kk);
    }
    hist_flush(sh, 4 * (KW + 1) * RADIX, hist);
}

// Refinement of small tie groups inside one CTA: the elements of a group (up
// to C, all of one text) get the rest of their window, chars [off, L), as W
// words of base-B chunks (lexicographic order of the words = order of the
// chars), a bitonic network in shared memory sorts 16-bit indices by them, and
// the group is written back with head flags where the words change.  Equal
// windows stay tied (head 0) for the cover-rank tie break.  The CTA loops over
// groups.
constexpr int RSEG_MAX_W = 6;
struct RefineSegPlan {
    uint32_t W;                       // words per element
    uint32_t off[RSEG_MAX_W];         // first char of each word, relative to the position
    RefinePlan8 rp[RSEG_MAX_W];
};

template <int C, int THREADS, int W, typename CharT>
__global__ __launch_bounds__(THREADS) void k_refine_seg(const CharT* __restrict__ text, SegView sv,
                                                        const uint32_t* __restrict__ segw,
                                                        const uint32_t* __restrict__ gstart,
                                                        const uint32_t* __restrict__ gsize, uint64_t ngroups,
                                                        uint32_t* __restrict__ sa, uint8_t* __restrict__ head,
                                                        RefineSegPlan plan) {
    static_assert(C <= 65536 && (C & (C - 1)) == 0, "power-of-two groups, 16-bit indices");
    extern __shared__ __align__(16) uint64_t s_dyn64[];  // refine_seg_smem<C, W>() bytes
    uint64_t(*s_key)[C] = reinterpret_cast<uint64_t(*)[C]>(s_dyn64);             // [W][C]
    uint32_t* s_pos = reinterpret_cast<uint32_t*>(s_dyn64 + (size_t)W * C);      // [C]
    uint16_t* s_idx = reinterpret_cast<uint16_t*>(s_pos + C);                    // [C]
    for (uint64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const uint32_t start = gstart[g], size = gsize[g];
        const uint64_t end = seg_end(sv, segw ? segw[start] : 0u);
        // all positions first, then all windows: the loads of a thread's
        // elements are independent and overlap
        constexpr int PER = C / THREADS;
        static_assert(PER * THREADS == C, "C is a multiple of THREADS");
        uint32_t pj[PER];
#pragma unroll
        for (int j = 0; j < PER; j++) {
            const uint32_t i = threadIdx.x + j * THREADS;
            s_idx[i] = (uint16_t)i;
            pj[j] = i < size ? sa[start + i] : 0u;
        }
#pragma unroll
        for (int j = 0; j < PER; j++) {
            const uint32_t i = threadIdx.x + j * THREADS;
            if (i < size) {
                s_pos[i] = pj[j];
#pragma unroll
                for (int w = 0; w < W; w++)
                    s_key[w][i] = window_value_t(text, (uint64_t)pj[j] + plan.off[w], end, plan.rp[w]);
            }
        }
        __syncthreads();
        auto less = [&](uint32_t a, uint32_t b) -> bool {  // padding (index >= size) sorts last
            if (a >= size) return false;
            if (b >= size) return true;
#pragma unroll
            for (int w = 0; w < W; w++) {
                const uint64_t ka = s_key[w][a], kb = s_key[w][b];
                if (ka != kb) return ka < kb;
            }
            return false;
        };
#pragma unroll
        for (uint32_t k = 2; k <= (uint32_t)C; k <<= 1) {
#pragma unroll
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
                for (uint32_t p = threadIdx.x; p < (uint32_t)C / 2; p += THREADS) {
                    const uint32_t i = ((p & ~(j - 1)) << 1) | (p & (j - 1));
                    const uint32_t q = i + j;
                    const uint32_t a = s_idx[i], b = s_idx[q];
                    if ((i & k) == 0 ? less(b, a) : less(a, b)) {
                        s_idx[i] = (uint16_t)b;
                        s_idx[q] = (uint16_t)a;
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t i = threadIdx.x; i < size; i += THREADS) {
            const uint32_t a = s_idx[i];
            sa[start + i] = s_pos[a];
            if (i > 0) {  // the group's first element keeps its head flag
                const uint32_t b = s_idx[i - 1];
                bool diff = false;
#pragma unroll
                for (int w = 0; w < W; w++) diff |= s_key[w][a] != s_key[w][b];
                head[start + i] = diff ? 1 : 0;
            }
        }
        __syncthreads();
    }
}

// Groups of exactly two: one thread per group.
template <int W, typename CharT>
__global__ __launch_bounds__(256) void k_refine_pair(const CharT* __restrict__ text, SegView sv,
                                                     const uint32_t* __restrict__ segw,
                                                     const uint32_t* __restrict__ gstart, uint64_t ngroups,
                                                     uint32_t* __restrict__ sa, uint8_t* __restrict__ head,
                                                     RefineSegPlan plan) {
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t start = gstart[g];
        const uint64_t end = seg_end(sv, segw ? segw[start] : 0u);
        const uint32_t a = sa[start], b = sa[start + 1];
        int cmp = 0;  // sign of key(a) - key(b)
#pragma unroll
        for (int w = 0; w < W; w++) {
            if (cmp) break;
            const uint64_t ka = window_value_t(text, (uint64_t)a + plan.off[w], end, plan.rp[w]);
            const uint64_t kb = window_value_t(text, (uint64_t)b + plan.off[w], end, plan.rp[w]);
            cmp = ka < kb ? -1 : (ka > kb ? 1 : 0);
        }
        if (cmp > 0) {
            sa[start] = b;
            sa[start + 1] = a;
        }
        head[start + 1] = cmp != 0;
    }
}

// Groups of 3..LANES elements (LANES = 4, 8, 16 or 32): LANES lanes per group,
// 32 / LANES groups per warp, one element per lane, a bitonic network over the
// group's lanes with shuffles.
template <int W, int LANES, typename CharT>
__global__ __launch_bounds__(256) void k_refine_warp(const CharT* __restrict__ text, SegView sv,
                                                     const uint32_t* __restrict__ segw,
                                                     const uint32_t* __restrict__ gstart,
                                                     const uint32_t* __restrict__ gsize, uint64_t ngroups,
                                                     uint32_t* __restrict__ sa, uint8_t* __restrict__ head,
                                                     RefineSegPlan plan) {
    static_assert(LANES >= 2 && LANES <= 32 && (LANES & (LANES - 1)) == 0, "power-of-two lanes");
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t l = lane % LANES;
    const uint64_t slots = ((uint64_t)gridDim.x * blockDim.x) / LANES;
    for (uint64_t g0 = ((uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u)) / LANES;
         g0 < ngroups; g0 += slots) {
        const uint64_t g = g0 + lane / LANES;  // every lane of the warp runs the network
        uint32_t start = 0, size = 0;
        uint64_t end = 0;
        if (g < ngroups) {
            start = gstart[g];
            size = gsize[g];
            end = seg_end(sv, segw ? segw[start] : 0u);
        }
        bool valid = l < size;
        uint32_t p = valid ? sa[start + l] : 0u;
        uint64_t key[W];
#pragma unroll
        for (int w = 0; w < W; w++) key[w] = valid ? window_value_t(text, (uint64_t)p + plan.off[w], end, plan.rp[w]) : 0ull;
#pragma unroll
        for (int k = 2; k <= LANES; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                const bool ov = __shfl_xor_sync(0xffffffffu, valid, j);
                const uint32_t op = __shfl_xor_sync(0xffffffffu, p, j);
                uint64_t ok[W];
#pragma unroll
                for (int w = 0; w < W; w++) ok[w] = __shfl_xor_sync(0xffffffffu, key[w], j);
                // other < me / me < other (invalid lanes sort last)
                int c = 0;
#pragma unroll
                for (int w = 0; w < W; w++)
                    if (!c && ok[w] != key[w]) c = ok[w] < key[w] ? -1 : 1;
                const bool o_less = ov && (!valid || c < 0);
                const bool m_less = valid && (!ov || c > 0);
                const bool up = (k == LANES) || ((l & k) == 0);
                const bool lower = (l & j) == 0;
                if ((lower == up) ? o_less : m_less) {
                    valid = ov;
                    p = op;
#pragma unroll
                    for (int w = 0; w < W; w++) key[w] = ok[w];
                }
            }
        }
        bool diff = false;
#pragma unroll
        for (int w = 0; w < W; w++) diff |= __shfl_up_sync(0xffffffffu, key[w], 1, LANES) != key[w];
        if (valid) {
            sa[start + l] = p;
            if (l > 0) head[start + l] = diff;
        }
    }
}

template <int C, int W>
constexpr size_t refine_seg_smem() {
    return sizeof(uint64_t) * W * C + sizeof(uint32_t) * C + sizeof(uint16_t) * C;
}

// Sets (value 1) or copies (from src) the flags of the elements of groups.
__global__ void k_group_flags(const uint32_t* __restrict__ gstart, const uint32_t* __restrict__ gsize, uint64_t ngroups,
                              uint8_t* __restrict__ dst, const uint8_t* __restrict__ src) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t g = warp; g < ngroups; g += warps) {
        const uint32_t st = gstart[g], sz = gsize[g];
        for (uint32_t i = lane; i < sz; i += 32) dst[st + i] = src ? src[st + i] : (uint8_t)1;
    }
}

}  // namespace dcx