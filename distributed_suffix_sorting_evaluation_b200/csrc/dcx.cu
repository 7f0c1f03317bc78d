// B200 DCX suffix-array engine: host orchestration of one DCX level and the C ABI.
//
// One level follows PDCX::compute_sa (lightweight_dcx/src/pdcx/pdcx.hpp:529-941):
//   phase 0  lengths, dummy sample, key plan           (pdcx.hpp:473-510)
//   phase 1  sort suffixes by their first L chars       (sample_string.hpp:129-239)
//   phase 2  lexicographic names + unique flags         (compute_ranks.hpp:89-134)
//   phase 3  recursion unless names are distinct        (pdcx.hpp:146-462,743-757)
//   phase 4  order ties by difference-cover ranks       (merge_samples.hpp:87-109,262-306)
// Design difference from the reference: phase 1 and phase 4 share ONE sort.  All
// n+1 suffixes (position n is the empty suffix / dummy sample) are radix sorted
// by their L-char window, which orders the samples exactly as phase 1 needs them
// (a sample sort restricted to samples) and orders every non-tied suffix finally
// (the reference's phase-4 comparator compares the same packed chars first).
// Only suffixes whose whole window ties need the rank comparison afterwards.
// The window sort runs as a short prefix radix sort followed by refinement sorts
// of just the tied elements (group number, next chars).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "keys.cuh"
#include "level_kernels.cuh"
#include "radix.cuh"
#include "segsort.cuh"
#include "small_sa.cuh"
#include "warpsort.cuh"
#include "lcp.cuh"
#include "lcp_scatter.cuh"
#include "bwt.cuh"
#include "gsa.cuh"

namespace dcx {

// ---------------------------------------------------------------------------
// Difference covers of lightweight_dcx/src/pdcx/difference_cover.hpp:14-5126 (the
// sets only; IN_DC, NEXT_RANK and cmpDepthRanks are generated in closed form).
// ---------------------------------------------------------------------------
struct DcHost {
    uint32_t X = 0, D = 0;
    std::vector<uint32_t> dc, next_rank, cmp;  // cmp: [X][X][3]
    std::vector<uint8_t> in_dc;
};

static bool cover_of(uint32_t X, std::vector<uint32_t>& s) {
    switch (X) {
        case 3: s = {1, 2}; return true;
        case 7: s = {1, 2, 4}; return true;
        case 13: s = {1, 2, 4, 10}; return true;
        case 21: s = {1, 2, 7, 9, 19}; return true;
        case 31: s = {1, 2, 4, 9, 13, 19}; return true;
        case 39: s = {1, 2, 17, 21, 23, 28, 31}; return true;
        case 57: s = {1, 2, 10, 12, 15, 36, 40, 52}; return true;
        case 73: s = {1, 2, 4, 8, 16, 32, 37, 55, 64}; return true;
        case 91: s = {1, 2, 8, 17, 28, 57, 61, 69, 71, 74}; return true;
        case 95: s = {1, 2, 6, 9, 19, 21, 30, 32, 46, 62, 68}; return true;
        case 133: s = {1, 2, 33, 43, 45, 49, 52, 60, 73, 78, 98, 112}; return true;
        default: return false;
    }
}

static bool make_dc(uint32_t X, DcHost& t) {
    if (!cover_of(X, t.dc)) return false;
    t.X = X;
    t.D = (uint32_t)t.dc.size();
    t.in_dc.assign(X, 0);
    for (uint32_t c : t.dc) t.in_dc[c] = 1;
    t.next_rank.assign(X, 0);
    for (uint32_t r = 0; r < X; r++)
        for (uint32_t c : t.dc) t.next_rank[r] += c < r;
    t.cmp.assign((size_t)X * X * 3, 0);
    for (uint32_t i = 0; i < X; i++)
        for (uint32_t j = 0; j < X; j++) {
            uint32_t l = 0;
            while (!(t.in_dc[(i + l) % X] && t.in_dc[(j + l) % X])) l++;
            uint32_t r1 = 0, r2 = 0;
            for (uint32_t k = 0; k < l; k++) {
                r1 += t.in_dc[(i + k) % X];
                r2 += t.in_dc[(j + k) % X];
            }
            uint32_t* e = &t.cmp[((size_t)i * X + j) * 3];
            e[0] = l;
            e[1] = r1;
            e[2] = r2;
        }
    return true;
}

// ---------------------------------------------------------------------------
// Key plans: number of chars of base B that fit in w words, and the chunking.
// ---------------------------------------------------------------------------
struct BigUInt {  // little-endian 32-bit limbs
    std::vector<uint32_t> l{1};
    void mul(uint32_t f) {
        uint64_t carry = 0;
        for (auto& x : l) {
            uint64_t t = (uint64_t)x * f + carry;
            x = (uint32_t)t;
            carry = t >> 32;
        }
        if (carry) l.push_back((uint32_t)carry);
    }
    uint32_t bits_of_minus_one() const {  // bit length of (this - 1), this >= 1
        std::vector<uint32_t> v = l;
        for (auto& x : v) {
            if (x) {
                x--;
                break;
            }
            x = 0xffffffffu;
        }
        while (v.size() > 1 && v.back() == 0) v.pop_back();
        uint32_t top = v.back();
        uint32_t b = 0;
        while (top) {
            b++;
            top >>= 1;
        }
        return (uint32_t)(v.size() - 1) * 32 + b;
    }
};

// Bits of the largest key K * B^P - 1 (K texts, P chars of base B).
static uint32_t key_bits_k(uint64_t B, uint32_t P, uint64_t K) {
    BigUInt x;
    if (K > 1) {
        x.mul((uint32_t)(K & 0xffffffffu));
        if (K >> 32) throw Error(DCX_ERR_ARG, "too many texts");
    }
    for (uint32_t i = 0; i < P; i++) x.mul((uint32_t)B);
    return std::max<uint32_t>(1, x.bits_of_minus_one());
}

// Largest P with K * B^P - 1 < 2^bits.
static uint32_t max_chars_in_bits_k(uint64_t B, uint32_t bits, uint64_t K) {
    uint32_t P = 0;
    BigUInt x;
    if (K > 1) x.mul((uint32_t)K);
    if (x.bits_of_minus_one() > bits) return 0;
    while (true) {
        BigUInt y = x;
        y.mul((uint32_t)B);
        if (y.bits_of_minus_one() > bits) break;
        x = y;
        P++;
        if (P > 4096) break;
    }
    return P;
}

static uint32_t max_chars_in_bits(uint64_t B, uint32_t bits) { return max_chars_in_bits_k(B, bits, 1); }
static uint32_t max_chars_in(uint64_t B, uint32_t words) { return max_chars_in_bits(B, 32 * words); }

// Chunked encoding of P chars of base B; the key words also hold a text id
// digit (0..K-1) above the chars.
static KeyPlan make_plan(uint64_t B, uint32_t P, uint64_t K = 1) {
    KeyPlan p{};
    p.base = (uint32_t)B;
    p.chars = P;
    p.kw = (key_bits_k(B, P, K) + 31) / 32;
    uint32_t kmax = 1;
    {
        uint64_t v = B;
        while (v * B <= 0xffffffffull) {
            v *= B;
            kmax++;
        }
    }
    uint32_t left = P;
    p.nchunks = 0;
    while (left) {
        uint32_t len = std::min(left, kmax);
        uint64_t mul = 1;
        for (uint32_t i = 0; i < len; i++) mul *= B;
        if (p.nchunks >= (uint32_t)MAX_CHUNKS) throw Error(DCX_ERR_INTERNAL, "key plan too long");
        p.chunk_len[p.nchunks] = len;
        p.chunk_mul[p.nchunks] = (uint32_t)mul;
        p.nchunks++;
        left -= len;
    }
    return p;
}

// ---------------------------------------------------------------------------
// Context: stream, memory accounting, scratch, options, statistics.
// ---------------------------------------------------------------------------
constexpr size_t PINNED_WORDS = 1 << 14;  // 64 KiB: two 16-pass x 256-bin tables

struct Options {
    double discarding_threshold = 0.7;
    uint32_t recursion_dc = 3;
    uint32_t small_threshold = SMALL_MAX;
    uint32_t prefix_chars = 0;
    // key words of the round-0 prefix at recursion levels (2 or 3; the rest of
    // the window is refined inside the tie groups)
    uint32_t rec_prefix_words = 3;
    // items per thread of a radix tile: 16 (4096-element tiles, the default) or 12 (3072)
    uint32_t radix_items = ONESWEEP_ITEMS;
    int trace = 0;
    uint32_t spin_limit = 1u << 24;
    // failure-detection test hook: this tile of every radix pass never publishes
    // its look-back status, so the next tile's bounded wait runs out
    uint32_t lookback_hold_tile = 0xffffffffu;
    uint64_t batch_round_cap = 0;  // max elements per batch round (0 = from the budget)
    // DC per size class of batched builds with dc_or_auto = 0: (longest text of
    // the class, X), ascending; longer texts and an empty table use DC39
    std::vector<std::pair<uint64_t, uint32_t>> batch_dc;
    // radix tile items per class of batch_dc (empty: the context's radix_items);
    // the autotuner fills it when batch_tune_tiles is set
    std::vector<uint32_t> batch_items;
    int batch_tune_tiles = 1;
    // serving
    uint32_t serve_lanes = 1;
    uint64_t serve_budget = 0;  // 0 = the context budget
    uint64_t serve_batch_bytes = 1ull << 30;
    uint32_t serve_batch_texts = 65536;
    uint64_t serve_host_bytes = 8ull << 30;  // pinned host arena for request copies
    uint64_t serve_express_bytes = 4ull << 20;  // longest request the express lanes take
    int serve_express_priority = 1;               // express lanes on high-priority streams
};

struct Ctx;

template <typename T>
struct DBuf {
    Ctx* c = nullptr;
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(Ctx* ctx, size_t count);
    DBuf(Ctx* ctx, size_t count, bool io);  // io: the context's staging pool (see Ctx::io_pool)
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept { *this = std::move(o); }
    DBuf& operator=(DBuf&& o) noexcept;
    ~DBuf() { reset(); }
    void reset();
    T* get() const { return p; }
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    uint64_t in_use = 0, peak = 0;
    Options opt;
    dcx_stats st{};
    // scratch
    uint32_t* d_hist = nullptr;     // [16 * RADIX]
    uint32_t* d_base = nullptr;     // [16 * RADIX]
    uint32_t* d_tiles = nullptr;    // [16]
    uint32_t* d_err = nullptr;      // [2]: error bits, look-back give-ups
    unsigned long long* d_h256 = nullptr;
    uint64_t* d_lookback = nullptr;
    size_t lookback_tiles = 0;
    uint32_t epoch = 0;
    uint32_t* h_pinned = nullptr;   // pinned staging for small transfers (PINNED_WORDS words)
    cudaMemPool_t pool = nullptr;   // own memory pool (serving lanes); null = the device's default pool
    // Staging buffers of host-pointer calls (text copy, SA before its download)
    // live in a pool of their own: placed among the build's scratch they would
    // split the scratch pool's free blocks differently from one call type to the
    // next and force the pool to map new memory inside the build.
    cudaMemPool_t io_pool = nullptr;
    std::map<uint32_t, DcHost> dc_host;
    std::map<uint32_t, DcFlags*> dc_flags_dev;  // per X (samples_before filled per level on a copy)
    std::map<uint32_t, DcDev*> dc_dev;
    // trace of level 0
    double level0_entropy = 0;  // order-0 entropy (bits/char) of the current level-0 text
    std::vector<uint32_t> trace_names;
    std::vector<uint8_t> trace_uniq;
    std::mutex build_mu;

    void* alloc(size_t bytes, bool io = false) {
        if (bytes == 0) bytes = 16;
        bytes = (bytes + 255) & ~size_t(255);
        if (budget && in_use + bytes > budget)
            throw Error(DCX_ERR_BUDGET, "device footprint above the context budget");
        void* p = nullptr;
        cudaMemPool_t from = (io && io_pool) ? io_pool : pool;
        cudaError_t e = from ? cudaMallocFromPoolAsync(&p, bytes, from, stream) : cudaMallocAsync(&p, bytes, stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(DCX_ERR_OOM, "cudaMallocAsync failed for " + std::to_string(bytes) + " bytes");
        }
        in_use += bytes;
        peak = std::max(peak, in_use);
        return p;
    }
    void release(void* p, size_t bytes) {
        if (!p) return;
        if (bytes == 0) bytes = 16;
        bytes = (bytes + 255) & ~size_t(255);
        cudaFreeAsync(p, stream);
        in_use -= bytes;
    }
    void launched(uint64_t k = 1) { st.kernel_launches += k; }
    void alg(uint64_t b) { st.bytes_alg += b; }
};

template <typename T>
DBuf<T>::DBuf(Ctx* ctx, size_t count) : c(ctx), n(count) {
    p = static_cast<T*>(ctx->alloc(count * sizeof(T)));
}
template <typename T>
DBuf<T>::DBuf(Ctx* ctx, size_t count, bool io) : c(ctx), n(count) {
    p = static_cast<T*>(ctx->alloc(count * sizeof(T), io));
}
template <typename T>
DBuf<T>& DBuf<T>::operator=(DBuf&& o) noexcept {
    if (this != &o) {
        reset();
        c = o.c;
        p = o.p;
        n = o.n;
        o.p = nullptr;
        o.n = 0;
    }
    return *this;
}
template <typename T>
void DBuf<T>::reset() {
    if (p && c) c->release(p, n * sizeof(T));
    p = nullptr;
    n = 0;
}

static int grid_for(uint64_t n, int threads, int max_blocks = 148 * 16) {
    uint64_t b = div_up(std::max<uint64_t>(n, 1), threads);
    return (int)std::min<uint64_t>(b, (uint64_t)max_blocks);
}

// Bytes the context's allocation pool holds from the device (reserved, used or
// not); a build that has to grow it pays for mapping new memory.
static uint64_t pool_reserved(Ctx& c) {
    cudaMemPool_t p = c.pool;
    if (!p && cudaDeviceGetDefaultMemPool(&p, c.device) != cudaSuccess) return 0;
    uint64_t v = 0;
    if (cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemCurrent, &v) != cudaSuccess) return 0;
    return (uint64_t)v;
}

// Small device->host reads go through the context's pinned staging area.
template <typename T>
static T d2h_scalar(Ctx& c, const T* dptr) {
    T* h = reinterpret_cast<T*>(c.h_pinned);
    DCX_CUDA(cudaMemcpyAsync(h, dptr, sizeof(T), cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    return *h;
}

// d_err[0]: error bits of the kernels; d_err[1]: CTAs whose look-back wait ran
// out (counted into the build's statistics).
static void check_device_error(Ctx& c) {
    const uint64_t v = d2h_scalar(c, reinterpret_cast<const uint64_t*>(c.d_err));
    const uint32_t e = (uint32_t)v, gave_up = (uint32_t)(v >> 32);
    if (v) DCX_CUDA(cudaMemsetAsync(c.d_err, 0, 8, c.stream));
    c.st.lookback_gave_up += gave_up;
    if (e) {
        if (e & DEV_ERR_TIMEOUT) throw Error(DCX_ERR_TIMEOUT, "a bounded device wait gave up");
        throw Error(DCX_ERR_INTERNAL, "device range check failed");
    }
}

// Device-wide exclusive scan with operator Op; returns the grand total.
template <typename T, typename Op>
static T device_scan(Ctx& c, const Op& op, uint64_t n) {
    if (n == 0) return T(0);
    const uint64_t tiles = div_up(n, SCAN_TILE);
    // One chunk of tiles per CTA, as many CTAs as the rescan kernel keeps
    // resident (its registers decide: 3-6 per SM), so both phases run as a single
    // wave; more chunks than that would leave a second, partly empty wave.
    static std::atomic<int> resident{0};  // per instantiation: one Op, one pair of kernels
    int per_sm = resident.load(std::memory_order_relaxed);
    if (per_sm == 0) {
        int r = 0, a = 0;
        DCX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_scan_reduce<T, Op>, SCAN_THREADS, 0));
        DCX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_scan_apply<T, Op>, SCAN_THREADS, 0));
        per_sm = std::max(1, std::min(r, a));
        resident.store(per_sm, std::memory_order_relaxed);
    }
    const uint64_t tpc = div_up(tiles, 148ull * per_sm);  // tiles per CTA
    const uint64_t chunks = div_up(tiles, tpc);
    DBuf<T> sums(&c, chunks + 1);
    k_scan_reduce<T, Op><<<(unsigned)chunks, SCAN_THREADS, 0, c.stream>>>(op, n, sums.get(), tpc);
    k_scan_tile_sums<T><<<1, 1024, 0, c.stream>>>(sums.get(), chunks, sums.get() + chunks);
    k_scan_apply<T, Op><<<(unsigned)chunks, SCAN_THREADS, 0, c.stream>>>(op, n, sums.get(), tpc);
    DCX_CHECK_LAUNCH();
    c.launched(3);
    return d2h_scalar(c, sums.get() + chunks);  // the grand total k_scan_tile_sums wrote
}

static const DcHost& get_dc(Ctx& c, uint32_t X) {
    auto it = c.dc_host.find(X);
    if (it != c.dc_host.end()) return it->second;
    DcHost h;
    if (!make_dc(X, h)) throw Error(DCX_ERR_ARG, "unsupported difference cover X=" + std::to_string(X));
    DcDev dd{};
    dd.X = X;
    dd.fx = make_fastdiv(X);
    dd.D = h.D;
    for (uint32_t i = 0; i < X; i++) dd.next_rank[i] = h.next_rank[i];
    for (uint32_t i = 0; i < h.D; i++) dd.dc[i] = h.dc[i];
    for (uint32_t i = 0; i < X; i++)
        for (uint32_t j = 0; j < X; j++) {
            const uint32_t* e = &h.cmp[((size_t)i * X + j) * 3];
            dd.cmp[i * X + j] = (uint16_t)(e[1] | (e[2] << 8));
        }
    DcDev* p = nullptr;
    DCX_CUDA(cudaMalloc(&p, sizeof(DcDev)));
    DCX_CUDA(cudaMemcpy(p, &dd, sizeof(DcDev), cudaMemcpyHostToDevice));
    c.dc_dev[X] = p;
    return c.dc_host.emplace(X, std::move(h)).first->second;
}

// ---------------------------------------------------------------------------
// Radix sort driver.  Keys/values in buffer 0, digit histograms of all 4*kw
// passes in c.d_hist.  Passes whose digit is constant are skipped.  Returns the
// index (0/1) of the buffer holding the sorted data.  With digit_shift >= 0 it
// runs the single pass on the 8-bit digit (key word 0 >> digit_shift) & 255,
// whose histogram is the first RADIX words of c.d_hist (digit_shift <= 24).
// ---------------------------------------------------------------------------
// Shift of the 8-bit digit that cuts [0, span) into 256 contiguous ranges (the
// two-step scatters group their stores by it).
static uint32_t top_digit_shift(uint64_t span) {
    uint32_t bits = 0;
    while (bits < 32 && ((span - 1) >> bits)) bits++;
    return bits > 8 ? bits - 8 : 0;
}

struct SortSpace {
    uint32_t* k[2][MAX_KEY_WORDS] = {};
    uint32_t* v[2] = {};
};

static int radix_sort(Ctx& c, uint32_t kw, uint64_t count, SortSpace& s, int digit_shift = -1) {
    if (kw > 3) throw Error(DCX_ERR_INTERNAL, "radix keys wider than 3 words");
    if (digit_shift > 24) throw Error(DCX_ERR_INTERNAL, "single-pass digit outside key word 0");
    const uint32_t passes = digit_shift >= 0 ? 1 : 4 * kw;
    // histograms in and digit bases out through pinned staging (PINNED_WORDS words each)
    uint32_t* h = reinterpret_cast<uint32_t*>(c.h_pinned);
    uint32_t* hb = h + PINNED_WORDS / 2;
    DCX_CUDA(cudaMemcpyAsync(h, c.d_hist, (size_t)passes * RADIX * 4, cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    std::vector<uint32_t> run;
    std::vector<uint32_t> bases;
    for (uint32_t p = 0; p < passes; p++) {
        const uint32_t* hp = &h[(size_t)p * RADIX];
        uint32_t mx = *std::max_element(hp, hp + RADIX);
        uint64_t sum = 0;
        for (int d = 0; d < RADIX; d++) sum += hp[d];
        // one digit value for all keys, or a digit the producer left uncounted
        // because it is zero in every key
        if ((uint64_t)mx == count || sum == 0) continue;
        run.push_back(digit_shift >= 0 ? (uint32_t)digit_shift : p * RADIX_BITS);
        uint32_t acc = 0;
        for (int d = 0; d < RADIX; d++) {
            bases.push_back(acc);
            acc += hp[d];
        }
    }
    if (run.empty()) return 0;
    const uint32_t items = c.opt.radix_items;
    const uint64_t tiles = div_up(count, (uint64_t)SORT_THREADS * items);
    if (tiles > c.lookback_tiles) {
        if (c.d_lookback) DCX_CUDA(cudaFree(c.d_lookback));
        c.d_lookback = nullptr;
        size_t want = std::max<size_t>(tiles, 1024);
        DCX_CUDA(cudaMalloc(&c.d_lookback, want * RADIX * sizeof(uint64_t)));
        DCX_CUDA(cudaMemset(c.d_lookback, 0, want * RADIX * sizeof(uint64_t)));
        c.lookback_tiles = want;
        c.epoch = 0;
    }
    std::copy(bases.begin(), bases.end(), hb);
    DCX_CUDA(cudaMemcpyAsync(c.d_base, hb, bases.size() * 4, cudaMemcpyHostToDevice, c.stream));
    DCX_CUDA(cudaMemsetAsync(c.d_tiles, 0, run.size() * 4, c.stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c.stream);
    int cur = 0;
    const size_t smem = onesweep_smem(kw, items);
    static std::atomic<bool> attr_set{false};  // the attribute is per function, the same for every context
    if (!attr_set.load()) {
        constexpr int I0 = ONESWEEP_ITEMS, I1 = ONESWEEP_ITEMS_ALT;
        DCX_CUDA(cudaFuncSetAttribute(k_onesweep<1, I0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem(1, I0)));
        DCX_CUDA(cudaFuncSetAttribute(k_onesweep<2, I0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem(2, I0)));
        DCX_CUDA(cudaFuncSetAttribute(k_onesweep<3, I0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem(3, I0)));
        DCX_CUDA(cudaFuncSetAttribute(k_onesweep<1, I1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem(1, I1)));
        DCX_CUDA(cudaFuncSetAttribute(k_onesweep<2, I1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem(2, I1)));
        DCX_CUDA(cudaFuncSetAttribute(k_onesweep<3, I1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem(3, I1)));
        attr_set.store(true);
    }
    // full tiles are staged with 16-byte copies: every buffer comes from the
    // context's allocator, which aligns to 256 bytes
    for (int b = 0; b < 2; b++) {
        for (uint32_t w = 0; w < kw; w++)
            if ((uintptr_t)s.k[b][w] & 15) throw Error(DCX_ERR_INTERNAL, "radix key buffer not 16-byte aligned");
        if ((uintptr_t)s.v[b] & 15) throw Error(DCX_ERR_INTERNAL, "radix value buffer not 16-byte aligned");
    }
    for (size_t i = 0; i < run.size(); i++) {
        if (++c.epoch >= (1u << 30)) {
            DCX_CUDA(cudaMemsetAsync(c.d_lookback, 0, c.lookback_tiles * RADIX * sizeof(uint64_t), c.stream));
            c.epoch = 1;
        }
        SortPassArgs a{};
        for (uint32_t w = 0; w < kw; w++) {
            a.keys_in[w] = s.k[cur][w];
            a.keys_out[w] = s.k[cur ^ 1][w];
        }
        a.vals_in = s.v[cur];
        a.vals_out = s.v[cur ^ 1];
        a.kw = kw;
        a.n = count;
        a.shift = run[i];
        a.digit_base = c.d_base + i * RADIX;
        a.lookback = c.d_lookback;
        a.tile_counter = c.d_tiles + i;
        a.epoch = c.epoch;
        a.err = c.d_err;
        a.spin_limit = c.opt.spin_limit;
        a.hold_tile = c.opt.lookback_hold_tile;
        a.gave_up = c.d_err + 1;
        if (items == ONESWEEP_ITEMS) {
            if (kw == 1) k_onesweep<1, ONESWEEP_ITEMS><<<(unsigned)tiles, SORT_THREADS, smem, c.stream>>>(a);
            else if (kw == 2) k_onesweep<2, ONESWEEP_ITEMS><<<(unsigned)tiles, SORT_THREADS, smem, c.stream>>>(a);
            else k_onesweep<3, ONESWEEP_ITEMS><<<(unsigned)tiles, SORT_THREADS, smem, c.stream>>>(a);
        } else {
            if (kw == 1) k_onesweep<1, ONESWEEP_ITEMS_ALT><<<(unsigned)tiles, SORT_THREADS, smem, c.stream>>>(a);
            else if (kw == 2) k_onesweep<2, ONESWEEP_ITEMS_ALT><<<(unsigned)tiles, SORT_THREADS, smem, c.stream>>>(a);
            else k_onesweep<3, ONESWEEP_ITEMS_ALT><<<(unsigned)tiles, SORT_THREADS, smem, c.stream>>>(a);
        }
        DCX_CHECK_LAUNCH();
        cur ^= 1;
    }
    cudaEventRecord(e1, c.stream);
    DCX_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // A look-back wait that gave up leaves the order wrong but every write in
    // range (the scatter checks its destinations); stop here with
    // DCX_ERR_TIMEOUT, before any kernel uses the sorted values as indices.
    check_device_error(c);
    c.st.ms_radix += ms;
    c.launched(run.size());
    c.st.radix_passes += run.size();
    c.st.radix_keys += run.size() * count;
    const uint64_t b = (uint64_t)run.size() * count * (kw + 1) * 4 * 2;
    c.st.bytes_radix += b;
    c.alg(b);
    return cur;
}

// ---------------------------------------------------------------------------
// Texts of one level (host view): text s occupies positions [start[s],
// start[s+1]-1) of the level buffer, followed by one 0 (its empty suffix).
// ---------------------------------------------------------------------------
struct Segs {
    std::vector<uint64_t> start;     // K + 1 entries, start[K] = N
    std::vector<uint64_t> out_base;  // level 0 only, optional [K]: first output entry of text s (default packed)
    uint32_t K() const { return (uint32_t)start.size() - 1; }
    uint64_t N() const { return start.back(); }
    uint64_t len(uint32_t s) const { return start[s + 1] - start[s] - 1; }
};

template <typename T>
static DBuf<T> upload(Ctx& c, const std::vector<T>& v) {
    DBuf<T> d(&c, std::max<size_t>(v.size(), 1));
    if (!v.empty()) DCX_CUDA(cudaMemcpyAsync(d.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c.stream));
    return d;
}

// Tie groups: maximal runs of the sorted order whose elements after the first
// have head 0, binned by size class (tie_class) into gstart/gsize.
struct TieGroups {
    bool complete = false;  // the groups hold every tie of the final head flags (tie break may split them)
    uint64_t G = 0;
    std::vector<uint32_t> counts;  // groups per class
    std::vector<uint64_t> off;     // first group of each class in gstart/gsize
    DBuf<uint32_t> gstart, gsize;
};

static TieGroups bin_groups(Ctx& c, uint64_t G, const uint32_t* starts, const uint32_t* ends);

static TieGroups group_ties_scan(Ctx& c, const uint8_t* head, uint64_t N) {
    DBuf<uint32_t> starts(&c, N / 2 + 1), ends(&c, N / 2 + 1);
    OpGroups op{head, N, starts.get(), ends.get()};
    const uint64_t tot = device_scan<uint64_t>(c, op, N);
    c.alg(N);
    return bin_groups(c, tot & 0xffffffffull, starts.get(), ends.get());
}

// Tie groups of all N head flags.  When few elements are tied (`tied`, the
// count of flags 0, below N/8) the groups are found by walking from each group
// start (k_groups_walk, one read of the flags), falling back to the scan when a
// group is longer than the walk's limit.  When most are tied, the scan: a walk
// per group then costs more than the scan, and the scan lists the groups in
// array order, which the group sorts that follow read with better locality.
static TieGroups group_ties(Ctx& c, const uint8_t* head, uint64_t N, uint64_t tied) {
    if (((uintptr_t)head & 15) != 0 || tied >= N / 8) return group_ties_scan(c, head, N);
    constexpr uint32_t WALK_LIMIT = 1u << 16;
    DBuf<uint32_t> starts(&c, N / 2 + 1), ends(&c, N / 2 + 1), cnt(&c, 2);
    DCX_CUDA(cudaMemsetAsync(cnt.get(), 0, 8, c.stream));
    k_groups_walk<<<grid_for(div_up(N, 16), 256, 148 * 8), 256, 0, c.stream>>>(N, head, WALK_LIMIT, starts.get(),
                                                                                ends.get(), cnt.get(), cnt.get() + 1);
    DCX_CHECK_LAUNCH();
    c.launched();
    c.alg(N + N / 8);
    uint32_t h[2];
    DCX_CUDA(cudaMemcpyAsync(h, cnt.get(), 8, cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    if (h[1]) return group_ties_scan(c, head, N);
    if (h[0] > N / 2 + 1) throw Error(DCX_ERR_INTERNAL, "more tie groups than the bound");
    return bin_groups(c, h[0], starts.get(), ends.get());
}

// Tie groups found inside parent groups that hold every tie (the round-0
// groups of the window sort): a walk over the parents' head flags instead of a
// scan of all N flags.
static TieGroups group_ties_within(Ctx& c, const uint8_t* head, const TieGroups& parents) {
    const uint64_t Gp = parents.G;
    uint64_t elems = 0;  // an upper bound on the sub-groups: half the parents' elements
    for (int k = 0; k < TIE_CLASSES - 1; k++) elems += (uint64_t)parents.counts[k] << (k + 1);
    const uint64_t cap = elems / 2 + 1;
    DBuf<uint32_t> starts(&c, cap), ends(&c, cap), cnt(&c, 1);
    DCX_CUDA(cudaMemsetAsync(cnt.get(), 0, 4, c.stream));
    if (Gp) {
        k_subgroups<<<grid_for(Gp, 256, 148 * 16), 256, 0, c.stream>>>(Gp, parents.gstart.get(), parents.gsize.get(),
                                                                       head, starts.get(), ends.get(), cnt.get());
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(elems + Gp * 8);
    }
    const uint32_t G = d2h_scalar(c, cnt.get());
    if (G > cap) throw Error(DCX_ERR_INTERNAL, "more tie groups than the bound");
    return bin_groups(c, G, starts.get(), ends.get());
}

// Tie groups (start, end) binned by size class into gstart/gsize.
static TieGroups bin_groups(Ctx& c, uint64_t G, const uint32_t* starts, const uint32_t* ends) {
    TieGroups tg;
    tg.G = G;
    tg.counts.assign(TIE_CLASSES, 0);
    tg.off.assign(TIE_CLASSES + 1, 0);
    if (tg.G == 0) return tg;
    DBuf<uint32_t> cnt(&c, 2 * TIE_CLASSES);
    DCX_CUDA(cudaMemsetAsync(cnt.get(), 0, 2 * TIE_CLASSES * 4, c.stream));
    k_tie_classify<<<grid_for(tg.G, 256), 256, 0, c.stream>>>(tg.G, starts, ends, cnt.get());
    DCX_CHECK_LAUNCH();
    DCX_CUDA(cudaMemcpyAsync(tg.counts.data(), cnt.get(), TIE_CLASSES * 4, cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    std::vector<uint32_t> cursor(TIE_CLASSES, 0);
    for (int k = 0; k < TIE_CLASSES; k++) {
        cursor[k] = (uint32_t)tg.off[k];
        tg.off[k + 1] = tg.off[k] + tg.counts[k];
    }
    DCX_CUDA(cudaMemcpyAsync(cnt.get() + TIE_CLASSES, cursor.data(), TIE_CLASSES * 4, cudaMemcpyHostToDevice, c.stream));
    tg.gstart = DBuf<uint32_t>(&c, tg.G);
    tg.gsize = DBuf<uint32_t>(&c, tg.G);
    k_tie_bin<<<grid_for(tg.G, 256), 256, 0, c.stream>>>(tg.G, starts, ends, cnt.get() + TIE_CLASSES,
                                                          tg.gstart.get(), tg.gsize.get());
    DCX_CHECK_LAUNCH();
    c.launched(2);
    return tg;
}

static RefinePlan8 make_refine8(uint64_t B, uint32_t P) {
    RefinePlan8 r8{};
    r8.P = P;
    r8.m = (P + 7) / 8;
    r8.r = P - 8 * (r8.m - 1);
    r8.B = B;
    r8.B2 = B * B;
    r8.B4 = r8.B2 * r8.B2;
    r8.pow8 = r8.B4 * r8.B4;  // only used when m > 1, i.e. B^8 < 2^64
    r8.powr = 1;
    for (uint32_t i = 0; i < r8.r; i++) r8.powr *= B;
    return r8;
}

template <int C, int T, int W, typename CharT>
static void launch_refine_seg(Ctx& c, const CharT* text, SegView sv, const uint32_t* segw, const uint32_t* gstart,
                              const uint32_t* gsize, uint64_t ng, uint32_t* sa, uint8_t* head,
                              const RefineSegPlan& plan) {
    const size_t shm = refine_seg_smem<C, W>();
    auto kern = k_refine_seg<C, T, W, CharT>;
    DCX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    int per_sm = 0;
    DCX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T, shm));
    const uint64_t grid = std::min<uint64_t>(ng, 148ull * std::max(per_sm, 1));
    kern<<<(unsigned)grid, T, shm, c.stream>>>(text, sv, segw, gstart, gsize, ng, sa, head, plan);
    DCX_CHECK_LAUNCH();
    c.launched();
}

// Groups of two (class 0) and of 3..32 (classes 1-4).
template <int W, typename CharT>
static void refine_small_w(Ctx& c, const CharT* text, SegView sv, const uint32_t* segw, const TieGroups& tg,
                           uint32_t* sa, uint8_t* head, const RefineSegPlan& plan) {
    if (tg.counts[0]) {
        k_refine_pair<W, CharT><<<grid_for(tg.counts[0], 256, 148 * 16), 256, 0, c.stream>>>(
            text, sv, segw, tg.gstart.get(), tg.counts[0], sa, head, plan);
        DCX_CHECK_LAUNCH();
        c.launched();
    }
    // classes 1..4 (3-4, 5-8, 9-16, 17-32 elements): 4, 8, 16 or 32 lanes per group
    auto sub = [&](int cls, auto lanes) {
        constexpr int LN = decltype(lanes)::value;
        const uint64_t g0 = tg.off[cls], ng = tg.counts[cls];
        if (!ng) return;
        k_refine_warp<W, LN, CharT><<<grid_for(ng * LN, 256, 148 * 16), 256, 0, c.stream>>>(
            text, sv, segw, tg.gstart.get() + g0, tg.gsize.get() + g0, ng, sa, head, plan);
        DCX_CHECK_LAUNCH();
        c.launched();
    };
    sub(1, std::integral_constant<int, 4>{});
    sub(2, std::integral_constant<int, 8>{});
    sub(3, std::integral_constant<int, 16>{});
    sub(4, std::integral_constant<int, 32>{});
}

// Groups of one size class (33-64, 65-128 or 129-256 elements: E = 2, 4, 8)
// refined by one window word, one warp per group.
template <int E, typename CharT>
static void refine_warp_class(Ctx& c, const CharT* text, SegView sv, const uint32_t* segw, const TieGroups& tg,
                              int cls, uint32_t* sa, uint8_t* head, const RefineSegPlan& plan) {
    const uint64_t ng = tg.counts[cls];
    if (!ng) return;
    auto kern = k_refine_warpsort<E, CharT>;
    int per_sm = 0;
    DCX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * WSORT_WARPS, 0));
    const uint64_t grid = std::min<uint64_t>(div_up(ng, WSORT_WARPS), 148ull * std::max(per_sm, 1));
    kern<<<(unsigned)grid, 32 * WSORT_WARPS, 0, c.stream>>>(text, sv, segw, tg.gstart.get() + tg.off[cls],
                                                            tg.gsize.get() + tg.off[cls], ng, sa, head, plan);
    DCX_CHECK_LAUNCH();
    c.launched();
}

template <int C, int T, typename CharT>
static void refine_seg_class(Ctx& c, const CharT* text, SegView sv, const uint32_t* segw, const TieGroups& tg,
                             int cls_lo, int cls_hi, uint32_t* sa, uint8_t* head, const RefineSegPlan& plan) {
    const uint64_t g0 = tg.off[cls_lo], ng = tg.off[cls_hi + 1] - g0;
    if (!ng) return;
    const uint32_t* gs = tg.gstart.get() + g0;
    const uint32_t* gz = tg.gsize.get() + g0;
    switch (plan.W) {
        case 1: launch_refine_seg<C, T, 1>(c, text, sv, segw, gs, gz, ng, sa, head, plan); break;
        case 2: launch_refine_seg<C, T, 2>(c, text, sv, segw, gs, gz, ng, sa, head, plan); break;
        case 3: launch_refine_seg<C, T, 3>(c, text, sv, segw, gs, gz, ng, sa, head, plan); break;
        case 4: launch_refine_seg<C, T, 4>(c, text, sv, segw, gs, gz, ng, sa, head, plan); break;
        case 5: launch_refine_seg<C, T, 5>(c, text, sv, segw, gs, gz, ng, sa, head, plan); break;
        default: launch_refine_seg<C, T, 6>(c, text, sv, segw, gs, gz, ng, sa, head, plan); break;
    }
}

// ---------------------------------------------------------------------------
// Phase 1: sort all N suffixes of the level by (text, first L chars).
// Produces the sorted positions `sa`, head flags (1 where the key differs from
// the previous one) and, for K > 1, the text id of every sorted element (segw).
// ---------------------------------------------------------------------------
template <typename CharT>
static void sort_windows(Ctx& c, const CharT* text, const Segs& sg, const uint64_t* d_start, uint64_t B, uint32_t L,
                         int depth, DBuf<uint32_t>& sa, DBuf<uint8_t>& head, DBuf<uint32_t>& segw,
                         TieGroups* parents) {
    const uint64_t N = sg.N();
    const uint32_t K = sg.K();
    const bool SEGK = K > 1;
    const SegView sv{K, d_start};
    const uint32_t words_full = (key_bits_k(B, L, K) + 31) / 32;
    uint32_t kw0_max = depth == 0 ? 2 : c.opt.rec_prefix_words;
    uint32_t P0 = std::min<uint32_t>(L, max_chars_in_bits_k(B, 32 * std::min(words_full, kw0_max), K));
    if (depth == 0 && c.level0_entropy > 0.05) {
        // Shortest byte-aligned prefix whose expected random collisions stay near
        // 1% of the longest text n: P * H >= log2(n) + 6, with H the order-0 entropy discounted by
        // 5% for context dependence.  Ties left over are resolved exactly by the
        // refinement rounds, so this only trades passes against refinement work.
        uint64_t longest = 1;  // windows of different texts never collide (text id digit)
        for (uint32_t t = 0; t < K; t++) longest = std::max<uint64_t>(longest, sg.len(t) + 1);
        const double need = std::log2((double)longest) + 6.0;
        uint32_t P = (uint32_t)std::ceil(need / (0.95 * c.level0_entropy));
        P = std::max<uint32_t>(1, std::min(P, P0));
        const uint32_t bytes = (key_bits_k(B, P, K) + 7) / 8;
        const uint32_t fill = std::min<uint32_t>(P0, max_chars_in_bits_k(B, 8 * bytes, K));
        P0 = std::max(P, fill);
    }
    if (c.opt.prefix_chars && depth == 0)  // forced prefix, within the 3 key words a sort takes
        P0 = std::min<uint32_t>({L, c.opt.prefix_chars, max_chars_in_bits_k(B, 96, K)});
    if (P0 == 0) P0 = 1;
    KeyPlan plan = make_plan(B, P0, K);  // key = text id * B^P0 + window
    if (plan.kw > 3) throw Error(DCX_ERR_INTERNAL, "prefix key wider than 3 words");
    const uint32_t kw = plan.kw;
    const uint32_t kwt = kw;

    // round 0
    unsigned long long round0_ties = 0;
    {
        DBuf<uint32_t> keys[2][3];
        DBuf<uint32_t> vals[2];
        SortSpace s;
        for (int b = 0; b < 2; b++) {
            for (uint32_t w = 0; w < kwt; w++) {
                keys[b][w] = DBuf<uint32_t>(&c, N);
                s.k[b][w] = keys[b][w].get();
            }
            vals[b] = DBuf<uint32_t>(&c, N);
            s.v[b] = vals[b].get();
        }
        DCX_CUDA(cudaMemsetAsync(c.d_hist, 0, 16 * RADIX * 4, c.stream));
        KeyOut ko{};
        for (uint32_t w = 0; w < kwt; w++) ko.w[w] = s.k[0][w];
        const int grid = grid_for(N, 256, 148 * 8);
        const size_t shm = (size_t)HIST_COPIES * 4 * kwt * RADIX * 4;
        if (kw <= 2 && P0 <= (uint32_t)SLIDE_MAX_CHARS) {
            // sliding-window builder: keys of consecutive positions share P-1 chars
            uint64_t pow_top = 1;
            for (uint32_t i = 1; i < P0; i++) pow_top *= B;
            const uint64_t seg_mul = pow_top * B;  // B^P0: weight of the text id digit
            const uint32_t nbytes = (key_bits_k(B, P0, K) + 7) / 8;  // digit bytes that can be nonzero
            const size_t sshm = keys_slide_smem<CharT>();
            const int sgrid = (int)std::min<uint64_t>(div_up(N, SLIDE_TILE), 148 * 3);  // 3 CTAs per SM by smem
            if (SEGK) {
                DCX_CUDA(cudaFuncSetAttribute(k_keys_slide<true, CharT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sshm));
                k_keys_slide<true, CharT><<<sgrid, SLIDE_THREADS, sshm, c.stream>>>(text, N, sv, plan, pow_top, seg_mul,
                                                                                    ko, s.v[0], c.d_hist, nbytes);
            } else {
                DCX_CUDA(cudaFuncSetAttribute(k_keys_slide<false, CharT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sshm));
                k_keys_slide<false, CharT><<<sgrid, SLIDE_THREADS, sshm, c.stream>>>(text, N, sv, plan, pow_top, seg_mul,
                                                                                     ko, s.v[0], c.d_hist, nbytes);
            }
        } else {
#define DCX_PREFIX(KWV, SEGV)                                                                                       \
    do {                                                                                                            \
        DCX_CUDA(cudaFuncSetAttribute(k_keys_prefix<KWV, SEGV, CharT>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                      64 << 10));                                                                   \
        k_keys_prefix<KWV, SEGV, CharT><<<grid, 256, shm, c.stream>>>(text, N, sv, plan, ko, s.v[0], c.d_hist);     \
    } while (0)
            if (kw == 1) { if (SEGK) DCX_PREFIX(1, true); else DCX_PREFIX(1, false); }
            else if (kw == 2) { if (SEGK) DCX_PREFIX(2, true); else DCX_PREFIX(2, false); }
            else { if (SEGK) DCX_PREFIX(3, true); else DCX_PREFIX(3, false); }
#undef DCX_PREFIX
        }
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(N * sizeof(CharT) + N * (kwt + 1) * 4);
        int f = radix_sort(c, kwt, N, s);
        KeyWords kk{};
        for (uint32_t w = 0; w < kwt; w++) kk.w[w] = s.k[f][w];
        head = DBuf<uint8_t>(&c, N);
        DCX_CUDA(cudaMemsetAsync(c.d_h256, 0, 8, c.stream));
        {
            const int hg = grid_for(std::max<uint64_t>(N / 16, 1), 256, 148 * 8);
            if (kwt == 1) k_heads16<1><<<hg, 256, 0, c.stream>>>(kk, N, head.get(), c.d_h256);
            else if (kwt == 2) k_heads16<2><<<hg, 256, 0, c.stream>>>(kk, N, head.get(), c.d_h256);
            else k_heads16<3><<<hg, 256, 0, c.stream>>>(kk, N, head.get(), c.d_h256);
        }
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(N * kwt * 4 + N);
        round0_ties = d2h_scalar(c, c.d_h256);
        sa = std::move(vals[f]);
        if (SEGK) {
            // the sort is text-major, so text s owns sorted slots [start[s], start[s+1])
            segw = DBuf<uint32_t>(&c, N);
            k_fill_segw<<<grid_for(div_up(N, FILL_TILE), 1, 148 * 8), 256, 0, c.stream>>>(sv, N, segw.get());
            DCX_CHECK_LAUNCH();
            c.launched();
            c.alg(N * 4);
        }
    }

    // refinement of tied windows (a group never spans two texts)
    uint32_t covered = round0_ties ? P0 : L;  // nothing tied: every window is already distinct
    uint8_t* hd = head.get();  // head flags the global rounds work on
    TieGroups tg;
    DBuf<uint8_t> head2;
    const bool seg_chars = sizeof(CharT) == 1 ? (B <= 256 && ((uintptr_t)text & 7) == 0) : true;
    if (covered < L && seg_chars && B <= 0xffffffffull) {
        // Groups of up to 2048 elements are sorted by the whole rest of the window
        // inside one CTA each; only larger groups take the global radix rounds.
        const uint32_t rem = L - covered;
        const uint32_t cpw = std::min<uint32_t>(sizeof(CharT) == 1 ? 64 : 16, max_chars_in_bits(B, 64));
        const uint32_t W = (rem + cpw - 1) / cpw;
        if (W <= (uint32_t)RSEG_MAX_W) {
            tg = group_ties(c, hd, N, round0_ties);
            RefineSegPlan plan{};
            plan.W = W;
            for (uint32_t w = 0; w < W; w++) {
                plan.off[w] = covered + w * cpw;
                plan.rp[w] = make_refine8(B, std::min(cpw, rem - w * cpw));
            }
            const CharT* t8 = text;
            const uint32_t* sw = SEGK ? segw.get() : nullptr;
            switch (W) {
                case 1: refine_small_w<1>(c, t8, sv, sw, tg, sa.get(), hd, plan); break;
                case 2: refine_small_w<2>(c, t8, sv, sw, tg, sa.get(), hd, plan); break;
                case 3: refine_small_w<3>(c, t8, sv, sw, tg, sa.get(), hd, plan); break;
                case 4: refine_small_w<4>(c, t8, sv, sw, tg, sa.get(), hd, plan); break;
                case 5: refine_small_w<5>(c, t8, sv, sw, tg, sa.get(), hd, plan); break;
                default: refine_small_w<6>(c, t8, sv, sw, tg, sa.get(), hd, plan); break;
            }
            if (W == 1) {  // one window word: one warp per group, elements in registers
                refine_warp_class<2>(c, t8, sv, sw, tg, 5, sa.get(), hd, plan);
                refine_warp_class<4>(c, t8, sv, sw, tg, 6, sa.get(), hd, plan);
                refine_warp_class<8>(c, t8, sv, sw, tg, 7, sa.get(), hd, plan);
            } else {
                refine_seg_class<64, 32>(c, t8, sv, sw, tg, 5, 5, sa.get(), hd, plan);
                refine_seg_class<256, 128>(c, t8, sv, sw, tg, 6, 7, sa.get(), hd, plan);
            }
            refine_seg_class<1024, 512>(c, t8, sv, sw, tg, 8, 9, sa.get(), hd, plan);
            refine_seg_class<2048, 512>(c, t8, sv, sw, tg, 10, 10, sa.get(), hd, plan);
            const uint64_t small = tg.off[TIE_CLASSES - 1];  // groups of at most 2048
            if (tg.counts[TIE_CLASSES - 1]) {
                // the global rounds see the small groups as resolved
                head2 = DBuf<uint8_t>(&c, N);
                DCX_CUDA(cudaMemcpyAsync(head2.get(), hd, N, cudaMemcpyDeviceToDevice, c.stream));
                k_group_flags<<<grid_for(small * 32, 256), 256, 0, c.stream>>>(tg.gstart.get(), tg.gsize.get(), small,
                                                                              head2.get(), nullptr);
                DCX_CHECK_LAUNCH();
                c.launched();
                hd = head2.get();
            } else {
                covered = L;
            }
        }
    }
    while (covered < L) {
        DBuf<uint32_t> slot(&c, N), grp(&c, N), tpos(&c, N), tseg;
        if (SEGK) tseg = DBuf<uint32_t>(&c, N);
        OpTied op{hd, N, sa.get(), SEGK ? segw.get() : nullptr, slot.get(), grp.get(), tpos.get(),
                  SEGK ? tseg.get() : nullptr};
        const uint64_t tot = device_scan<uint64_t>(c, op, N);
        c.alg(N + N / 2);
        const uint64_t cnt = tot >> 32;
        if (cnt == 0) break;
        const uint32_t Pr = std::min<uint32_t>(L - covered, max_chars_in(B, 2));
        KeyPlan rp = make_plan(B, Pr);
        const uint32_t kwr = rp.kw + 1;  // + group number
        DBuf<uint32_t> keys[2][3];
        DBuf<uint32_t> vals[2];
        SortSpace s;
        for (int b = 0; b < 2; b++) {
            for (uint32_t w = 0; w < kwr; w++) {
                keys[b][w] = DBuf<uint32_t>(&c, cnt);
                s.k[b][w] = keys[b][w].get();
            }
            vals[b] = DBuf<uint32_t>(&c, cnt);
            s.v[b] = vals[b].get();
        }
        DCX_CUDA(cudaMemsetAsync(c.d_hist, 0, 16 * RADIX * 4, c.stream));
        KeyOut ko{};
        for (uint32_t w = 0; w < kwr; w++) ko.w[w] = s.k[0][w];
        const int grid = grid_for(cnt, 256, 148 * 8);
        const size_t shm = (size_t)HIST_COPIES * 4 * kwr * RADIX * 4;
        const bool swar = sizeof(CharT) == 1 && B <= 256 && Pr <= 64 && ((uintptr_t)text & 7) == 0;
        if (swar) {
            // byte text: aligned word loads + SWAR digit folding
            const RefinePlan8 r8 = make_refine8(B, Pr);
            const uint8_t* t8 = reinterpret_cast<const uint8_t*>(text);
            DCX_CUDA(cudaFuncSetAttribute(k_keys_refine8<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 << 10));
            DCX_CUDA(cudaFuncSetAttribute(k_keys_refine8<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 << 10));
            if (rp.kw == 1)
                k_keys_refine8<1><<<grid, 256, shm, c.stream>>>(t8, sv, cnt, tpos.get(), SEGK ? tseg.get() : nullptr,
                                                                 grp.get(), covered, r8, ko, s.v[0], c.d_hist);
            else
                k_keys_refine8<2><<<grid, 256, shm, c.stream>>>(t8, sv, cnt, tpos.get(), SEGK ? tseg.get() : nullptr,
                                                                 grp.get(), covered, r8, ko, s.v[0], c.d_hist);
        } else {
        DCX_CUDA(cudaFuncSetAttribute(k_keys_refine<1, CharT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 << 10));
        DCX_CUDA(cudaFuncSetAttribute(k_keys_refine<2, CharT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 << 10));
        if (rp.kw == 1)
            k_keys_refine<1, CharT><<<grid, 256, shm, c.stream>>>(text, sv, cnt, tpos.get(), SEGK ? tseg.get() : nullptr,
                                                                  grp.get(), covered, rp, ko, s.v[0], c.d_hist);
        else
            k_keys_refine<2, CharT><<<grid, 256, shm, c.stream>>>(text, sv, cnt, tpos.get(), SEGK ? tseg.get() : nullptr,
                                                                  grp.get(), covered, rp, ko, s.v[0], c.d_hist);
        }
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(cnt * (12 + Pr * sizeof(CharT)) + cnt * (kwr + 1) * 4);
        int f = radix_sort(c, kwr, cnt, s);
        KeyWords kk{};
        for (uint32_t w = 0; w < kwr; w++) kk.w[w] = s.k[f][w];
        k_refine_scatter<<<grid_for(cnt, 256), 256, 0, c.stream>>>(cnt, slot.get(), kk, kwr, s.v[f], sa.get(), hd);
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(cnt * (4 + kwr * 4 * 2 + 4 + 4 + 1));
        covered += Pr;
    }
    if (hd != head.get()) {  // big groups' flags back into the real head array
        const uint64_t g0 = tg.off[TIE_CLASSES - 1], nbig = tg.counts[TIE_CLASSES - 1];
        k_group_flags<<<grid_for(nbig * 32, 256), 256, 0, c.stream>>>(tg.gstart.get() + g0, tg.gsize.get() + g0, nbig,
                                                                     head.get(), hd);
        DCX_CHECK_LAUNCH();
        c.launched();
    }
    // The round-0 groups hold every tie that is left: the tie break looks for its
    // groups inside them instead of scanning all N head flags again.
    if (parents) {
        if (!round0_ties) {
            parents->complete = true;
            parents->G = 0;
            parents->counts.assign(TIE_CLASSES, 0);
            parents->off.assign(TIE_CLASSES + 1, 0);
        } else if (!tg.counts.empty() && tg.counts[TIE_CLASSES - 1] == 0) {
            *parents = std::move(tg);
            parents->complete = true;
        }
    }
}

// ---------------------------------------------------------------------------
// Phase 4: order every tie group (equal text and L-char window) by cover ranks.
// ---------------------------------------------------------------------------
template <int D>
static void tie_break_d(Ctx& c, uint32_t* sa, uint64_t N, const uint32_t* rank_text, const DcDev* dcd, TieSeg ts,
                        const std::vector<uint32_t>& counts, const uint32_t* gstart, const uint32_t* gsize,
                        uint32_t X) {
    std::vector<uint64_t> off(TIE_CLASSES + 1, 0);
    for (int k = 0; k < TIE_CLASSES; k++) off[k + 1] = off[k] + counts[k];
    auto warp_launch = [&](int cls, auto W) {
        constexpr int Wv = decltype(W)::value;
        const uint64_t g = counts[cls];
        if (!g) return;
        const uint64_t warps = div_up(g, 32 / Wv);
        const uint64_t blocks = div_up(warps * 32, 256);
        k_tie_warp<D, Wv><<<(unsigned)blocks, 256, tie_tab_smem(X), c.stream>>>(gstart + off[cls], gsize + off[cls], (uint32_t)g,
                                                                  sa, rank_text, dcd, ts);
        DCX_CHECK_LAUNCH();
        c.launched();
    };
    if (counts[0]) {  // pairs
        k_tie_pair<<<grid_for(counts[0], 256, 148 * 16), 256, tie_tab_smem(X), c.stream>>>(gstart + off[0], counts[0], sa, rank_text,
                                                                           dcd, ts);
        DCX_CHECK_LAUNCH();
        c.launched();
    }
    warp_launch(1, std::integral_constant<int, 4>{});
    warp_launch(2, std::integral_constant<int, 8>{});
    warp_launch(3, std::integral_constant<int, 16>{});
    warp_launch(4, std::integral_constant<int, 32>{});
    auto cta_launch = [&](const uint32_t* gs, const uint32_t* gz, uint64_t g, auto Cc) {
        constexpr int C = decltype(Cc)::value;
        constexpr int T = C / 2 < 512 ? C / 2 : 512;
        if (!g) return;
        const size_t shm = tie_cta_smem<D, C>(X);
        DCX_CUDA(cudaFuncSetAttribute(k_tie_cta<D, C, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        int per_sm = 0;  // CTAs that fit one SM: the grid loops over the groups
        DCX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tie_cta<D, C, T>, T, shm));
        const uint64_t grid = std::min<uint64_t>(g, 148ull * std::max(per_sm, 1));
        k_tie_cta<D, C, T><<<(unsigned)grid, T, shm, c.stream>>>(gs, gz, g, sa, rank_text, dcd, ts);
        DCX_CHECK_LAUNCH();
        c.launched();
    };
    // 33-64, 65-128, 129-256 elements: one warp per group
    auto warpsort_launch = [&](int cls, auto Ec) {
        constexpr int E = decltype(Ec)::value;
        const uint64_t g = counts[cls];
        if (!g) return;
        const size_t shm = tie_warpsort_smem<D, E>(X);
        DCX_CUDA(cudaFuncSetAttribute(k_tie_warpsort<D, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        int per_sm = 0;
        DCX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tie_warpsort<D, E>, 32 * WSORT_WARPS, shm));
        const uint64_t grid = std::min<uint64_t>(div_up(g, WSORT_WARPS), 148ull * std::max(per_sm, 1));
        k_tie_warpsort<D, E><<<(unsigned)grid, 32 * WSORT_WARPS, shm, c.stream>>>(gstart + off[cls], gsize + off[cls], g,
                                                                                sa, rank_text, dcd, ts);
        DCX_CHECK_LAUNCH();
        c.launched();
    };
    warpsort_launch(5, std::integral_constant<int, 2>{});
    warpsort_launch(6, std::integral_constant<int, 4>{});
    warpsort_launch(7, std::integral_constant<int, 8>{});
    cta_launch(gstart + off[8], gsize + off[8], counts[8], std::integral_constant<int, 512>{});
    cta_launch(gstart + off[9], gsize + off[9], counts[9], std::integral_constant<int, 1024>{});
    cta_launch(gstart + off[10], gsize + off[10], counts[10], std::integral_constant<int, 2048>{});
    const uint64_t nbig = counts[11];
    if (!nbig) return;
    // big groups: sort 2048-chunks, then merge rounds
    std::vector<uint32_t> bstart(nbig), bsize(nbig);
    DCX_CUDA(cudaMemcpyAsync(bstart.data(), gstart + off[11], nbig * 4, cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaMemcpyAsync(bsize.data(), gsize + off[11], nbig * 4, cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    std::vector<uint32_t> cstart, csize;
    std::vector<uint64_t> offs(nbig + 1, 0);
    uint32_t maxsz = 0;
    for (uint64_t g = 0; g < nbig; g++) {
        for (uint32_t o = 0; o < bsize[g]; o += 2048) {
            cstart.push_back(bstart[g] + o);
            csize.push_back(std::min<uint32_t>(2048, bsize[g] - o));
        }
        offs[g + 1] = offs[g] + bsize[g];
        maxsz = std::max(maxsz, bsize[g]);
    }
    DBuf<uint32_t> dcs = upload(c, cstart), dcz = upload(c, csize), dbs = upload(c, bstart);
    DBuf<uint64_t> doff = upload(c, offs);
    cta_launch(dcs.get(), dcz.get(), cstart.size(), std::integral_constant<int, 2048>{});
    DBuf<uint32_t> tmp(&c, N);
    uint32_t* src = sa;
    uint32_t* dst = tmp.get();
    const uint64_t total = offs[nbig];
    for (uint64_t w = 2048; w < maxsz; w <<= 1) {
        k_tie_merge<D><<<grid_for(total, 256), 256, 0, c.stream>>>(doff.get(), (uint32_t)nbig, dbs.get(), total,
                                                                   (uint32_t)w, src, dst, rank_text, dcd, ts);
        DCX_CHECK_LAUNCH();
        c.launched();
        std::swap(src, dst);
    }
    if (src != sa) {
        k_copy_ranges<<<grid_for(total, 256), 256, 0, c.stream>>>(doff.get(), (uint32_t)nbig, dbs.get(), total, src, sa);
        DCX_CHECK_LAUNCH();
        c.launched();
    }
    DCX_CUDA(cudaStreamSynchronize(c.stream));
}

static void tie_break(Ctx& c, uint32_t* sa, const uint8_t* head, uint64_t N, const uint32_t* rank_text,
                      const DcHost& dc, TieSeg ts, const TieGroups* parents) {
    TieGroups tg = parents ? group_ties_within(c, head, *parents) : group_ties_scan(c, head, N);
    const uint64_t G = tg.G;
    if (G == 0) return;
    const std::vector<uint32_t>& counts = tg.counts;
    DBuf<uint32_t>& gstart = tg.gstart;
    DBuf<uint32_t>& gsize = tg.gsize;
    const DcDev* dcd = c.dc_dev[dc.X];
    switch (dc.D) {
#define DCX_TIE(DV) \
    case DV: tie_break_d<DV>(c, sa, N, rank_text, dcd, ts, counts, gstart.get(), gsize.get(), dc.X); break;
        DCX_TIE(2) DCX_TIE(3) DCX_TIE(4) DCX_TIE(5) DCX_TIE(6) DCX_TIE(7) DCX_TIE(8) DCX_TIE(9) DCX_TIE(10)
        DCX_TIE(11) DCX_TIE(12)
#undef DCX_TIE
        default: throw Error(DCX_ERR_INTERNAL, "unsupported D");
    }
    c.st.tie_groups += G;
}

// ---------------------------------------------------------------------------
// One DCX level over K texts.
// ---------------------------------------------------------------------------
template <typename CharT>
static void level(Ctx& c, const CharT* text, const Segs& sg, uint64_t sigma, uint32_t X, int depth, bool packing,
                  void* sa_out, int out_width = 32);

// In-CTA base case for K texts of at most SMALL_MAX chars each (one launch).
static void small_sa_batch(Ctx& c, const void* text, bool wide, const Segs& sg, void* out, int out_width) {
    const uint32_t K = sg.K();
    std::vector<uint64_t> obase(K + 1, 0);
    for (uint32_t s = 0; s < K; s++) obase[s + 1] = obase[s] + sg.len(s);
    if (!sg.out_base.empty()) std::copy(sg.out_base.begin(), sg.out_base.end(), obase.begin());
    DBuf<uint64_t> dst = upload(c, sg.start), dob = upload(c, obase);
    for (uint32_t b = 0; b < K; b += 65535) {
        const uint32_t nb = std::min<uint32_t>(K - b, 65535);
        if (wide)
            k_small_sa<uint32_t><<<nb, SMALL_THREADS, 0, c.stream>>>((const uint32_t*)text, dst.get() + b, dob.get() + b,
                                                                      out, out_width);
        else
            k_small_sa<uint8_t><<<nb, SMALL_THREADS, 0, c.stream>>>((const uint8_t*)text, dst.get() + b, dob.get() + b,
                                                                     out, out_width);
        DCX_CHECK_LAUNCH();
        c.launched();
    }
    DCX_CUDA(cudaStreamSynchronize(c.stream));
}

static uint32_t level0_sample_chars(uint32_t X, uint64_t sigma, bool packing) {
    if (!packing) return X;
    // cli.cpp:488-533: 3 bits if sigma <= 7, 5 if <= 31, else 8; K = ceil(X / chars_per_word);
    // the sample window is X * (K*cpw/X) chars computed in double (sample_string.hpp:131-133).
    const uint32_t bits = sigma <= 7 ? 3 : (sigma <= 31 ? 5 : 8);
    const uint32_t cpw = 64 / bits;
    const uint32_t K = (X + cpw - 1) / cpw;
    const double ratio = (double)(K * cpw) / X;
    return (uint32_t)(X * ratio);
}

template <typename CharT>
static void level(Ctx& c, const CharT* text, const Segs& sg, uint64_t sigma, uint32_t X, int depth, bool packing,
                  void* sa_out, int out_width) {
    const uint32_t K = sg.K();
    const uint64_t N = sg.N();
    if (N <= K) return;  // only empty texts
    if (depth > 64) throw Error(DCX_ERR_INTERNAL, "recursion deeper than 64 levels");
    c.st.levels = std::max<uint32_t>(c.st.levels, (uint32_t)depth + 1);
    {
        uint64_t maxlen = 0;
        for (uint32_t s = 0; s < K; s++) maxlen = std::max(maxlen, sg.len(s));
        if (maxlen <= c.opt.small_threshold && maxlen <= (uint64_t)SMALL_MAX) {
            small_sa_batch(c, text, sizeof(CharT) == 4, sg, sa_out, out_width);
            return;
        }
    }
    const DcHost& dc = get_dc(c, X);
    const uint32_t D = dc.D;
    const uint32_t L = depth == 0 ? level0_sample_chars(X, sigma, packing) : X;
    const uint64_t B = sigma + 1;

    // ---- phase 0: per-text lengths, samples, slot bases (pdcx.hpp:473-510)
    std::vector<uint64_t> m_s(K), rbase(K + 1, 0), qbase(K + 1, 0), obase(K + 1, 0), sbt((size_t)K * (D + 1), 0);
    std::vector<uint64_t> num_at_mod(X);
    for (uint32_t s = 0; s < K; s++) {
        const uint64_t n = sg.len(s);
        const uint64_t rem = n % X;
        const bool dummy = dc.in_dc[rem] != 0;
        uint64_t m = (n / X) * D;
        for (uint64_t r = 0; r < rem; r++) m += dc.in_dc[r];
        m += dummy;
        m_s[s] = m;
        for (uint64_t i = 0; i < X; i++) num_at_mod[i] = (n + X - 1 - i) / X;
        num_at_mod[rem] += dummy;
        uint64_t* sb = &sbt[(size_t)s * (D + 1)];
        for (uint32_t i = 1; i <= D; i++) sb[i] = sb[i - 1] + num_at_mod[dc.dc[i - 1]];
        rbase[s + 1] = rbase[s] + m + D;
        qbase[s + 1] = qbase[s] + m;
        obase[s + 1] = obase[s] + n;
    }
    if (!sg.out_base.empty()) std::copy(sg.out_base.begin(), sg.out_base.end(), obase.begin());
    const uint64_t m = qbase[K];
    const uint64_t slots = rbase[K];
    if (m >= (1ull << 31)) throw Error(DCX_ERR_ARG, "more than 2^31 samples in one level");
    DcFlags fl{};
    fl.X = X;
    fl.D = D;
    fl.fx = make_fastdiv(X);
    for (uint32_t i = 0; i < X; i++) {
        fl.in_dc[i] = dc.in_dc[i];
        fl.next_rank[i] = dc.next_rank[i];
    }
    for (uint32_t i = 0; i < D; i++) fl.dc[i] = dc.dc[i];
    DBuf<DcFlags> dfl(&c, 1);
    DCX_CUDA(cudaMemcpyAsync(dfl.get(), &fl, sizeof(fl), cudaMemcpyHostToDevice, c.stream));
    DBuf<uint64_t> d_start = upload(c, sg.start), d_rbase = upload(c, rbase), d_qbase = upload(c, qbase),
                   d_obase = upload(c, obase), d_sb = upload(c, sbt);
    DBuf<uint8_t> d_mode(&c, K);
    DBuf<uint64_t> d_kbase(&c, K + 1), d_start2(&c, K);
    LevelSeg ls{K, d_start.get(), d_rbase.get(), d_qbase.get(), d_sb.get(), d_obase.get(), d_mode.get(),
                d_kbase.get(), d_start2.get()};

    cudaEvent_t ev[5];
    for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], c.stream);

    // ---- phase 1: window sort
    DBuf<uint32_t> sa, segw;
    DBuf<uint8_t> head;
    TieGroups parents;  // round-0 tie groups, kept for the tie break
    sort_windows<CharT>(c, text, sg, d_start.get(), B, L, depth, sa, head, segw, &parents);
    const uint32_t* segw_p = K > 1 ? segw.get() : nullptr;

    // ---- phase 2: names
    DBuf<uint32_t> s_pos(&c, m), s_seg, s_grp(&c, m);
    if (K > 1) s_seg = DBuf<uint32_t>(&c, m);  // one text: every sample's text is 0
    {
        OpSamples op{head.get(), sa.get(), segw_p, dfl.get(), ls, s_pos.get(), s_seg.get(), s_grp.get(), m};
        const uint64_t tot = device_scan<uint64_t>(c, op, N);
        c.alg(N * 5 + m * 12);
        if ((tot >> 32) != m) throw Error(DCX_ERR_INTERNAL, "sample count mismatch");
    }
    DBuf<uint32_t> name(&c, m);
    DBuf<uint8_t> uniq(&c, m);
    {
        OpNames op{s_grp.get(), m, name.get(), uniq.get()};
        device_scan<uint32_t>(c, op, m);
        c.alg(m * 9);
    }
    s_grp.reset();
    const uint32_t last_rank = d2h_scalar(c, name.get() + (m - 1));
    // sample records in sample text order (one random scatter)
    DBuf<uint64_t> srec(&c, slots);
    DCX_CUDA(cudaMemsetAsync(srec.get(), 0xff, slots * 8, c.stream));
    if (slots <= (1u << 20)) {  // 8 MB of records: a direct scatter stays in L2
        k_scatter_samples<<<grid_for(m, 256), 256, 0, c.stream>>>(m, s_pos.get(), s_seg.get(), name.get(), uniq.get(),
                                                                 dfl.get(), ls, srec.get());
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(m * 21);
    } else {
        // group the records by the top 8 bits of their slot first
        const uint32_t shift = top_digit_shift(slots);
        SortSpace s;
        DBuf<uint32_t> rk[2][2], rv[2];
        for (int b = 0; b < 2; b++) {
            for (int w = 0; w < 2; w++) {
                rk[b][w] = DBuf<uint32_t>(&c, m);
                s.k[b][w] = rk[b][w].get();
            }
            rv[b] = DBuf<uint32_t>(&c, m);
            s.v[b] = rv[b].get();
        }
        DCX_CUDA(cudaMemsetAsync(c.d_hist, 0, 16 * RADIX * 4, c.stream));
        k_sample_records<<<grid_for(m, 256, 148 * 8), 256, 0, c.stream>>>(m, s_pos.get(), s_seg.get(), name.get(),
                                                                          uniq.get(), dfl.get(), ls, s.k[0][0],
                                                                          s.k[0][1], s.v[0], c.d_hist, shift);
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(m * 21);
        const int f = radix_sort(c, 2, m, s, (int)shift);
        // one record per thread (see build_phi)
        k_scatter_records<<<(unsigned)div_up(m, 256), 256, 0, c.stream>>>(m, s.k[f][0], s.k[f][1], s.v[f],
                                                                           srec.get());
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(m * 20);
    }
    s_pos.reset();
    s_seg.reset();
    uniq.reset();
    if (depth == 0) {
        c.st.level0_samples = m;
        c.st.level0_last_rank = last_rank;
        c.st.level0_recursion = 0;
        c.st.level0_reduction = 0;
        if (c.opt.trace && K == 1) {
            DBuf<uint32_t> tn(&c, slots);
            DBuf<uint8_t> tu(&c, slots);
            k_ranks_from_names<<<grid_for(slots, 256), 256, 0, c.stream>>>(slots, srec.get(), nullptr, tn.get(), tu.get());
            DCX_CHECK_LAUNCH();
            c.trace_names.resize(m);
            c.trace_uniq.resize(m);
            DCX_CUDA(cudaMemcpyAsync(c.trace_names.data(), tn.get(), m * 4, cudaMemcpyDeviceToHost, c.stream));
            DCX_CUDA(cudaMemcpyAsync(c.trace_uniq.data(), tu.get(), m, cudaMemcpyDeviceToHost, c.stream));
            DCX_CUDA(cudaStreamSynchronize(c.stream));
        }
    }
    cudaEventRecord(ev[1], c.stream);

    // ---- phase 3: ranks of the samples in sample text order (D zero slots per text)
    DBuf<uint32_t> rank_text(&c, slots);
    DCX_CUDA(cudaMemsetAsync(rank_text.get(), 0, slots * 4, c.stream));
    if (last_rank >= m) {  // every text's names are distinct (pdcx.hpp:743-757)
        name.reset();
        k_ranks_from_names<<<grid_for(slots, 256), 256, 0, c.stream>>>(slots, srec.get(), rank_text.get(), nullptr, nullptr);
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(slots * 12);
    } else {
        const uint32_t Xr = c.opt.recursion_dc ? c.opt.recursion_dc : X;
        DBuf<uint32_t> rec(&c, m), kidx(&c, m);
        DBuf<uint8_t> rec_flag(&c, m);
        k_rec_from_slots<<<(unsigned)div_up(slots, 256), 256, 0, c.stream>>>(slots, srec.get(), dfl.get(), ls,
                                                                            rec.get(), rec_flag.get());
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(slots * 8 + m * 5);
        // per-text discarding counts (num_ranks_after_discarding, pdcx.hpp:215-228)
        const uint32_t kept_total = device_scan<uint32_t>(c, OpKeepCount{rec_flag.get(), kidx.get()}, m);
        c.alg(m * 6);
        std::vector<uint32_t> kb(K + 1);
        {
            DBuf<uint32_t> dkb(&c, K + 1);
            k_gather_u32<<<grid_for(K + 1, 256), 256, 0, c.stream>>>(kidx.get(), d_qbase.get(), K + 1, m, kept_total,
                                                                    dkb.get());
            DCX_CHECK_LAUNCH();
            DCX_CUDA(cudaMemcpyAsync(kb.data(), dkb.get(), (K + 1) * 4, cudaMemcpyDeviceToHost, c.stream));
            DCX_CUDA(cudaStreamSynchronize(c.stream));
        }
        // per text: recursion iff some name repeats (then more than the first element is
        // kept); discarding iff the reduction <= threshold (pdcx.hpp:150-165)
        std::vector<uint8_t> mode(K);
        std::vector<uint64_t> kbase(K + 1, 0), start2(K, 0);
        std::vector<uint64_t> rec_start(1, 0);
        std::vector<uint32_t> rec_text;
        uint64_t pos2 = 0;
        for (uint32_t s = 0; s < K; s++) {
            const uint64_t cnt = kb[s + 1] - kb[s];
            uint64_t kept = 0;
            if (cnt >= 2) {
                const double reduction = (double)cnt / (double)m_s[s];
                const bool discard = reduction <= c.opt.discarding_threshold;
                mode[s] = discard ? REC_DISCARD : REC_DIRECT;
                kept = discard ? cnt : m_s[s];
                if (depth == 0 && K == 1) {
                    c.st.level0_recursion = discard ? 2 : 1;
                    c.st.level0_reduction = reduction;
                }
            } else {
                mode[s] = REC_NONE;
            }
            kbase[s + 1] = kbase[s] + kept;
            if (kept) {
                start2[s] = pos2;
                pos2 += kept + 1;
                rec_start.push_back(pos2);
                rec_text.push_back(s);
            }
        }
        DCX_CUDA(cudaMemcpyAsync(d_mode.get(), mode.data(), K, cudaMemcpyHostToDevice, c.stream));
        DCX_CUDA(cudaMemcpyAsync(d_kbase.get(), kbase.data(), (K + 1) * 8, cudaMemcpyHostToDevice, c.stream));
        DCX_CUDA(cudaMemcpyAsync(d_start2.get(), start2.data(), K * 8, cudaMemcpyHostToDevice, c.stream));
        const uint32_t R = (uint32_t)rec_text.size();
        const uint64_t total2 = kbase[K];
        bool any_discard = false;
        for (uint32_t s = 0; s < K; s++) any_discard |= mode[s] == REC_DISCARD;
        if (R > 0) {
            // recursion input: the kept names of every recursing text, each followed by a 0
            DBuf<uint32_t> rec2(&c, pos2);
            DCX_CUDA(cudaMemsetAsync(rec2.get(), 0, pos2 * 4, c.stream));
            if (K == 1) {
                // one text: the kept indices are q itself (direct) or the keep-count
                // prefix already in kidx (discarding), so an elementwise copy compacts
                k_compact_one<<<grid_for(m, 256), 256, 0, c.stream>>>(m, rec_flag.get(), rec.get(), mode[0],
                                                                       start2[0], rec2.get(), kidx.get());
                DCX_CHECK_LAUNCH();
                c.launched();
                c.alg(m * 9 + total2 * 4);
            } else {
                device_scan<uint32_t>(c, OpCompact{rec_flag.get(), rec.get(), ls, rec2.get(), kidx.get()}, m);
                c.alg(m * 10 + total2 * 4);
            }
            rec.reset();
            rec_flag.reset();
            Segs sg2;
            sg2.start = rec_start;
            DBuf<uint32_t> sa2(&c, total2);
            level<uint32_t>(c, rec2.get(), sg2, last_rank, Xr, depth + 1, false, sa2.get(), 32);
            rec2.reset();
            std::vector<uint64_t> o2(R + 1, 0);
            for (uint32_t r = 0; r < R; r++) o2[r + 1] = o2[r] + sg2.len(r);
            DBuf<uint64_t> d_o2 = upload(c, o2);
            DBuf<uint32_t> d_rt = upload(c, rec_text);
            DBuf<uint32_t> rank_of;
            if (any_discard) rank_of = DBuf<uint32_t>(&c, total2);
            if (total2 <= (1u << 20)) {  // 4 MB of ranks: a direct scatter stays in L2
                k_after_recursion<<<grid_for(total2, 256), 256, 0, c.stream>>>(total2, sa2.get(), d_o2.get(), R,
                                                                               d_rt.get(), dfl.get(), ls,
                                                                               rank_text.get(),
                                                                               any_discard ? rank_of.get() : nullptr);
                DCX_CHECK_LAUNCH();
                c.launched();
                c.alg(total2 * 12);
            } else {
                // group the rank stores by the top 8 bits of their destination first
                const uint32_t shift = top_digit_shift(std::max<uint64_t>(slots, any_discard ? total2 : 0));
                SortSpace s;
                DBuf<uint32_t> rk1(&c, total2), rv0(&c, total2), rv1(&c, total2);
                s.k[0][0] = sa2.get();  // the records overwrite sa2 in place, element by element
                s.k[1][0] = rk1.get();
                s.v[0] = rv0.get();
                s.v[1] = rv1.get();
                DCX_CUDA(cudaMemsetAsync(c.d_hist, 0, 16 * RADIX * 4, c.stream));
                k_after_records<<<grid_for(total2, 256, 148 * 8), 256, 0, c.stream>>>(
                    total2, sa2.get(), d_o2.get(), R, d_rt.get(), dfl.get(), ls, s.k[0][0], s.v[0], c.d_hist, shift);
                DCX_CHECK_LAUNCH();
                c.launched();
                c.alg(total2 * 12);
                const int f = radix_sort(c, 1, total2, s, (int)shift);
                // one record per thread (see build_phi)
                k_scatter_ranks<<<(unsigned)div_up(total2, 256), 256, 0, c.stream>>>(
                    total2, s.k[f][0], s.v[f], rank_text.get(), any_discard ? rank_of.get() : nullptr);
                DCX_CHECK_LAUNCH();
                c.launched();
                c.alg(total2 * 12);
            }
            sa2.reset();
            if (any_discard) {
                // non-unique samples of discarding texts: sort by (name, rank2) (pdcx.hpp:296-346).
                // One scan compacts them into first buffers sized for every sample
                // (their count is not known before it); the second buffers get the count.
                DBuf<uint32_t> keys[2][2];
                DBuf<uint32_t> vals[2];
                SortSpace s;
                for (int w = 0; w < 2; w++) {
                    keys[0][w] = DBuf<uint32_t>(&c, m);
                    s.k[0][w] = keys[0][w].get();
                }
                vals[0] = DBuf<uint32_t>(&c, m);
                s.v[0] = vals[0].get();
                const uint32_t mu = device_scan<uint32_t>(c, OpNonUniqueSeg{srec.get(), dfl.get(), ls, kidx.get(),
                                                                          rank_of.get(), s.k[0][0], s.k[0][1],
                                                                          s.v[0]},
                                                          slots);
                if (mu > m) throw Error(DCX_ERR_INTERNAL, "more non-unique samples than samples");
                if (mu) {
                    for (int w = 0; w < 2; w++) {
                        keys[1][w] = DBuf<uint32_t>(&c, mu);
                        s.k[1][w] = keys[1][w].get();
                    }
                    vals[1] = DBuf<uint32_t>(&c, mu);
                    s.v[1] = vals[1].get();
                    c.alg(slots * 9 + mu * 12);
                    rank_of.reset();
                    kidx.reset();
                    DCX_CUDA(cudaMemsetAsync(c.d_hist, 0, 16 * RADIX * 4, c.stream));
                    SortPassArgs ha{};
                    ha.keys_in[0] = s.k[0][0];
                    ha.keys_in[1] = s.k[0][1];
                    ha.kw = 2;
                    ha.n = mu;
                    k_digit_hist<<<grid_for(mu, 256, 148 * 4), 256, 8 * RADIX * 4, c.stream>>>(ha, c.d_hist);
                    DCX_CHECK_LAUNCH();
                    c.launched();
                    c.alg(mu * 8);
                    int f = radix_sort(c, 2, mu, s);
                    DBuf<uint32_t> start_s(&c, (uint64_t)last_rank + 1), start_l(&c, (uint64_t)last_rank + 1);
                    k_name_starts<<<grid_for(m, 256), 256, 0, c.stream>>>(m, name.get(), start_s.get());
                    k_name_starts<<<grid_for(mu, 256), 256, 0, c.stream>>>(mu, s.k[f][1], start_l.get());
                    k_ranks_nonunique<<<grid_for(mu, 256), 256, 0, c.stream>>>(mu, s.k[f][1], s.v[f], start_s.get(),
                                                                              start_l.get(), rank_text.get());
                    DCX_CHECK_LAUNCH();
                    c.launched(3);
                    c.alg(m * 8 + mu * 8 + mu * 24);
                }
            }
        }
        // texts without recursion keep their names; unique samples of discarding texts their order
        k_ranks_rest<<<grid_for(slots, 256), 256, 0, c.stream>>>(slots, srec.get(), ls, rank_text.get());
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(slots * 12);
    }
    srec.reset();
    name.reset();
    cudaEventRecord(ev[2], c.stream);

    // ---- phase 4: tie groups, then emit
    tie_break(c, sa.get(), head.get(), N, rank_text.get(), dc, TieSeg{segw_p, d_start.get(), d_rbase.get()},
              parents.complete ? &parents : nullptr);
    parents = TieGroups{};
    head.reset();
    rank_text.reset();
    if (K == 1 && sg.out_base.empty()) {
        const uint64_t n_out = N - 1;
        if (out_width == 40 && ((uintptr_t)sa_out & 15) == 0 && n_out >= EMIT40_TILE) {
            // full 1024-entry tiles through shared memory, the rest entry by entry
            const uint64_t head_n = n_out / EMIT40_TILE * EMIT40_TILE;
            k_emit40<<<grid_for(head_n / EMIT40_TILE, 1, 148 * 8), 256, 0, c.stream>>>(sa.get(), n_out,
                                                                                      (uint8_t*)sa_out);
            DCX_CHECK_LAUNCH();
            c.launched();
            if (head_n < n_out)
                k_emit<<<1, 256, 0, c.stream>>>(sa.get() + head_n, n_out - head_n,
                                                (uint8_t*)sa_out + 5 * head_n, out_width);
        } else {
            k_emit<<<grid_for(N / 4 + 1, 256), 256, 0, c.stream>>>(sa.get(), N - 1, sa_out, out_width);
        }
    } else {
        k_emit_seg<<<grid_for(N, 256), 256, 0, c.stream>>>(sa.get(), segw_p, N, ls, sa_out, out_width);
    }
    DCX_CHECK_LAUNCH();
    c.launched();
    c.alg(N * (4 + out_width / 8));
    cudaEventRecord(ev[3], c.stream);
    DCX_CUDA(cudaEventSynchronize(ev[3]));
    if (depth == 0) {
        float a = 0, b = 0, d = 0;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        cudaEventElapsedTime(&d, ev[2], ev[3]);
        c.st.ms_phase12 += a;
        c.st.ms_phase3 += b;
        c.st.ms_phase4 += d;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    check_device_error(c);
}

// ---------------------------------------------------------------------------
// Whole build for one text (device or host pointers).
// ---------------------------------------------------------------------------
static void build_one(Ctx& c, const uint8_t* text, uint64_t n, int X, int width, void* sa_out, uint32_t flags,
                      bool strict) {
    if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "text longer than 2^32 - 2");
    if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (n && (!text || !sa_out)) throw Error(DCX_ERR_ARG, "null pointer");
    get_dc(c, (uint32_t)X);
    c.st = dcx_stats{};
    c.peak = c.in_use;
    if (n == 0) return;
    const bool dev = flags & DCX_DEVICE_PTRS;
    const bool packing = !(flags & DCX_NO_PACKING);
    cudaEvent_t e0, e1, e2, e3;
    const uint64_t pool0 = pool_reserved(c);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventCreate(&e3);
    cudaEventRecord(e0, c.stream);
    // Staging (host-pointer calls; device buffers the byte kernels cannot use in
    // place) is ONE allocation of the same size every call, so the staging pool
    // reuses it instead of splitting blocks: text copy first, then the SA.
    const size_t wb = width / 8;
    const bool stage_text = !dev || ((uintptr_t)text & 15);  // the byte kernels load 16 bytes at a time
    const bool stage_sa = !dev || ((uintptr_t)sa_out & 15);
    const size_t text_region = stage_text ? ((n + 16 + 255) & ~size_t(255)) : 0;
    DBuf<uint8_t> io;
    if (stage_text || stage_sa) io = DBuf<uint8_t>(&c, text_region + (stage_sa ? n * wb + 16 : 0), true);
    const uint8_t* dtext = text;
    if (stage_text) {
        DCX_CUDA(cudaMemcpyAsync(io.get(), text, n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 c.stream));
        dtext = io.get();
    }
    cudaEventRecord(e1, c.stream);
    // phase 0: alphabet (compress_alphabet, cli.cpp:417-463)
    DBuf<uint8_t> t_map(&c, n + 16);
    uint64_t sigma = 0;
    bool wide_text = false;
    if (flags & DCX_NO_REMAP) {
        DCX_CUDA(cudaMemcpyAsync(t_map.get(), dtext, n, cudaMemcpyDeviceToDevice, c.stream));
        DCX_CUDA(cudaMemsetAsync(c.d_h256, 0, 256 * 8, c.stream));
        k_hist256<<<grid_for(n / 16 + 1, 256, 148 * 4), 256, 0, c.stream>>>(t_map.get(), n, c.d_h256);
        DCX_CHECK_LAUNCH();
        unsigned long long h[256];
        DCX_CUDA(cudaMemcpyAsync(h, c.d_h256, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
        DCX_CUDA(cudaStreamSynchronize(c.stream));
        if (h[0]) throw Error(DCX_ERR_ARG, "char 0 is reserved for padding");
        c.level0_entropy = 0;
        for (int i = 1; i < 256; i++)
            if (h[i]) {
                const double p = (double)h[i] / (double)n;
                c.level0_entropy -= p * std::log2(p);
            }
        for (int i = 255; i > 0; i--)
            if (h[i]) {
                sigma = i;
                break;
            }
    } else {
        DCX_CUDA(cudaMemsetAsync(c.d_h256, 0, 256 * 8, c.stream));
        k_hist256<<<grid_for(n / 16 + 1, 256, 148 * 4), 256, 0, c.stream>>>(dtext, n, c.d_h256);
        DCX_CHECK_LAUNCH();
        unsigned long long h[256];
        DCX_CUDA(cudaMemcpyAsync(h, c.d_h256, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
        DCX_CUDA(cudaStreamSynchronize(c.stream));
        ByteMap map{};
        uint32_t next = 1;
        c.level0_entropy = 0;
        for (int i = 0; i < 256; i++)
            if (h[i]) {
                map.m[i] = (uint8_t)(next++);
                const double p = (double)h[i] / (double)n;
                c.level0_entropy -= p * std::log2(p);
            }
        sigma = next - 1;
        if (sigma == 256 && strict)
            throw Error(DCX_ERR_ALPHABET, "256 distinct symbols: 0 is reserved for padding");
        if (sigma == 256) wide_text = true;  // chars 1..256 need 32-bit storage
        else k_remap<<<grid_for(n / 16 + 1, 256, 148 * 8), 256, 0, c.stream>>>(dtext, t_map.get(), n, map);
        DCX_CHECK_LAUNCH();
    }
    c.launched(2);
    c.alg(n * 3);
    c.st.sigma = (uint32_t)sigma;
    cudaEventRecord(e2, c.stream);
    Segs one;  // the text as the only segment of level 0, followed by its 0
    one.start = {0, n + 1};
    DCX_CUDA(cudaMemsetAsync(t_map.get() + n, 0, 16, c.stream));
    // SA straight into the caller's device buffer, or into a staging buffer for host pointers
    void* dout = stage_sa ? (void*)(io.get() + text_region) : sa_out;
    if (wide_text) {
        // all 256 byte values occur: remap b -> b + 1 into 32-bit chars and build
        // with 257-symbol keys (the reference cli refuses this input)
        DBuf<uint32_t> t32(&c, n + 1);
        DCX_CUDA(cudaMemsetAsync(t32.get() + n, 0, 4, c.stream));
        k_widen_text<<<grid_for(n, 256), 256, 0, c.stream>>>(dtext, n, t32.get());
        DCX_CHECK_LAUNCH();
        c.launched();
        t_map.reset();
        level<uint32_t>(c, t32.get(), one, sigma, (uint32_t)X, 0, packing, dout, width);
    } else {
        level<uint8_t>(c, t_map.get(), one, sigma, (uint32_t)X, 0, packing, dout, width);
    }
    t_map.reset();
    if (dev && dout != sa_out)
        DCX_CUDA(cudaMemcpyAsync(sa_out, dout, n * wb, cudaMemcpyDeviceToDevice, c.stream));
    cudaEventRecord(e3, c.stream);
    cudaEvent_t e4;
    cudaEventCreate(&e4);
    if (!dev) DCX_CUDA(cudaMemcpyAsync(sa_out, dout, n * wb, cudaMemcpyDeviceToHost, c.stream));
    cudaEventRecord(e4, c.stream);
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    float d2h = 0;
    cudaEventElapsedTime(&d2h, e3, e4);
    c.st.ms_d2h = d2h;
    cudaEventDestroy(e4);
    float h2d = 0, p0 = 0, total = 0;
    cudaEventElapsedTime(&h2d, e0, e1);
    cudaEventElapsedTime(&p0, e1, e2);
    cudaEventElapsedTime(&total, e1, e3);
    c.st.ms_h2d = h2d;
    c.st.ms_phase0 = p0;
    c.st.ms_total = total;
    c.st.peak_bytes = c.peak;
    const uint64_t pool1 = pool_reserved(c);
    c.st.pool_growth_bytes = pool1 > pool0 ? pool1 - pool0 : 0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    cudaEventDestroy(e3);
}

// ---------------------------------------------------------------------------
// Building blocks of the multi-GPU single-text build (distributed.py): a stable
// device sort of (key words, value) pairs and the SA of a 32-bit string.
// ---------------------------------------------------------------------------
// Sorts n pairs in place by their kw little-endian uint32 key words (word kw-1
// most significant), stable, with the onesweep passes of every other sort.
static void sort_u32(Ctx& c, uint32_t* const* keys, uint32_t kw, uint32_t* vals, uint64_t n) {
    if (kw < 1 || kw > 3) throw Error(DCX_ERR_ARG, "1 to 3 key words");
    if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "more than 2^32 - 2 pairs");
    if (n <= 1) return;
    if (!keys || !vals) throw Error(DCX_ERR_ARG, "null pointer");
    for (uint32_t w = 0; w < kw; w++)
        if (!keys[w] || ((uintptr_t)keys[w] & 15)) throw Error(DCX_ERR_ARG, "key arrays must be 16-byte aligned");
    if ((uintptr_t)vals & 15) throw Error(DCX_ERR_ARG, "value array must be 16-byte aligned");
    c.st = dcx_stats{};
    c.peak = c.in_use;
    SortSpace s;
    DBuf<uint32_t> k1[3], v1(&c, n);
    for (uint32_t w = 0; w < kw; w++) {
        k1[w] = DBuf<uint32_t>(&c, n);
        s.k[0][w] = keys[w];
        s.k[1][w] = k1[w].get();
    }
    s.v[0] = vals;
    s.v[1] = v1.get();
    DCX_CUDA(cudaMemsetAsync(c.d_hist, 0, 16 * RADIX * 4, c.stream));
    SortPassArgs ha{};
    for (uint32_t w = 0; w < kw; w++) ha.keys_in[w] = keys[w];
    ha.kw = kw;
    ha.n = n;
    k_digit_hist<<<grid_for(n, 256, 148 * 4), 256, 4 * kw * RADIX * 4, c.stream>>>(ha, c.d_hist);
    DCX_CHECK_LAUNCH();
    c.launched();
    c.alg(n * 4 * kw);
    const int f = radix_sort(c, kw, n, s);
    if (f == 1) {
        for (uint32_t w = 0; w < kw; w++)
            DCX_CUDA(cudaMemcpyAsync(keys[w], k1[w].get(), n * 4, cudaMemcpyDeviceToDevice, c.stream));
        DCX_CUDA(cudaMemcpyAsync(vals, v1.get(), n * 4, cudaMemcpyDeviceToDevice, c.stream));
    }
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    c.st.peak_bytes = c.peak;
}

// SA of a device string of n 32-bit symbols in [1, sigma] (the recursion
// strings of the multi-GPU build): one DCX pipeline as for a recursion level.
static void build_u32(Ctx& c, const uint32_t* text, uint64_t n, uint64_t sigma, int X, int width, void* sa_out) {
    if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "string longer than 2^32 - 2");
    if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (sigma == 0 || sigma >= 0xffffffffull) throw Error(DCX_ERR_ARG, "alphabet bound must be in [1, 2^32 - 2]");
    if (n && (!text || !sa_out)) throw Error(DCX_ERR_ARG, "null pointer");
    get_dc(c, (uint32_t)X);
    c.st = dcx_stats{};
    c.peak = c.in_use;
    if (n == 0) return;
    DBuf<uint32_t> t(&c, n + 1);
    DCX_CUDA(cudaMemcpyAsync(t.get(), text, n * 4, cudaMemcpyDeviceToDevice, c.stream));
    DCX_CUDA(cudaMemsetAsync(t.get() + n, 0, 4, c.stream));
    Segs one;
    one.start = {0, n + 1};
    c.level0_entropy = 0;
    level<uint32_t>(c, t.get(), one, sigma, (uint32_t)X, 1, false, sa_out, width);
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    check_device_error(c);
    c.st.peak_bytes = c.peak;
}

// ---------------------------------------------------------------------------
// Batch: one SA per text.  Texts of at most SMALL_MAX chars are solved together
// by the in-CTA base case (one launch); the others run through segmented DCX
// levels, as many texts per round as the memory budget allows.  The alphabet
// remap of a round is the union of its texts' alphabets, which keeps every
// text's order (and therefore its SA) unchanged.
// ---------------------------------------------------------------------------
// X of a text of length len in a batched build with dc_or_auto = 0.
static uint32_t batch_x_for(const Options& o, uint64_t len) {
    for (const auto& e : o.batch_dc)
        if (len <= e.first) return e.second;
    return 39u;
}

// Radix tile items of a text's size class (the context's default past the table).
static uint32_t batch_items_for(const Options& o, uint64_t len) {
    for (size_t i = 0; i < o.batch_dc.size(); i++)
        if (len <= o.batch_dc[i].first) return i < o.batch_items.size() ? o.batch_items[i] : o.radix_items;
    return o.radix_items;
}

static void build_batch(Ctx& c, const uint8_t* texts, const uint64_t* offsets, uint32_t K, int dc_or_auto, int width,
                        void* sa_out, uint32_t flags) {
    if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (K == 0) return;
    if (!offsets || !texts || !sa_out) throw Error(DCX_ERR_ARG, "null pointer");
    const uint32_t X = dc_or_auto == 0 ? 39u : (uint32_t)dc_or_auto;  // auto: DC39 unless the size-class table says
    get_dc(c, X);
    const bool by_class = dc_or_auto == 0 && !c.opt.batch_dc.empty();
    if (by_class)
        for (const auto& e : c.opt.batch_dc) get_dc(c, e.second);
    const bool dev = flags & DCX_DEVICE_PTRS;
    const bool packing = !(flags & DCX_NO_PACKING);
    const size_t wb = width / 8;
    for (uint32_t s = 0; s < K; s++) {
        if (offsets[s + 1] < offsets[s]) throw Error(DCX_ERR_ARG, "offsets must be non-decreasing");
        if (offsets[s + 1] - offsets[s] >= 0xffffffffull) throw Error(DCX_ERR_ARG, "text longer than 2^32 - 2");
    }
    c.st = dcx_stats{};
    c.peak = c.in_use;
    const uint64_t base0 = offsets[0];
    // rounds: consecutive texts whose total stays below the per-round element cap
    const uint64_t budget_left = c.budget > c.in_use ? c.budget - c.in_use : 0;
    uint64_t cap = std::min<uint64_t>(1ull << 30, std::max<uint64_t>(budget_left / 48, 1ull << 20));
    if (c.opt.batch_round_cap) cap = c.opt.batch_round_cap;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c.stream);
    uint32_t s0 = 0;
    while (s0 < K) {
        uint32_t s1 = s0;
        uint64_t tot = 0;
        while (s1 < K && (s1 == s0 || tot + (offsets[s1 + 1] - offsets[s1] + 1) <= cap)) {
            tot += offsets[s1 + 1] - offsets[s1] + 1;
            s1++;
        }
        const uint64_t in_bytes = offsets[s1] - offsets[s0];
        // input of the round on the device (one copy)
        DBuf<uint8_t> din;
        const uint8_t* dsrc = texts + (offsets[s0] - base0);
        if (!dev) {
            din = DBuf<uint8_t>(&c, in_bytes + 16, true);
            if (in_bytes) DCX_CUDA(cudaMemcpyAsync(din.get(), dsrc, in_bytes, cudaMemcpyHostToDevice, c.stream));
            dsrc = din.get();
        }
        // alphabet of the round
        unsigned long long h[256];
        DCX_CUDA(cudaMemsetAsync(c.d_h256, 0, 256 * 8, c.stream));
        if (in_bytes) {
            if ((uintptr_t)dsrc & 15) {
                DBuf<uint8_t> al(&c, in_bytes + 16);
                DCX_CUDA(cudaMemcpyAsync(al.get(), dsrc, in_bytes, cudaMemcpyDeviceToDevice, c.stream));
                k_hist256<<<grid_for(in_bytes / 16 + 1, 256, 148 * 4), 256, 0, c.stream>>>(al.get(), in_bytes, c.d_h256);
                DCX_CHECK_LAUNCH();
                DCX_CUDA(cudaMemcpyAsync(h, c.d_h256, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
                DCX_CUDA(cudaStreamSynchronize(c.stream));
            } else {
                k_hist256<<<grid_for(in_bytes / 16 + 1, 256, 148 * 4), 256, 0, c.stream>>>(dsrc, in_bytes, c.d_h256);
                DCX_CHECK_LAUNCH();
                DCX_CUDA(cudaMemcpyAsync(h, c.d_h256, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
                DCX_CUDA(cudaStreamSynchronize(c.stream));
            }
        } else {
            memset(h, 0, sizeof(h));
        }
        ByteMap map{};
        uint32_t next = 1;
        c.level0_entropy = 0;
        for (int i = 0; i < 256; i++)
            if (h[i]) {
                map.m[i] = (uint8_t)(next++);
                const double p = (double)h[i] / (double)std::max<uint64_t>(in_bytes, 1);
                c.level0_entropy -= p * std::log2(p);
            }
        const uint64_t sigma = std::max<uint32_t>(next - 1, 1);
        const bool wide = sigma == 256;
        std::vector<uint64_t> in_off(offsets + s0, offsets + s1 + 1);
        for (auto& v : in_off) v -= offsets[s0];
        DBuf<uint64_t> d_inoff = upload(c, in_off);
        DBuf<ByteMap> d_map(&c, 1);
        DCX_CUDA(cudaMemcpyAsync(d_map.get(), &map, sizeof(map), cudaMemcpyHostToDevice, c.stream));
        // small texts first (one launch), then the rest as segments of DCX levels
        Segs small, big;
        small.start = {0};
        big.start = {0};
        std::vector<uint32_t> small_ids, big_ids;
        for (uint32_t s = s0; s < s1; s++) {
            const uint64_t len = offsets[s + 1] - offsets[s];
            if (len <= (uint64_t)std::min<uint32_t>(c.opt.small_threshold, SMALL_MAX)) {
                small.start.push_back(small.start.back() + len + 1);
                small_ids.push_back(s - s0);
            } else {
                big.start.push_back(big.start.back() + len + 1);
                big_ids.push_back(s - s0);
            }
        }
        // round output: the caller's device buffer, or a staging buffer copied back once
        DBuf<uint8_t> rstage;
        uint8_t* rout = (uint8_t*)sa_out + (offsets[s0] - base0) * wb;
        if (!dev) {
            rstage = DBuf<uint8_t>(&c, std::max<uint64_t>(in_bytes, 1) * wb + 16, true);
            rout = rstage.get();
        }
        auto run_group = [&](const Segs& g, const std::vector<uint32_t>& ids, uint32_t Xg) {
            if (ids.empty()) return;
            const uint32_t Kg = g.K();
            std::vector<uint64_t> goff(Kg + 1, 0), gsrc(Kg), cbase(Kg + 1, 0);
            for (uint32_t k = 0; k < Kg; k++) {
                const uint64_t len = in_off[ids[k] + 1] - in_off[ids[k]];
                gsrc[k] = in_off[ids[k]];
                goff[k + 1] = goff[k] + len;
                cbase[k + 1] = cbase[k] + std::max<uint64_t>(1, div_up(len, TEXT_CHUNK));
            }
            DBuf<uint64_t> d_goff = upload(c, goff), d_gsrc = upload(c, gsrc), d_cbase = upload(c, cbase);
            const uint64_t Ng = g.N();
            const uint64_t chunks = cbase[Kg];
            Segs gd = g;  // each text's SA goes straight to its slot of the round output
            gd.out_base = gsrc;
            const uint32_t blocks = (uint32_t)std::min<uint64_t>(chunks, 148 * 16);
            if (wide) {
                DBuf<uint32_t> buf(&c, Ng + 1);
                k_spread_texts<uint32_t><<<blocks, 256, 0, c.stream>>>(dsrc, d_gsrc.get(), d_goff.get(), d_cbase.get(),
                                                                       Kg, chunks, buf.get(), d_map.get(), true);
                DCX_CHECK_LAUNCH();
                level<uint32_t>(c, buf.get(), gd, sigma, Xg, 0, packing, rout, width);
            } else {
                DBuf<uint8_t> buf(&c, Ng + 16);
                k_spread_texts<uint8_t><<<blocks, 256, 0, c.stream>>>(dsrc, d_gsrc.get(), d_goff.get(), d_cbase.get(),
                                                                      Kg, chunks, buf.get(), d_map.get(), false);
                DCX_CHECK_LAUNCH();
                level<uint8_t>(c, buf.get(), gd, sigma, Xg, 0, packing, rout, width);
            }
            c.launched();
        };
        run_group(small, small_ids, X);
        if (by_class) {
            // one group per (X, radix tile) of the size-class table, each a level of its own
            std::map<std::pair<uint32_t, uint32_t>, std::pair<Segs, std::vector<uint32_t>>> by_x;
            for (uint32_t id : big_ids) {
                const uint64_t len = in_off[id + 1] - in_off[id];
                auto& e = by_x[{batch_x_for(c.opt, len), batch_items_for(c.opt, len)}];
                if (e.first.start.empty()) e.first.start = {0};
                e.first.start.push_back(e.first.start.back() + len + 1);
                e.second.push_back(id);
            }
            const uint32_t items0 = c.opt.radix_items;
            try {
                for (const auto& kv : by_x) {
                    c.opt.radix_items = kv.first.second;
                    run_group(kv.second.first, kv.second.second, kv.first.first);
                }
            } catch (...) {
                c.opt.radix_items = items0;
                throw;
            }
            c.opt.radix_items = items0;
        } else {
            run_group(big, big_ids, X);
        }
        if (!dev && in_bytes)
            DCX_CUDA(cudaMemcpyAsync((uint8_t*)sa_out + (offsets[s0] - base0) * wb, rout, in_bytes * wb,
                                     cudaMemcpyDeviceToHost, c.stream));
        DCX_CUDA(cudaStreamSynchronize(c.stream));
        s0 = s1;
    }
    cudaEventRecord(e1, c.stream);
    DCX_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    c.st.ms_total = ms;
    c.st.peak_bytes = c.peak;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// Autotuner of the size-class table: the texts of a host sample batch in each
// class (length in (class_max[i-1], class_max[i]]) are built as one batch with
// each candidate X (device-resident, one warm-up, median device time of
// `repeats` runs), and the fastest X per class becomes the context's table.
// Classes without sample texts keep DC39 (chosen[i] = 0).
static void autotune_batch(Ctx& c, const uint8_t* texts, const uint64_t* offsets, uint32_t K,
                           const uint64_t* class_max, uint32_t ncls, const int* cand, uint32_t ncand,
                           uint32_t repeats, int* chosen, double* ms_out) {
    if (!texts || !offsets || !class_max || !cand || !chosen || K == 0 || ncls == 0 || ncand == 0)
        throw Error(DCX_ERR_ARG, "null pointer or empty sample / classes / candidates");
    for (uint32_t i = 1; i < ncls; i++)
        if (class_max[i] <= class_max[i - 1]) throw Error(DCX_ERR_ARG, "class bounds must ascend");
    for (uint32_t j = 0; j < ncand; j++) {
        if (cand[j] <= 0) throw Error(DCX_ERR_ARG, "unsupported difference cover");
        get_dc(c, (uint32_t)cand[j]);
    }
    for (uint32_t s = 0; s < K; s++)
        if (offsets[s + 1] < offsets[s]) throw Error(DCX_ERR_ARG, "offsets must be non-decreasing");
    repeats = std::max<uint32_t>(repeats, 1);
    std::vector<std::pair<uint64_t, uint32_t>> table;
    std::vector<uint32_t> tiles;
    for (uint32_t i = 0; i < ncls; i++) {
        const uint64_t lo = i ? class_max[i - 1] : 0, hi = class_max[i];
        std::vector<uint64_t> offs = {0};
        std::vector<uint8_t> cat;
        for (uint32_t s = 0; s < K; s++) {
            const uint64_t len = offsets[s + 1] - offsets[s];
            if (len <= lo || len > hi) continue;
            const uint8_t* src = texts + (offsets[s] - offsets[0]);
            cat.insert(cat.end(), src, src + len);
            offs.push_back(offs.back() + len);
        }
        chosen[i] = 0;
        if (offs.size() == 1) {
            if (ms_out)
                for (uint32_t j = 0; j < ncand; j++) ms_out[(size_t)i * ncand + j] = -1.0;
            continue;
        }
        const uint32_t Kc = (uint32_t)(offs.size() - 1);
        const uint64_t bytes = offs.back();
        DBuf<uint8_t> d_text(&c, bytes + 16);
        DBuf<uint32_t> d_sa(&c, std::max<uint64_t>(bytes, 1));
        DCX_CUDA(cudaMemcpyAsync(d_text.get(), cat.data(), bytes, cudaMemcpyHostToDevice, c.stream));
        double best = 0;
        for (uint32_t j = 0; j < ncand; j++) {
            std::vector<double> t;
            for (uint32_t r = 0; r <= repeats; r++) {
                build_batch(c, d_text.get(), offs.data(), Kc, cand[j], 32, d_sa.get(), DCX_DEVICE_PTRS);
                if (r) t.push_back(c.st.ms_total);
            }
            std::sort(t.begin(), t.end());
            const double med = t[t.size() / 2];
            if (ms_out) ms_out[(size_t)i * ncand + j] = med;
            if (chosen[i] == 0 || med < best) {
                best = med;
                chosen[i] = cand[j];
            }
        }
        // the radix tile for the chosen X: the alternative size against the default
        uint32_t items = c.opt.radix_items;
        if (c.opt.batch_tune_tiles) {
            const uint32_t items0 = c.opt.radix_items;
            const uint32_t alt = items0 == ONESWEEP_ITEMS ? ONESWEEP_ITEMS_ALT : ONESWEEP_ITEMS;
            std::vector<double> t;
            try {
                c.opt.radix_items = alt;
                for (uint32_t r = 0; r <= repeats; r++) {
                    build_batch(c, d_text.get(), offs.data(), Kc, chosen[i], 32, d_sa.get(), DCX_DEVICE_PTRS);
                    if (r) t.push_back(c.st.ms_total);
                }
            } catch (...) {
                c.opt.radix_items = items0;
                throw;
            }
            c.opt.radix_items = items0;
            std::sort(t.begin(), t.end());
            if (t[t.size() / 2] < best) items = alt;
        }
        table.push_back({hi, (uint32_t)chosen[i]});
        tiles.push_back(items);
    }
    c.opt.batch_dc = table;
    c.opt.batch_items = tiles;
}

// Checks that sa (n entries of `width` bits) is the suffix array of text.
static bool check_one(Ctx& c, const uint8_t* text, uint64_t n, const void* sa, int width, uint32_t flags) {
    if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "text longer than 2^32 - 2");
    if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (n == 0) return true;
    if (!text || !sa) throw Error(DCX_ERR_ARG, "null pointer");
    const bool dev = flags & DCX_DEVICE_PTRS;
    const size_t wb = width / 8;
    DBuf<uint8_t> t_in, sa_in;
    const uint8_t* dtext = text;
    const void* dsa = sa;
    if (!dev) {
        t_in = DBuf<uint8_t>(&c, n);
        sa_in = DBuf<uint8_t>(&c, n * wb);
        DCX_CUDA(cudaMemcpyAsync(t_in.get(), text, n, cudaMemcpyHostToDevice, c.stream));
        DCX_CUDA(cudaMemcpyAsync(sa_in.get(), sa, n * wb, cudaMemcpyHostToDevice, c.stream));
        dtext = t_in.get();
        dsa = sa_in.get();
    }
    DBuf<uint32_t> isa(&c, n);
    DBuf<unsigned long long> bad(&c, 1);
    DCX_CUDA(cudaMemsetAsync(isa.get(), 0, n * 4, c.stream));
    DCX_CUDA(cudaMemsetAsync(bad.get(), 0, 8, c.stream));
    k_check_isa<<<grid_for(n, 256), 256, 0, c.stream>>>(dsa, width, n, isa.get(), bad.get());
    k_check_order<<<grid_for(n, 256), 256, 0, c.stream>>>(dsa, width, n, dtext, isa.get(), bad.get());
    DCX_CHECK_LAUNCH();
    return d2h_scalar(c, bad.get()) == 0;
}

// ---------------------------------------------------------------------------
// SA files in the reference's raw layout: the entries back to back, little
// endian, no header (write_data, lightweight_dcx/src/mpi/io.hpp:80-98; 40-bit
// entries are util/uint_types.hpp's uint40).  Device <-> file through two
// pinned chunk buffers, so the copy of one chunk overlaps the file access of
// the other.
// ---------------------------------------------------------------------------
struct ChunkStage {
    cudaStream_t stream = nullptr;
    void* buf[2] = {};
    cudaEvent_t done[2] = {};
    FILE* f = nullptr;
    ~ChunkStage() {
        if (stream) cudaStreamSynchronize(stream);  // no copy may still target the buffers
        for (int b = 0; b < 2; b++) {
            if (buf[b]) cudaFreeHost(buf[b]);
            if (done[b]) cudaEventDestroy(done[b]);
        }
        if (f) fclose(f);
    }
};

static uint64_t sa_file_chunk(uint64_t total, uint64_t chunk) {
    if (chunk == 0) chunk = 64ull << 20;
    return std::max<uint64_t>(std::min<uint64_t>(chunk, total), 1);
}

static void open_stage(Ctx& c, ChunkStage& cs, const char* path, const char* mode, uint64_t chunk) {
    cs.f = fopen(path, mode);
    if (!cs.f) throw Error(DCX_ERR_IO, std::string("cannot open ") + path);
    cs.stream = c.stream;
    for (int b = 0; b < 2; b++) {
        DCX_CUDA(cudaHostAlloc(&cs.buf[b], chunk, cudaHostAllocDefault));
        DCX_CUDA(cudaEventCreateWithFlags(&cs.done[b], cudaEventDisableTiming));
    }
}

static void write_sa_file(Ctx& c, const char* path, const void* sa_dev, uint64_t n, int width, uint64_t chunk) {
    if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (!path || (n && !sa_dev)) throw Error(DCX_ERR_ARG, "null pointer");
    const uint64_t total = n * (uint64_t)(width / 8);
    chunk = sa_file_chunk(total, chunk);
    ChunkStage cs;
    open_stage(c, cs, path, "wb", chunk);
    const uint64_t chunks = div_up(total, chunk);
    auto len_of = [&](uint64_t i) { return std::min<uint64_t>(chunk, total - i * chunk); };
    for (uint64_t i = 0; i < chunks; i++) {
        const int b = (int)(i & 1);
        // buffer b last held chunk i-2, written to the file in the previous iteration
        DCX_CUDA(cudaMemcpyAsync(cs.buf[b], (const uint8_t*)sa_dev + i * chunk, len_of(i), cudaMemcpyDeviceToHost,
                                 c.stream));
        DCX_CUDA(cudaEventRecord(cs.done[b], c.stream));
        if (i > 0) {
            DCX_CUDA(cudaEventSynchronize(cs.done[b ^ 1]));
            if (fwrite(cs.buf[b ^ 1], 1, len_of(i - 1), cs.f) != len_of(i - 1))
                throw Error(DCX_ERR_IO, std::string("short write to ") + path);
        }
    }
    if (chunks) {
        const int b = (int)((chunks - 1) & 1);
        DCX_CUDA(cudaEventSynchronize(cs.done[b]));
        if (fwrite(cs.buf[b], 1, len_of(chunks - 1), cs.f) != len_of(chunks - 1))
            throw Error(DCX_ERR_IO, std::string("short write to ") + path);
    }
    FILE* f = cs.f;
    cs.f = nullptr;
    if (fclose(f) != 0) throw Error(DCX_ERR_IO, std::string("cannot close ") + path);
}

static void read_sa_file(Ctx& c, const char* path, void* sa_dev, uint64_t n, int width, uint64_t chunk) {
    if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (!path || (n && !sa_dev)) throw Error(DCX_ERR_ARG, "null pointer");
    const uint64_t total = n * (uint64_t)(width / 8);
    chunk = sa_file_chunk(total, chunk);
    ChunkStage cs;
    open_stage(c, cs, path, "rb", chunk);
    if (fseeko(cs.f, 0, SEEK_END) != 0) throw Error(DCX_ERR_IO, std::string("cannot seek in ") + path);
    const off_t size = ftello(cs.f);
    if (size < 0 || (uint64_t)size < total) throw Error(DCX_ERR_ARG, "SA file shorter than n entries");
    rewind(cs.f);
    const uint64_t chunks = div_up(total, chunk);
    for (uint64_t i = 0; i < chunks; i++) {
        const int b = (int)(i & 1);
        const uint64_t len = std::min<uint64_t>(chunk, total - i * chunk);
        if (i >= 2) DCX_CUDA(cudaEventSynchronize(cs.done[b]));  // the copy of chunk i-2 left buffer b
        if (fread(cs.buf[b], 1, len, cs.f) != len) throw Error(DCX_ERR_IO, std::string("short read of ") + path);
        DCX_CUDA(cudaMemcpyAsync((uint8_t*)sa_dev + i * chunk, cs.buf[b], len, cudaMemcpyHostToDevice, c.stream));
        DCX_CUDA(cudaEventRecord(cs.done[b], c.stream));
    }
    DCX_CUDA(cudaStreamSynchronize(c.stream));
}

// dcx_check_sa for an SA file: the file streamed into device memory, the text
// (host or device per flags) beside it.
static bool check_sa_file(Ctx& c, const uint8_t* text, uint64_t n, const char* path, int width, uint32_t flags) {
    if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "text longer than 2^32 - 2");
    if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (!path || (n && !text)) throw Error(DCX_ERR_ARG, "null pointer");
    DBuf<uint8_t> dsa(&c, std::max<uint64_t>(n * (width / 8), 1));
    read_sa_file(c, path, dsa.get(), n, width, 0);
    if (n == 0) return true;
    const uint8_t* dtext = text;
    DBuf<uint8_t> t;
    if (!(flags & DCX_DEVICE_PTRS)) {
        t = DBuf<uint8_t>(&c, n);
        DCX_CUDA(cudaMemcpyAsync(t.get(), text, n, cudaMemcpyHostToDevice, c.stream));
        dtext = t.get();
    }
    return check_one(c, dtext, n, dsa.get(), width, DCX_DEVICE_PTRS);
}

// phi[SA[k]] = SA[k-1]: a direct scatter while phi fits L2 (16 MB), else the
// two-step form (records, one radix pass on the top 8 bits of SA[k], an
// L2-local scatter).
static void build_phi(Ctx& c, const uint32_t* sa32, uint64_t n, uint32_t* phi) {
    if (n <= (1u << 22)) {
        k_phi<<<grid_for(n, 256), 256, 0, c.stream>>>(sa32, n, phi);
        DCX_CHECK_LAUNCH();
        c.launched();
        c.alg(n * 12);
        return;
    }
    const uint32_t shift = top_digit_shift(n);
    SortSpace s;
    DBuf<uint32_t> pk[2], pv[2];
    for (int b = 0; b < 2; b++) {
        pk[b] = DBuf<uint32_t>(&c, n);
        pv[b] = DBuf<uint32_t>(&c, n);
        s.k[b][0] = pk[b].get();
        s.v[b] = pv[b].get();
    }
    DCX_CUDA(cudaMemsetAsync(c.d_hist, 0, 16 * RADIX * 4, c.stream));
    k_phi_records<<<grid_for(n, 256, 148 * 8), 256, 0, c.stream>>>(sa32, n, s.k[0][0], s.v[0], c.d_hist, shift);
    DCX_CHECK_LAUNCH();
    c.launched();
    c.alg(n * 16);
    const int f = radix_sort(c, 1, n, s, (int)shift);
    // One pair per thread: blocks start in index order, so the blocks in flight
    // cover a narrow run of the grouped pairs and their stores stay in the one
    // or two ranges in flight, which L2 fills before writing back.  (A
    // grid-stride loop over resident CTAs lets warps drift apart across the
    // ranges; on 2^28 8-byte records grouped by their top 8 bits that ran 5.5x
    // slower: 9.6 ms against 1.74 ms, fully random 11.5 ms, in order 0.94 ms.)
    k_phi_scatter<<<(unsigned)div_up(n, 256), 256, 0, c.stream>>>(s.k[f][0], s.v[f], n, phi);
    DCX_CHECK_LAUNCH();
    c.launched();
    c.alg(n * 12);
}

// LCP (or PLCP with DCX_LCP_PERMUTED) of a text and its SA; lcp_width 32 or 64.
static void build_lcp(Ctx& c, const uint8_t* text, uint64_t n, const void* sa, int sa_width, void* out,
                      int lcp_width, uint32_t flags) {
    if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "text longer than 2^32 - 2");
    if (!(sa_width == 32 || sa_width == 40 || sa_width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (!(lcp_width == 32 || lcp_width == 64)) throw Error(DCX_ERR_ARG, "lcp_width must be 32 or 64");
    if (n == 0) return;
    if (!text || !sa || !out) throw Error(DCX_ERR_ARG, "null pointer");
    const bool dev = flags & DCX_DEVICE_PTRS;
    const size_t wb = sa_width / 8, lb = lcp_width / 8;
    // padded text copy: the comparison loads read up to 15 bytes past the end
    DBuf<uint8_t> t(&c, n + 16);
    DCX_CUDA(cudaMemsetAsync(t.get() + n, 0, 16, c.stream));
    DCX_CUDA(cudaMemcpyAsync(t.get(), text, n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream));
    DBuf<uint8_t> sa_in;
    const void* dsa = sa;
    if (!dev) {
        sa_in = DBuf<uint8_t>(&c, n * wb);
        DCX_CUDA(cudaMemcpyAsync(sa_in.get(), sa, n * wb, cudaMemcpyHostToDevice, c.stream));
        dsa = sa_in.get();
    }
    DBuf<uint32_t> phi(&c, n), sa32(&c, n), plcp(&c, n);
    k_sa_to_u32<<<grid_for(div_up(n, 4), 256), 256, 0, c.stream>>>(dsa, sa_width, n, sa32.get());
    DCX_CHECK_LAUNCH();
    c.launched();
    build_phi(c, sa32.get(), n, phi.get());
    sa_in.reset();
    if (flags & DCX_LCP_GSA) {
        // a generalized SA: separators (0 bytes) are distinct symbols, no match runs through one
        if (d2h_scalar(c, t.get() + n - 1) != 0) throw Error(DCX_ERR_ARG, "a string set ends with a 0 byte");
        DBuf<uint32_t> zb(&c, n), sep(&c, n);
        device_scan<uint32_t>(c, OpSeparators{t.get(), zb.get(), sep.get()}, n);
        k_plcp_to_separator<<<grid_for(div_up(n, LCP_RUN), 128, 148 * 64), 128, 0, c.stream>>>(
            t.get(), n, phi.get(), zb.get(), sep.get(), plcp.get(), 0);
        c.launched();
    } else {
        k_plcp<<<grid_for(div_up(n, LCP_RUN), 128, 148 * 64), 128, 0, c.stream>>>(t.get(), n, phi.get(), plcp.get());
    }
    DCX_CHECK_LAUNCH();
    phi.reset();
    DBuf<uint8_t> stage;
    void* dout = out;
    if (!dev) {
        stage = DBuf<uint8_t>(&c, n * lb);
        dout = stage.get();
    }
    k_lcp_gather<<<grid_for(n, 256), 256, 0, c.stream>>>(sa32.get(), plcp.get(), n, dout, lcp_width,
                                                        (flags & DCX_LCP_PERMUTED) != 0);
    DCX_CHECK_LAUNCH();
    c.launched(2);
    if (!dev) DCX_CUDA(cudaMemcpyAsync(out, dout, n * lb, cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaStreamSynchronize(c.stream));
}

// BWT (libsais64_bwt convention) of a text and its SA; returns the primary index.
static uint64_t build_bwt(Ctx& c, const uint8_t* text, uint64_t n, const void* sa, int sa_width, uint8_t* out,
                          uint32_t flags) {
    if (!(sa_width == 32 || sa_width == 40 || sa_width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    if (sa_width < 64 && n > (1ull << sa_width)) throw Error(DCX_ERR_ARG, "text too long for the SA width");
    if (n == 0) return 0;
    if (!text || !sa || !out) throw Error(DCX_ERR_ARG, "null pointer");
    const bool dev = flags & DCX_DEVICE_PTRS;
    const size_t wb = sa_width / 8;
    if (dev && sa_width != 40 && ((uintptr_t)sa % wb) != 0) throw Error(DCX_ERR_ARG, "SA not aligned to its width");
    DBuf<uint8_t> t, sa_in, stage;
    const uint8_t* dtext = text;
    const void* dsa = sa;
    uint8_t* dout = out;
    if (!dev) {
        t = DBuf<uint8_t>(&c, n, true);
        sa_in = DBuf<uint8_t>(&c, n * wb, true);
        stage = DBuf<uint8_t>(&c, n, true);
        DCX_CUDA(cudaMemcpyAsync(t.get(), text, n, cudaMemcpyHostToDevice, c.stream));
        DCX_CUDA(cudaMemcpyAsync(sa_in.get(), sa, n * wb, cudaMemcpyHostToDevice, c.stream));
        dtext = t.get();
        dsa = sa_in.get();
        dout = stage.get();
    }
    DBuf<BwtScan> st(&c, 1);
    unsigned long long* stw = reinterpret_cast<unsigned long long*>(st.get());  // first_zero, zeros, out_of_range
    DCX_CUDA(cudaMemsetAsync(stw, 0xff, sizeof(unsigned long long), c.stream));
    DCX_CUDA(cudaMemsetAsync(stw + 1, 0, 2 * sizeof(unsigned long long), c.stream));
    k_bwt_primary<<<grid_for(n, 256), 256, 0, c.stream>>>(dsa, sa_width, n, st.get());
    DCX_CHECK_LAUNCH();
    const BwtScan h = d2h_scalar(c, st.get());
    if (h.out_of_range || h.zeros != 1)
        throw Error(DCX_ERR_ARG, "not a suffix array of the text (an entry >= n, or not exactly one 0)");
    const uint64_t p = h.first_zero + 1;
    k_bwt_gather<<<grid_for(n, 256), 256, 0, c.stream>>>(dtext, n, dsa, sa_width, p, dout);
    DCX_CHECK_LAUNCH();
    c.launched(2);
    if (!dev) DCX_CUDA(cudaMemcpyAsync(out, dout, n, cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    return p;
}

// BWT of a text, its SA built on the GPU and dropped (libsais64_bwt's call).
static uint64_t bwt_of_text(Ctx& c, const uint8_t* text, uint64_t n, int X, uint8_t* out, uint32_t flags) {
    if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "text longer than 2^32 - 2");
    get_dc(c, (uint32_t)X);
    if (n == 0) return 0;
    if (!text || !out) throw Error(DCX_ERR_ARG, "null pointer");
    const bool dev = flags & DCX_DEVICE_PTRS;
    DBuf<uint8_t> t, o;
    const uint8_t* dtext = text;
    uint8_t* dout = out;
    if (!dev) {
        t = DBuf<uint8_t>(&c, n + 16, true);
        o = DBuf<uint8_t>(&c, n, true);
        DCX_CUDA(cudaMemcpyAsync(t.get(), text, n, cudaMemcpyHostToDevice, c.stream));
        dtext = t.get();
        dout = o.get();
    }
    DBuf<uint32_t> sa32(&c, n);
    build_one(c, dtext, n, X, 32, sa32.get(), DCX_DEVICE_PTRS | (flags & (DCX_NO_PACKING | DCX_NO_REMAP)), false);
    const uint64_t p = build_bwt(c, dtext, n, sa32.get(), 32, dout, DCX_DEVICE_PTRS);
    if (!dev) {
        DCX_CUDA(cudaMemcpyAsync(out, dout, n, cudaMemcpyDeviceToHost, c.stream));
        DCX_CUDA(cudaStreamSynchronize(c.stream));
    }
    return p;
}

// Generalized SA of a string set (libsais64_gsa convention) from the plain SA:
// runs of plain-SA neighbours that agree through their separators re-sorted by
// position.
static void build_gsa(Ctx& c, const uint8_t* text, uint64_t n, int X, int width, void* out, uint32_t flags) {
    if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "text longer than 2^32 - 2");
    if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
    get_dc(c, (uint32_t)X);
    if (n == 0) return;
    if (!text || !out) throw Error(DCX_ERR_ARG, "null pointer");
    const bool dev = flags & DCX_DEVICE_PTRS;
    const size_t wb = width / 8;
    if (dev && width != 40 && ((uintptr_t)out % wb) != 0) throw Error(DCX_ERR_ARG, "SA not aligned to its width");
    // the set, zero-padded: the LCP word loads read up to 15 bytes past its end
    DBuf<uint8_t> t(&c, n + 16);
    DCX_CUDA(cudaMemsetAsync(t.get() + n, 0, 16, c.stream));
    DCX_CUDA(cudaMemcpyAsync(t.get(), text, n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream));
    {
        DBuf<unsigned long long> bad(&c, 1);
        DCX_CUDA(cudaMemsetAsync(bad.get(), 0, 8, c.stream));
        k_gsa_check<<<grid_for(n, 256), 256, 0, c.stream>>>(t.get(), n, bad.get());
        DCX_CHECK_LAUNCH();
        if (d2h_scalar(c, bad.get()))
            throw Error(DCX_ERR_ARG, "not a string set: the last byte must be 0 and no string may be empty");
    }
    if (n == 1) {  // the set "\0"
        if (dev) DCX_CUDA(cudaMemsetAsync(out, 0, wb, c.stream));
        else memset(out, 0, wb);
        DCX_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    // plain SA of the whole set
    DBuf<uint32_t> sa32(&c, n);
    build_one(c, t.get(), n, X, 32, sa32.get(), DCX_DEVICE_PTRS | (flags & DCX_NO_PACKING), false);
    // separators, capped PLCP, run heads
    DBuf<uint8_t> head(&c, n);
    {
        DBuf<uint32_t> zb(&c, n), sep(&c, n / 2 + 1);  // no empty string: at most n/2 separators
        device_scan<uint32_t>(c, OpSeparators{t.get(), zb.get(), sep.get()}, n);
        DBuf<uint32_t> phi(&c, n), plcp(&c, n);
        build_phi(c, sa32.get(), n, phi.get());
        k_plcp_to_separator<<<grid_for(div_up(n, LCP_RUN), 128, 148 * 64), 128, 0, c.stream>>>(
            t.get(), n, phi.get(), zb.get(), sep.get(), plcp.get(), 1);
        DCX_CHECK_LAUNCH();
        phi.reset();
        k_gsa_heads<<<grid_for(n, 256), 256, 0, c.stream>>>(sa32.get(), n, plcp.get(), zb.get(), sep.get(),
                                                            head.get());
        DCX_CHECK_LAUNCH();
        c.launched(2);
    }
    // runs re-sorted by (run number, position)
    {
        DBuf<uint32_t> slot(&c, n), grp(&c, n), tpos(&c, n);
        OpTied op{head.get(), n, sa32.get(), nullptr, slot.get(), grp.get(), tpos.get(), nullptr};
        const uint64_t cnt = device_scan<uint64_t>(c, op, n) >> 32;
        if (cnt) {
            DBuf<uint32_t> k1[2], vals[2];
            SortSpace s;
            s.k[0][0] = tpos.get();
            s.k[0][1] = grp.get();
            for (int w = 0; w < 2; w++) {
                k1[w] = DBuf<uint32_t>(&c, cnt);
                s.k[1][w] = k1[w].get();
                vals[w] = DBuf<uint32_t>(&c, cnt);
                s.v[w] = vals[w].get();
            }
            DCX_CUDA(cudaMemsetAsync(c.d_hist, 0, 16 * RADIX * 4, c.stream));
            SortPassArgs ha{};
            ha.keys_in[0] = s.k[0][0];
            ha.keys_in[1] = s.k[0][1];
            ha.kw = 2;
            ha.n = cnt;
            k_digit_hist<<<grid_for(cnt, 256, 148 * 4), 256, 8 * RADIX * 4, c.stream>>>(ha, c.d_hist);
            DCX_CHECK_LAUNCH();
            const int f = radix_sort(c, 2, cnt, s);
            k_gsa_scatter<<<grid_for(cnt, 256), 256, 0, c.stream>>>(cnt, slot.get(), s.k[f][0], sa32.get());
            DCX_CHECK_LAUNCH();
            c.launched(2);
        }
    }
    head.reset();
    DBuf<uint8_t> stage;
    void* dout = out;
    if (!dev) {
        stage = DBuf<uint8_t>(&c, n * wb, true);
        dout = stage.get();
    }
    k_store_sa<<<grid_for(n, 256), 256, 0, c.stream>>>(sa32.get(), n, dout, width);
    DCX_CHECK_LAUNCH();
    c.launched();
    if (!dev) DCX_CUDA(cudaMemcpyAsync(out, dout, n * wb, cudaMemcpyDeviceToHost, c.stream));
    DCX_CUDA(cudaStreamSynchronize(c.stream));
    check_device_error(c);
}

}  // namespace dcx

#include "serve.cuh"

namespace dcx {

static void ctx_init(Ctx& c, int device, uint64_t budget) {
    c.device = device;
    DCX_CUDA(cudaSetDevice(device));
    DCX_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    cudaMemPool_t pool;
    DCX_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = UINT64_MAX;
    DCX_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    size_t fr = 0, tot = 0;
    DCX_CUDA(cudaMemGetInfo(&fr, &tot));
    c.budget = budget ? budget : (uint64_t)(fr * 0.9);
    DCX_CUDA(cudaMalloc(&c.d_hist, 16 * RADIX * 4));
    DCX_CUDA(cudaMalloc(&c.d_base, 16 * RADIX * 4));
    DCX_CUDA(cudaMalloc(&c.d_tiles, 64 * 4));
    DCX_CUDA(cudaMalloc(&c.d_err, 8));
    DCX_CUDA(cudaMemset(c.d_err, 0, 8));
    DCX_CUDA(cudaMalloc(&c.d_h256, 256 * 8));
    DCX_CUDA(cudaHostAlloc((void**)&c.h_pinned, PINNED_WORDS * 4, cudaHostAllocDefault));
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    DCX_CUDA(cudaMemPoolCreate(&c.io_pool, &props));
    DCX_CUDA(cudaMemPoolSetAttribute(c.io_pool, cudaMemPoolAttrReleaseThreshold, &thr));
}

static void ctx_free(Ctx& c) {
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    cudaFree(c.d_hist);
    cudaFree(c.d_base);
    cudaFree(c.d_tiles);
    cudaFree(c.d_err);
    cudaFree(c.d_h256);
    if (c.d_lookback) cudaFree(c.d_lookback);
    if (c.h_pinned) cudaFreeHost(c.h_pinned);
    for (auto& kv : c.dc_dev) cudaFree(kv.second);
    for (auto& kv : c.dc_flags_dev) cudaFree(kv.second);
    if (c.stream) cudaStreamDestroy(c.stream);
    if (c.io_pool) cudaMemPoolDestroy(c.io_pool);
    c.io_pool = nullptr;
    c.stream = nullptr;
    c.d_lookback = nullptr;
    c.h_pinned = nullptr;
    c.dc_dev.clear();
    c.dc_flags_dev.clear();
}

}  // namespace dcx

// ===========================================================================
// C ABI
// ===========================================================================
struct dcx_ctx {
    dcx::Ctx c;
    std::mutex serve_mu;
    std::unique_ptr<dcx::Server> server;  // started by the first dcx_serve_submit
};

using dcx::Error;

template <typename F>
static int guarded(F&& f) {
    try {
        f();
        return DCX_OK;
    } catch (const Error& e) {
        if (getenv("DCX_VERBOSE")) fprintf(stderr, "dcx: %s\n", e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        return DCX_ERR_OOM;
    } catch (...) {
        return DCX_ERR_INTERNAL;
    }
}

extern "C" {

const char* dcx_version(void) { return "dcx-b200 0.1"; }

const char* dcx_strerror(int code) {
    switch (code) {
        case DCX_OK: return "ok";
        case DCX_ERR_ARG: return "invalid argument";
        case DCX_ERR_ALPHABET: return "alphabet of 256 symbols (0 is reserved for padding)";
        case DCX_ERR_OOM: return "out of device memory";
        case DCX_ERR_BUDGET: return "projected device footprint above the budget";
        case DCX_ERR_TIMEOUT: return "bounded device wait gave up";
        case DCX_ERR_CUDA: return "CUDA error";
        case DCX_ERR_INTERNAL: return "internal error";
        case DCX_ERR_BUSY: return "busy";
        case DCX_ERR_NOTFOUND: return "unknown request";
        case DCX_ERR_IO: return "file error";
        default: return "unknown error";
    }
}

int dcx_dc_table(int X, uint32_t* D, uint32_t* dc, uint32_t* next_rank, uint32_t* cmp) {
    dcx::DcHost h;
    if (X <= 0 || !dcx::make_dc((uint32_t)X, h)) return DCX_ERR_ARG;
    if (D) *D = h.D;
    if (dc) memcpy(dc, h.dc.data(), h.D * 4);
    if (next_rank) memcpy(next_rank, h.next_rank.data(), X * 4);
    if (cmp) memcpy(cmp, h.cmp.data(), h.cmp.size() * 4);
    return DCX_OK;
}

int dcx_shard_texts(const uint64_t* lengths, uint32_t num_texts, uint32_t world, uint32_t* owner,
                    uint64_t* load_out) {
    if (world == 0 || (num_texts > 0 && (!lengths || !owner))) return DCX_ERR_ARG;
    std::vector<uint32_t> order(num_texts);
    for (uint32_t i = 0; i < num_texts; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return lengths[a] > lengths[b]; });
    // min-heap of (load, rank): the lightest rank, the lower rank on equal loads
    using Slot = std::pair<uint64_t, uint32_t>;
    std::vector<Slot> heap(world);
    for (uint32_t r = 0; r < world; ++r) heap[r] = {0, r};
    auto heavier = [](const Slot& a, const Slot& b) { return a > b; };
    std::make_heap(heap.begin(), heap.end(), heavier);
    for (uint32_t i : order) {
        std::pop_heap(heap.begin(), heap.end(), heavier);
        owner[i] = heap.back().second;
        heap.back().first += lengths[i];
        std::push_heap(heap.begin(), heap.end(), heavier);
    }
    if (load_out)
        for (const Slot& s : heap) load_out[s.second] = s.first;
    return DCX_OK;
}

int dcx_ctx_create(dcx_ctx** out, int device, uint64_t budget) {
    if (!out) return DCX_ERR_ARG;
    *out = nullptr;
    return guarded([&] {
        auto* x = new dcx_ctx();
        try {
            dcx::ctx_init(x->c, device, budget);
        } catch (...) {
            dcx::ctx_free(x->c);
            delete x;
            throw;
        }
        *out = x;
    });
}

int dcx_ctx_destroy(dcx_ctx* x) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        x->server.reset();  // joins the lanes, frees unreleased results
        dcx::ctx_free(x->c);
        delete x;
    });
}

int dcx_set_option(dcx_ctx* x, const char* name, double value) {
    if (!x || !name) return DCX_ERR_ARG;
    dcx::Options& o = x->c.opt;
    std::string s(name);
    if (s == "discarding_threshold") o.discarding_threshold = value;
    else if (s == "recursion_dc") {
        dcx::DcHost h;
        if (value != 0 && !dcx::make_dc((uint32_t)value, h)) return DCX_ERR_ARG;
        o.recursion_dc = (uint32_t)value;
    } else if (s == "small_threshold") {
        if (value < 0 || value > dcx::SMALL_MAX) return DCX_ERR_ARG;
        o.small_threshold = (uint32_t)value;
    } else if (s == "prefix_chars") o.prefix_chars = (uint32_t)value;
    else if (s == "batch_tune_tiles") o.batch_tune_tiles = value != 0;
    else if (s == "radix_tile") {
        if (value != dcx::SORT_THREADS * dcx::ONESWEEP_ITEMS && value != dcx::SORT_THREADS * dcx::ONESWEEP_ITEMS_ALT) return DCX_ERR_ARG;
        o.radix_items = (uint32_t)value / dcx::SORT_THREADS;
    } else if (s == "rec_prefix_words") {
        if (value < 2 || value > 3) return DCX_ERR_ARG;
        o.rec_prefix_words = (uint32_t)value;
    }
    else if (s == "trace") o.trace = value != 0;
    else if (s == "spin_limit") o.spin_limit = (uint32_t)value;
    else if (s == "lookback_hold_tile") o.lookback_hold_tile = value < 0 ? 0xffffffffu : (uint32_t)value;
    else if (s == "batch_round_cap") o.batch_round_cap = (uint64_t)value;
    else if (s == "serve_lanes") {
        if (value < 1 || value > 16) return DCX_ERR_ARG;
        o.serve_lanes = (uint32_t)value;
    } else if (s == "serve_budget") o.serve_budget = (uint64_t)value;
    else if (s == "serve_host_bytes") o.serve_host_bytes = (uint64_t)value;
    else if (s == "serve_express_bytes") o.serve_express_bytes = (uint64_t)value;
    else if (s == "serve_express_priority") o.serve_express_priority = value != 0;
    else if (s == "serve_batch_bytes") {
        if (value < 1) return DCX_ERR_ARG;
        o.serve_batch_bytes = (uint64_t)value;
    } else if (s == "serve_batch_texts") {
        if (value < 1) return DCX_ERR_ARG;
        o.serve_batch_texts = (uint32_t)value;
    } else return DCX_ERR_ARG;
    return DCX_OK;
}

static int build_entry(dcx_ctx* x, const uint8_t* text, uint64_t n, int dc, int w, void* out, uint32_t flags,
                       bool strict) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::build_one(x->c, text, n, dc, w, out, flags, strict);
    });
}

int dcx_build_sa(dcx_ctx* x, const uint8_t* text, uint64_t n, int dc, int w, void* out, uint32_t flags) {
    return build_entry(x, text, n, dc, w, out, flags, false);
}

int dcx_build_sa_strict(dcx_ctx* x, const uint8_t* text, uint64_t n, int dc, int w, void* out, uint32_t flags) {
    return build_entry(x, text, n, dc, w, out, flags, true);
}

int dcx_build_lcp(dcx_ctx* x, const uint8_t* text, uint64_t n, const void* sa, int sa_width, void* lcp_out,
                  int lcp_width, uint32_t flags) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::build_lcp(x->c, text, n, sa, sa_width, lcp_out, lcp_width, flags);
    });
}

int dcx_build_gsa(dcx_ctx* x, const uint8_t* text, uint64_t n, int dc, int w, void* out, uint32_t flags) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::build_gsa(x->c, text, n, dc, w, out, flags);
    });
}

int dcx_bwt(dcx_ctx* x, const uint8_t* text, uint8_t* bwt_out, uint64_t n, int dc, uint64_t* primary_index,
            uint32_t flags) {
    if (!x || !primary_index) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        *primary_index = dcx::bwt_of_text(x->c, text, n, dc, bwt_out, flags);
    });
}

int dcx_build_bwt(dcx_ctx* x, const uint8_t* text, uint64_t n, const void* sa, int sa_width, uint8_t* bwt_out,
                  uint64_t* primary_index, uint32_t flags) {
    if (!x || !primary_index) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        *primary_index = dcx::build_bwt(x->c, text, n, sa, sa_width, bwt_out, flags);
    });
}

int dcx_check_sa(dcx_ctx* x, const uint8_t* text, uint64_t n, const void* sa, int sa_width, uint32_t flags,
                 int* ok) {
    if (!x || !ok) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        *ok = dcx::check_one(x->c, text, n, sa, sa_width, flags) ? 1 : 0;
    });
}

int dcx_write_sa_file(dcx_ctx* x, const char* path, const void* sa_dev, uint64_t n, int sa_width,
                      uint64_t chunk_bytes) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::write_sa_file(x->c, path, sa_dev, n, sa_width, chunk_bytes);
    });
}

int dcx_read_sa_file(dcx_ctx* x, const char* path, void* sa_dev, uint64_t n, int sa_width, uint64_t chunk_bytes) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::read_sa_file(x->c, path, sa_dev, n, sa_width, chunk_bytes);
    });
}

int dcx_check_sa_file(dcx_ctx* x, const uint8_t* text, uint64_t n, const char* path, int sa_width, uint32_t flags,
                      int* ok) {
    if (!x || !ok) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        *ok = dcx::check_sa_file(x->c, text, n, path, sa_width, flags) ? 1 : 0;
    });
}

int dcx_get_stream(dcx_ctx* x, void** out) {
    if (!x || !out) return DCX_ERR_ARG;
    *out = (void*)x->c.stream;
    return DCX_OK;
}

int dcx_get_stats(dcx_ctx* x, dcx_stats* out) {
    if (!x || !out) return DCX_ERR_ARG;
    *out = x->c.st;
    return DCX_OK;
}

int dcx_get_trace(dcx_ctx* x, uint64_t* m_out, uint32_t* names, uint8_t* unique, uint64_t cap) {
    if (!x) return DCX_ERR_ARG;
    const uint64_t m = x->c.trace_names.size();
    if (m_out) *m_out = m;
    if (names || unique) {
        if (cap < m) return DCX_ERR_ARG;
        if (names) memcpy(names, x->c.trace_names.data(), m * 4);
        if (unique) memcpy(unique, x->c.trace_uniq.data(), m);
    }
    return DCX_OK;
}

int dcx_sort_u32(dcx_ctx* x, uint32_t* const* keys_dev, uint32_t kw, uint32_t* vals_dev, uint64_t n) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::sort_u32(x->c, keys_dev, kw, vals_dev, n);
    });
}

int dcx_build_sa_u32(dcx_ctx* x, const uint32_t* text_dev, uint64_t n, uint64_t sigma, int dc, int sa_width,
                     void* sa_out_dev) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::build_u32(x->c, text_dev, n, sigma, dc, sa_width, sa_out_dev);
    });
}

int dcx_build_sa_batch(dcx_ctx* x, const uint8_t* texts, const uint64_t* offsets, uint32_t num_texts,
                       int dc_or_auto, int sa_width, void* sa_out, uint32_t flags) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::build_batch(x->c, texts, offsets, num_texts, dc_or_auto, sa_width, sa_out, flags);
    });
}
int dcx_set_batch_dc_table(dcx_ctx* x, const uint64_t* max_len, const int* dc, uint32_t count) {
    if (!x || (count && (!max_len || !dc))) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        std::vector<std::pair<uint64_t, uint32_t>> t;
        for (uint32_t i = 0; i < count; i++) {
            if (i && max_len[i] <= max_len[i - 1]) throw dcx::Error(DCX_ERR_ARG, "class bounds must ascend");
            if (dc[i] <= 0) throw dcx::Error(DCX_ERR_ARG, "unsupported difference cover");
            dcx::get_dc(x->c, (uint32_t)dc[i]);
            t.push_back({max_len[i], (uint32_t)dc[i]});
        }
        x->c.opt.batch_dc = t;
        x->c.opt.batch_items.clear();  // every class on the context's radix tile
    });
}

int dcx_get_batch_dc_table(dcx_ctx* x, uint64_t* max_len, int* dc, uint32_t capacity, uint32_t* count) {
    if (!x || !count) return DCX_ERR_ARG;
    std::lock_guard<std::mutex> lk(x->c.build_mu);
    const auto& t = x->c.opt.batch_dc;
    *count = (uint32_t)t.size();
    for (uint32_t i = 0; i < capacity && i < t.size(); i++) {
        if (max_len) max_len[i] = t[i].first;
        if (dc) dc[i] = (int)t[i].second;
    }
    return DCX_OK;
}

int dcx_get_batch_tile_table(dcx_ctx* x, uint32_t* tile_elems, uint32_t capacity, uint32_t* count) {
    if (!x || !count) return DCX_ERR_ARG;
    std::lock_guard<std::mutex> lk(x->c.build_mu);
    const auto& o = x->c.opt;
    *count = (uint32_t)o.batch_dc.size();
    for (uint32_t i = 0; i < capacity && i < o.batch_dc.size(); i++)
        if (tile_elems)
            tile_elems[i] = dcx::SORT_THREADS * (i < o.batch_items.size() ? o.batch_items[i] : o.radix_items);
    return DCX_OK;
}

int dcx_autotune_batch(dcx_ctx* x, const uint8_t* texts, const uint64_t* offsets, uint32_t num_texts,
                       const uint64_t* class_max_len, uint32_t num_classes, const int* candidates,
                       uint32_t num_candidates, uint32_t repeats, int* chosen_dc, double* ms_out) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->c.build_mu);
        DCX_CUDA(cudaSetDevice(x->c.device));
        dcx::autotune_batch(x->c, texts, offsets, num_texts, class_max_len, num_classes, candidates, num_candidates,
                            repeats, chosen_dc, ms_out);
    });
}

static dcx::Server& server_of(dcx_ctx* x) {
    std::lock_guard<std::mutex> lk(x->serve_mu);
    if (!x->server) {
        const dcx::Options& o = x->c.opt;
        const uint64_t budget = o.serve_budget ? o.serve_budget : x->c.budget;
        x->server = std::make_unique<dcx::Server>(x->c, (int)o.serve_lanes, budget, o.serve_batch_bytes,
                                                  o.serve_batch_texts, o.serve_host_bytes, o.serve_express_bytes,
                                                  o.serve_express_priority != 0);
    }
    return *x->server;
}

int dcx_serve_submit(dcx_ctx* x, const uint8_t* text, uint64_t n, int dc, int sa_width, uint64_t* req_id) {
    if (!x || !req_id) return DCX_ERR_ARG;
    return guarded([&] { *req_id = server_of(x).submit(text, n, dc, sa_width, 0); });
}

int dcx_serve_submit_ex(dcx_ctx* x, const uint8_t* text, uint64_t n, int dc, int sa_width, uint32_t flags,
                        uint64_t* req_id) {
    if (!x || !req_id) return DCX_ERR_ARG;
    return guarded([&] { *req_id = server_of(x).submit(text, n, dc, sa_width, flags); });
}

int dcx_serve_poll(dcx_ctx* x, uint64_t req_id, void* sa_host, int* status, double* latency_ms) {
    if (!x || !status) return DCX_ERR_ARG;
    return guarded([&] { server_of(x).poll(req_id, sa_host, status, latency_ms); });
}

int dcx_serve_result_device(dcx_ctx* x, uint64_t req_id, const void** sa_dev) {
    if (!x || !sa_dev) return DCX_ERR_ARG;
    return guarded([&] { *sa_dev = server_of(x).result_device(req_id); });
}

int dcx_serve_release(dcx_ctx* x, uint64_t req_id) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] { server_of(x).release(req_id); });
}

int dcx_serve_drain(dcx_ctx* x) {
    if (!x) return DCX_ERR_ARG;
    return guarded([&] {
        dcx::Server* sv;
        {
            std::lock_guard<std::mutex> lk(x->serve_mu);
            sv = x->server.get();
        }
        if (sv) sv->drain();
    });
}

int dcx_serve_get_stats(dcx_ctx* x, dcx_serve_stats* out) {
    if (!x || !out) return DCX_ERR_ARG;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(x->serve_mu);
        *out = x->server ? x->server->stats() : dcx_serve_stats{};
    });
}

}  // extern "C"
