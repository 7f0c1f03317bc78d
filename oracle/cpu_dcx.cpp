// CPU restatement of lightweight_dcx's PDCX suffix-array construction.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle: tests, the smoke check
// and bench.py's CPU-baseline leg call it as a checker.  The GPU product never
// links, loads or calls it.
//
// It is a single-process (p = 1) restatement of the reference algorithm, step
// by step, so that intermediate arrays (level-0 lexicographic names, unique
// flags, recursion decisions) can be compared with the GPU build.  The final
// suffix array is unique for a text, so it is additionally pinned against
// libsais (built from the reference tree into oracle/_ref) and the golden SA
// files of the reference tree.
//
// Reference files followed (paths inside the reference project):
//   lightweight_dcx/src/executables/cli.cpp:417-463   compress_alphabet
//   lightweight_dcx/src/executables/cli.cpp:475-539   packing width / words
//   lightweight_dcx/src/pdcx/pdcx.hpp:465-510         lengths, dummy sample
//   lightweight_dcx/src/pdcx/pdcx.hpp:623-633         base case on root
//   lightweight_dcx/src/pdcx/sample_string.hpp:112-164,241-249  samples, padding
//   lightweight_dcx/src/pdcx/compute_ranks.hpp:49-56,89-134     names, unique
//   lightweight_dcx/src/pdcx/pdcx.hpp:83-94,112-462   recursion, discarding
//   lightweight_dcx/src/pdcx/merge_samples.hpp:87-109,181-260   phase-4 tuples
//   lightweight_dcx/src/util/string_util.hpp:86-106   slow_suffixarray
//   lightweight_dcx/src/strings/char_container.hpp:50-104,483-545 packing
//   lightweight_dcx/src/pdcx/difference_cover.hpp     DC sets (tables are
//                                                      regenerated in closed form)
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#ifdef ORACLE_PARALLEL
#include <omp.h>
#include <parallel/algorithm>
#define ORACLE_SORT __gnu_parallel::sort
#else
#define ORACLE_SORT std::sort
#endif

extern "C" {
#include "cpu_dcx.h"
}

namespace {

// ---------------------------------------------------------------------------
// Difference covers (the sets of difference_cover.hpp:14-5126) and the derived
// tables.  IN_DC, NEXT_RANK and cmpDepthRanks are generated from the set:
//   NEXT_RANK[r]        = |{c in DC : c < r}|
//   cmpDepthRanks[i][j] = (l, #DC positions in [i, i+l), #DC positions in [j, j+l))
//   with l = min{ l >= 0 : (i+l) mod X in DC and (j+l) mod X in DC }.
// ---------------------------------------------------------------------------
struct DcTable {
    uint32_t X = 0, D = 0;
    std::vector<uint32_t> dc;
    std::vector<uint8_t> in_dc;
    std::vector<uint32_t> next_rank;
    std::vector<uint32_t> cmp;  // [X][X][3]
};

bool dc_set_for(uint32_t X, std::vector<uint32_t>& out) {
    switch (X) {
        case 3: out = {1, 2}; return true;
        case 7: out = {1, 2, 4}; return true;
        case 13: out = {1, 2, 4, 10}; return true;
        case 21: out = {1, 2, 7, 9, 19}; return true;
        case 31: out = {1, 2, 4, 9, 13, 19}; return true;
        case 39: out = {1, 2, 17, 21, 23, 28, 31}; return true;
        case 57: out = {1, 2, 10, 12, 15, 36, 40, 52}; return true;
        case 73: out = {1, 2, 4, 8, 16, 32, 37, 55, 64}; return true;
        case 91: out = {1, 2, 8, 17, 28, 57, 61, 69, 71, 74}; return true;
        case 95: out = {1, 2, 6, 9, 19, 21, 30, 32, 46, 62, 68}; return true;
        case 133: out = {1, 2, 33, 43, 45, 49, 52, 60, 73, 78, 98, 112}; return true;
        default: return false;
    }
}

bool make_table(uint32_t X, DcTable& t) {
    if (!dc_set_for(X, t.dc)) return false;
    t.X = X;
    t.D = (uint32_t)t.dc.size();
    t.in_dc.assign(X, 0);
    for (uint32_t c : t.dc) t.in_dc[c] = 1;
    t.next_rank.assign(X, 0);
    for (uint32_t r = 0; r < X; r++) {
        uint32_t cnt = 0;
        for (uint32_t c : t.dc) cnt += c < r;
        t.next_rank[r] = cnt;
    }
    t.cmp.assign((size_t)X * X * 3, 0);
    for (uint32_t i = 0; i < X; i++) {
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
    }
    return true;
}

// ---------------------------------------------------------------------------
// Packed character containers: chars MSB-first in 64-bit words, `bits` per
// char, `words` words, zero-filled tail (char_container.hpp:50-104,483-545).
// Comparison is word-lexicographic.  Unpacked containers keep one char per
// slot and compare slot by slot (CharArray, char_container.hpp:14-48).
// ---------------------------------------------------------------------------
template <typename CharT>
void pack_chars(const CharT* first, uint64_t count, uint32_t bits, uint32_t words,
                uint64_t* out) {
    const uint32_t cpw = 64 / bits;
    const uint64_t mask = (bits == 64) ? ~0ull : ((1ull << bits) - 1);
    for (uint32_t k = 0; k < words; k++) {
        uint64_t v = 0;
        uint64_t lo = (uint64_t)k * cpw;
        uint64_t hi = std::min<uint64_t>((uint64_t)(k + 1) * cpw, count);
        uint32_t cnt = 0;
        for (uint64_t c = lo; c < hi; c++, cnt += bits) {
            v |= ((uint64_t)first[c] & mask) << (64 - bits - cnt);
        }
        out[k] = v;
    }
}

// slow_suffixarray (string_util.hpp:86-106): std::sort with substring compare,
// a shorter suffix that is a prefix of a longer one sorts first.
template <typename CharT>
std::vector<uint64_t> slow_suffixarray(const std::vector<CharT>& arr) {
    const int64_t m = (int64_t)arr.size();
    std::vector<uint64_t> sa(arr.size());
    std::iota(sa.begin(), sa.end(), 0);
    std::sort(sa.begin(), sa.end(), [&](uint64_t a, uint64_t b) {
        int64_t j = 0;
        while ((int64_t)a + j < m && (int64_t)b + j < m && arr[a + j] == arr[b + j]) j++;
        if ((int64_t)a + j == m) return true;
        if ((int64_t)b + j == m) return false;
        return arr[a + j] < arr[b + j];
    });
    return sa;
}

struct RankIndex {
    uint64_t rank;
    uint64_t index;
    bool unique;
};

struct Settings {
    double discarding_threshold;
    uint64_t base_case_threshold;
    int pack_samples;
    int pack_merging;
    uint32_t bits;   // packing width at level 0
    uint32_t words;  // packed words at level 0
};

struct Pdcx {
    const DcTable& dc;
    const Settings& cfg;
    cpu_dcx_trace* trace;

    Pdcx(const DcTable& d, const Settings& s, cpu_dcx_trace* t) : dc(d), cfg(s), trace(t) {}

    // pdcx.hpp:83-94
    static uint64_t map_back(uint64_t idx, const std::vector<uint64_t>& samples_before,
                             const DcTable& dc) {
        for (uint32_t i = 0; i < dc.D; i++) {
            if (idx < samples_before[i + 1]) {
                uint64_t k = idx - samples_before[i];
                return (uint64_t)dc.X * k + dc.dc[i];
            }
        }
        return 0;
    }

    template <typename CharT>
    std::vector<uint64_t> compute_sa(std::vector<CharT>& s, int depth) {
        const uint32_t X = dc.X, D = dc.D;
        const uint64_t n = s.size();
        if (trace && depth + 1 > trace->max_depth) trace->max_depth = depth + 1;

        // Base case: solve sequentially (pdcx.hpp:623-633 with p = 1).
        uint64_t threshold = std::max<uint64_t>(2ull * X, cfg.base_case_threshold);
        if (n <= threshold) {
            if (trace && depth == 0) trace->base_case = 1;
            return slow_suffixarray(s);
        }

        // Phase 0: lengths and the dummy sample (pdcx.hpp:473-510).
        const uint64_t rem = n % X;
        const bool dummy = dc.in_dc[rem] != 0;
        uint64_t m = 0;
        for (uint64_t i = 0; i < n; i++) m += dc.in_dc[i % X];
        m += dummy;
        std::vector<uint64_t> num_at_mod(X);
        for (uint64_t i = 0; i < X; i++) num_at_mod[i] = (n + X - 1 - i) / X;
        num_at_mod[rem] += dummy;
        std::vector<uint64_t> samples_before(D + 1, 0);
        for (uint32_t i = 1; i <= D; i++) samples_before[i] = samples_before[i - 1] + num_at_mod[dc.dc[i - 1]];

        // Packing only at depth 0 (pdcx.hpp:559-560); sample/merge char counts use the
        // reference's double arithmetic (sample_string.hpp:131-133, merge_samples.hpp:201).
        const bool packed_s = cfg.pack_samples && depth == 0;
        const bool packed_m = cfg.pack_merging && depth == 0;
        const bool packed_container = (cfg.pack_samples || cfg.pack_merging) && depth == 0;
        double ratio = 1.0;
        if (packed_container) ratio = (double)((uint64_t)cfg.words * (64 / cfg.bits)) / X;
        const double ratio_s = packed_s ? ratio : 1.0;
        const double ratio_m = packed_m ? ratio : 1.0;
        const uint64_t sample_chars = (uint64_t)(X * ratio_s);
        const uint64_t merge_chars = (uint64_t)(ratio_m * X - 1);
        const uint64_t padding = (uint64_t)(std::max(ratio_s, ratio_m) * X);

        // make_padding_and_shifts (sample_string.hpp:241-249).
        const uint64_t n_orig = n;
        s.resize(n + padding + 1, CharT(0));

        // Phase 1: materialise and sort samples by chars (sample_string.hpp:145-164,225-239).
        // Packed keys are materialised as words; unpacked keys (X chars followed by a 0
        // slot, CharArray<X+1>) are compared in place on the padded string.
        const uint32_t sw = packed_container ? cfg.words : 0;
        std::vector<uint64_t> skeys(m * sw, 0);
        std::vector<uint64_t> sidx(m);
        {
            uint64_t k = 0;
            for (uint64_t i = 0; i < n + dummy; i++) {
                if (!dc.in_dc[i % X]) continue;
                if (packed_container) pack_chars(&s[i], sample_chars, cfg.bits, cfg.words, &skeys[k * sw]);
                sidx[k++] = i;
            }
        }
        std::vector<uint64_t> order(m);
        std::iota(order.begin(), order.end(), 0);
        auto key_less = [&](uint64_t a, uint64_t b) {
            if (packed_container)
                return std::lexicographical_compare(&skeys[a * sw], &skeys[a * sw] + sw,
                                                    &skeys[b * sw], &skeys[b * sw] + sw);
            const CharT* pa = &s[sidx[a]];
            const CharT* pb = &s[sidx[b]];
            return std::lexicographical_compare(pa, pa + sample_chars, pb, pb + sample_chars);
        };
        auto key_eq = [&](uint64_t a, uint64_t b) {
            if (packed_container) return std::equal(&skeys[a * sw], &skeys[a * sw] + sw, &skeys[b * sw]);
            return std::equal(&s[sidx[a]], &s[sidx[a]] + sample_chars, &s[sidx[b]]);
        };
        ORACLE_SORT(order.begin(), order.end(), key_less);

        // Phase 2: lexicographic names and unique flags (compute_ranks.hpp:89-134).
        std::vector<RankIndex> ranks(m);
        {
            uint64_t prev = 0;
            for (uint64_t k = 0; k < m; k++) {
                ranks[k] = RankIndex{prev + 1, sidx[order[k]], false};
                if (k + 1 < m) prev += key_eq(order[k], order[k + 1]) ? 0 : 1;
            }
            auto distinct = [](uint64_t a, uint64_t b, uint64_t c) { return a != b && a != c; };
            for (uint64_t k = 0; k < m; k++) {
                uint64_t before = k > 0 ? ranks[k - 1].rank : 0;
                uint64_t after = k + 1 < m ? ranks[k + 1].rank : 0;
                ranks[k].unique = distinct(ranks[k].rank, before, after);
            }
        }
        skeys.clear();
        skeys.shrink_to_fit();

        const uint64_t last_rank = m ? ranks[m - 1].rank : 0;
        if (trace && depth == 0) {
            trace->m = m;
            trace->last_rank = last_rank;
            trace->sample_chars = sample_chars;
            trace->merge_chars = merge_chars;
            if (trace->names && trace->unique && trace->capacity >= m) {
                // in sample text order: the k-th sample in increasing position
                for (uint64_t k = 0; k < m; k++) {
                    uint64_t pos = ranks[k].index;
                    uint64_t slot = (pos / X) * D + dc.next_rank[pos % X];
                    trace->names[slot] = ranks[k].rank;
                    trace->unique[slot] = ranks[k].unique;
                }
            }
        }

        // Phase 3: recursion unless all names are distinct (pdcx.hpp:743-757).
        auto cmp_by_index = [](const RankIndex& a, const RankIndex& b) { return a.index < b.index; };
        if (last_rank >= m) {
            ORACLE_SORT(ranks.begin(), ranks.end(), cmp_by_index);
        } else {
            if (trace && depth == 0) trace->recursion = 1;
            recurse(ranks, samples_before, depth);
            ORACLE_SORT(ranks.begin(), ranks.end(), cmp_by_index);
        }

        // Phase 4: merge tuples (merge_samples.hpp:162-174,181-260,87-109).
        std::vector<uint64_t> sample_ranks(m + D, 0);
        for (uint64_t k = 0; k < m; k++) sample_ranks[k] = ranks[k].rank;
        ranks.clear();
        ranks.shrink_to_fit();

        const uint32_t mw = packed_container ? cfg.words : 0;
        std::vector<uint64_t> mkeys(n_orig * mw, 0);
        if (packed_container)
            for (uint64_t i = 0; i < n_orig; i++) pack_chars(&s[i], merge_chars, cfg.bits, cfg.words, &mkeys[i * mw]);
        auto rank_pos = [&](uint64_t i) { return (i / X) * D + dc.next_rank[i % X]; };
        std::vector<uint64_t> sa(n_orig);
        std::iota(sa.begin(), sa.end(), 0);
        auto merge_less = [&](uint64_t a, uint64_t b) {
            const uint32_t* e = &dc.cmp[((size_t)(a % X) * X + (b % X)) * 3];
            if (packed_container) {
                const uint64_t* ka = &mkeys[a * mw];
                const uint64_t* kb = &mkeys[b * mw];
                for (uint32_t w = 0; w < mw; w++)
                    if (ka[w] != kb[w]) return ka[w] < kb[w];
            } else {
                // first d of the X-1 materialised chars (merge_samples.hpp:96-102)
                for (uint32_t c = 0; c < e[0]; c++)
                    if (s[a + c] != s[b + c]) return s[a + c] < s[b + c];
            }
            return sample_ranks[rank_pos(a) + e[1]] < sample_ranks[rank_pos(b) + e[2]];
        };
        ORACLE_SORT(sa.begin(), sa.end(), merge_less);

        s.resize(n_orig);  // clean_up (pdcx.hpp:104-109)
        return sa;
    }

    // handle_recursive_call (pdcx.hpp:146-180) and its two variants.
    void recurse(std::vector<RankIndex>& ranks, const std::vector<uint64_t>& samples_before,
                 int depth) {
        const uint32_t X = dc.X;
        const uint64_t m = ranks.size();
        std::sort(ranks.begin(), ranks.end(), [X](const RankIndex& a, const RankIndex& b) {
            uint64_t am = a.index % X, bm = b.index % X;
            if (am != bm) return am < bm;
            return a.index / X < b.index / X;
        });

        // num_ranks_after_discarding (pdcx.hpp:215-228)
        uint64_t discarded = 0;
        for (uint64_t i = 1; i < m; i++) discarded += ranks[i].unique && ranks[i - 1].unique;
        const uint64_t after = m - discarded;
        const double reduction = (double)after / (double)m;
        const bool use_discarding = reduction <= cfg.discarding_threshold;
        if (trace && depth == 0) {
            trace->reduction = reduction;
            trace->recursion = use_discarding ? 2 : 1;
        }

        if (!use_discarding) {
            // recursive_call_direct (pdcx.hpp:183-212)
            std::vector<uint64_t> rec(m);
            for (uint64_t i = 0; i < m; i++) rec[i] = ranks[i].rank;
            std::vector<uint64_t> sa = compute_sa(rec, depth + 1);
            for (uint64_t k = 0; k < m; k++)
                ranks[k] = RankIndex{k + 1, map_back(sa[k], samples_before, dc), true};
            return;
        }

        // recursive_call_with_discarding (pdcx.hpp:231-462), non-bucketed branch
        std::vector<uint64_t> rec;
        std::vector<uint8_t> red_unique;
        rec.reserve(after);
        red_unique.reserve(after);
        rec.push_back(ranks[0].rank);
        red_unique.push_back(ranks[0].unique);
        for (uint64_t i = 1; i < m; i++) {
            bool drop = ranks[i].unique && ranks[i - 1].unique;
            if (!drop) {
                rec.push_back(ranks[i].rank);
                red_unique.push_back(ranks[i].unique);
            }
        }
        std::vector<uint64_t> rsa = compute_sa(rec, depth + 1);
        std::vector<uint64_t> rank_of(rsa.size());
        for (uint64_t k = 0; k < rsa.size(); k++) rank_of[rsa[k]] = k + 1;

        struct Rri {
            uint64_t r1, r2, index;
        };
        std::vector<Rri> rri(m);
        uint64_t ir = 0;
        for (uint64_t i = 0; i < m; i++) {
            uint64_t r2 = 0;
            if (!ranks[i].unique) {
                while (red_unique[ir]) ir++;
                r2 = rank_of[ir++];
            }
            rri[i] = Rri{ranks[i].rank, r2, ranks[i].index};
        }
        ORACLE_SORT(rri.begin(), rri.end(), [](const Rri& a, const Rri& b) {
            if (a.r1 != b.r1) return a.r1 < b.r1;
            return a.r2 < b.r2;
        });
        for (uint64_t k = 0; k < m; k++) ranks[k] = RankIndex{k + 1, rri[k].index, true};
    }
};

}  // namespace

extern "C" {

int cpu_dcx_table(uint32_t X, uint32_t* D_out, uint32_t* dc_out, uint8_t* in_dc_out,
                  uint32_t* next_rank_out, uint32_t* cmp_out) {
    DcTable t;
    if (!make_table(X, t)) return -1;
    if (D_out) *D_out = t.D;
    if (dc_out) std::memcpy(dc_out, t.dc.data(), t.D * sizeof(uint32_t));
    if (in_dc_out) std::memcpy(in_dc_out, t.in_dc.data(), X);
    if (next_rank_out) std::memcpy(next_rank_out, t.next_rank.data(), X * sizeof(uint32_t));
    if (cmp_out) std::memcpy(cmp_out, t.cmp.data(), t.cmp.size() * sizeof(uint32_t));
    return 0;
}

int cpu_compress_alphabet(uint8_t* text, uint64_t n, uint32_t* sigma_out) {
    uint64_t counts[256] = {0};
    for (uint64_t i = 0; i < n; i++) counts[text[i]]++;
    uint32_t sigma = 0;
    for (int c = 0; c < 256; c++) sigma += counts[c] > 0;
    if (sigma_out) *sigma_out = sigma;
    if (sigma == 256) return CPU_DCX_ERR_ALPHABET;  // cli.cpp:440-446
    uint8_t map[256] = {0};
    uint32_t next = 1;
    for (int c = 0; c < 256; c++)
        if (counts[c]) map[c] = (uint8_t)next++;
    for (uint64_t i = 0; i < n; i++) text[i] = map[text[i]];
    return 0;
}

void cpu_packing_for_sigma(uint32_t X, uint32_t sigma, uint32_t* bits, uint32_t* words) {
    // cli.cpp:488-533
    uint32_t b = sigma <= 7 ? 3 : (sigma <= 31 ? 5 : 8);
    uint32_t cpw = 64 / b;
    *bits = b;
    *words = (X + cpw - 1) / cpw;
}

int cpu_dcx_sa(const uint8_t* text, uint64_t n, uint32_t X, int pack_samples, int pack_merging,
               double discarding_threshold, uint64_t base_case_threshold, uint32_t sigma,
               uint64_t* sa_out, cpu_dcx_trace* trace) {
    DcTable dc;
    if (!make_table(X, dc)) return CPU_DCX_ERR_ARG;
    Settings cfg{};
    cfg.discarding_threshold = discarding_threshold;
    cfg.base_case_threshold = base_case_threshold;
    cfg.pack_samples = pack_samples;
    cfg.pack_merging = pack_merging;
    cpu_packing_for_sigma(X, sigma, &cfg.bits, &cfg.words);
    if (trace) {
        trace->m = 0;
        trace->last_rank = 0;
        trace->recursion = 0;
        trace->reduction = 0.0;
        trace->max_depth = 0;
        trace->base_case = 0;
        trace->sample_chars = 0;
        trace->merge_chars = 0;
    }
    std::vector<uint8_t> s(text, text + n);
    for (uint64_t i = 0; i < n; i++)
        if (s[i] == 0) return CPU_DCX_ERR_ARG;  // 0 is reserved for padding
    Pdcx p(dc, cfg, trace);
    std::vector<uint64_t> sa = p.compute_sa(s, 0);
    std::memcpy(sa_out, sa.data(), n * sizeof(uint64_t));
    return 0;
}

int cpu_slow_sa(const uint8_t* text, uint64_t n, uint64_t* sa_out) {
    std::vector<uint8_t> s(text, text + n);
    std::vector<uint64_t> sa = slow_suffixarray(s);
    std::memcpy(sa_out, sa.data(), n * sizeof(uint64_t));
    return 0;
}

int cpu_dcx_threads(void) {
#ifdef ORACLE_PARALLEL
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
