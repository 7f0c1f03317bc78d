// Runs the library's LCP/BWT/GSA kernels on the host through cuda_shim.h: the
// kernel headers are compiled unchanged (tests/test_kernels_on_host.py copies
// them beside a common.cuh that holds only store_sa_entry), and the host steps
// of build_bwt / build_lcp / build_gsa (distributed_suffix_sorting_evaluation_b200/csrc/dcx.cu)
// are restated around them: the device scan as a sequential loop, the tie
// compaction (OpTied) and the (run, position) radix sort as a loop and
// std::sort.
#include <algorithm>
#include <cstdlib>
#include <vector>
#include "bwt.cuh"
#include "gsa.cuh"
using namespace dcx;

static const unsigned G = 3, B = 7;  // odd launch shapes: every grid-stride loop wraps

static uint8_t* padded(const uint8_t* text, uint64_t n) {
    uint8_t* t = (uint8_t*)aligned_alloc(16, ((n + 16 + 15) / 16) * 16);
    memset(t, 0, ((n + 16 + 15) / 16) * 16);
    memcpy(t, text, n);
    return t;
}

extern "C" int kshim_bwt(const uint8_t* text, uint64_t n, const void* sa, int width, uint8_t* out, uint64_t* primary) {
    if (n == 0) { *primary = 0; return 0; }
    BwtScan st{~0ull, 0, 0};
    LAUNCH(k_bwt_primary, G, B, sa, width, n, &st);
    if (st.out_of_range || st.zeros != 1) return -1;
    const uint64_t p = st.first_zero + 1;
    LAUNCH(k_bwt_gather, G, B, text, n, sa, width, p, out);
    *primary = p;
    return 0;
}

static void separators(const uint8_t* t, uint64_t n, std::vector<uint32_t>& zb, std::vector<uint32_t>& sep) {
    zb.assign(n, 0);
    sep.assign(n + 1, 0);
    OpSeparators op{t, zb.data(), sep.data()};
    uint32_t ex = 0;
    for (uint64_t k = 0; k < n; k++) { uint32_t v = op.load(k); op.store(k, ex, v); ex += v; }
}

extern "C" int kshim_gsa(const uint8_t* text, uint64_t n, const uint32_t* plain_sa, uint32_t* out) {
    if (n == 0) return 0;
    uint8_t* t = padded(text, n);
    unsigned long long bad = 0;
    LAUNCH(k_gsa_check, G, B, t, n, &bad);
    if (bad) { free(t); return -1; }
    if (n == 1) { out[0] = 0; free(t); return 0; }
    std::vector<uint32_t> sa32(plain_sa, plain_sa + n), zb, sep, phi(n), plcp(n);
    separators(t, n, zb, sep);
    LAUNCH(k_phi, G, B, sa32.data(), n, phi.data());
    LAUNCH(k_plcp_to_separator, G, B, t, n, phi.data(), zb.data(), sep.data(), plcp.data(), 1u);
    std::vector<uint8_t> head(n);
    LAUNCH(k_gsa_heads, G, B, sa32.data(), n, plcp.data(), zb.data(), sep.data(), head.data());
    // tie compaction (OpTied's outputs) and the (run, position) sort, restated
    std::vector<uint32_t> slot;
    std::vector<std::pair<uint32_t, uint32_t>> key;
    uint32_t grp = 0;
    for (uint64_t k = 0; k < n; k++) {
        grp += head[k];
        const uint32_t nh = k + 1 < n ? head[k + 1] : 1;
        if (!(head[k] && nh)) { slot.push_back((uint32_t)k); key.push_back({grp, sa32[k]}); }
    }
    std::sort(key.begin(), key.end());
    std::vector<uint32_t> pos(key.size());
    for (size_t j = 0; j < key.size(); j++) pos[j] = key[j].second;
    const uint64_t cnt = slot.size();
    if (cnt) LAUNCH(k_gsa_scatter, G, B, cnt, slot.data(), pos.data(), sa32.data());
    LAUNCH(k_store_sa, G, B, sa32.data(), n, (void*)out, 32);
    free(t);
    return 0;
}

// uint32 SA entries written at any width (k_store_sa / store_sa_entry).
extern "C" int kshim_store_sa(const uint32_t* sa32, uint64_t n, void* out, int width) {
    LAUNCH(k_store_sa, G, B, sa32, n, out, width);
    return 0;
}

// The SA of any width to uint32 (k_sa_to_u32: 40-bit entries four at a time).
extern "C" int kshim_sa_to_u32(const void* sa, int width, uint64_t n, uint32_t* out) {
    LAUNCH(k_sa_to_u32, G, B, sa, width, n, out);
    return 0;
}

extern "C" int kshim_lcp(const uint8_t* text, uint64_t n, const uint32_t* sa, int gsa, uint32_t* lcp_out) {
    if (n == 0) return 0;
    uint8_t* t = padded(text, n);
    std::vector<uint32_t> phi(n), plcp(n), zb, sep;
    LAUNCH(k_phi, G, B, sa, n, phi.data());
    if (gsa) {
        if (t[n - 1] != 0) { free(t); return -1; }
        separators(t, n, zb, sep);
        LAUNCH(k_plcp_to_separator, G, B, t, n, phi.data(), zb.data(), sep.data(), plcp.data(), 0u);
    } else {
        LAUNCH(k_plcp, G, B, t, n, phi.data(), plcp.data());
    }
    LAUNCH(k_lcp_gather, G, B, sa, plcp.data(), n, (void*)lcp_out, 32, false);
    free(t);
    return 0;
}
