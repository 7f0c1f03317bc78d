// Seeded synthetic text generators for the benchmark workloads (no public corpus
// is used; every input is regenerated bit-identically from its seed).
//   iid       : i.i.d. uniform over an alphabet (e.g. {A,C,G,T})
//   markov    : order-3 Markov chain over {A,C,G,T} with random transition rows,
//               then a fraction of positions overwritten by copies of earlier
//               segments (log-uniform lengths) with point substitutions
//   pangenome : copies of one i.i.d. base with substitutions and short indels,
//               joined by '$', cut to the requested length
//   zipf      : i.i.d. Zipf(s) over 256 byte values
// Long sequential chains are cut into independently seeded chunks so that all
// host cores generate in parallel; the output depends only on (seed, n).
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {  // splitmix64; the seed is hashed so that nearby seeds give unrelated streams
    uint64_t s;
    explicit Rng(uint64_t seed) : s(mix64(mix64(seed + 0x9E3779B97F4A7C15ull) ^ 0xD1B54A32D192ED03ull)) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t k) { return (uint64_t)(uniform() * (double)k) % k; }
};

const uint8_t DNA[4] = {'A', 'C', 'G', 'T'};
constexpr uint64_t CHUNK = 1ull << 22;

}  // namespace

extern "C" {

void tg_iid(uint8_t* out, uint64_t n, const uint8_t* alphabet, uint32_t k, uint64_t seed) {
    const uint64_t chunks = (n + CHUNK - 1) / CHUNK;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < (int64_t)chunks; c++) {
        Rng r(seed * 1000003ull + (uint64_t)c);
        const uint64_t lo = (uint64_t)c * CHUNK, hi = std::min(n, lo + CHUNK);
        for (uint64_t i = lo; i < hi; i++) out[i] = alphabet[r.next() % k];
    }
}

// order-3 Markov chain over {A,C,G,T}; each row drawn from Dirichlet(4,4,4,4)
// (Gamma(4) = sum of four exponentials), entropy rate about 1.87 bits per base
void tg_markov(uint8_t* out, uint64_t n, uint64_t seed) {
    double cum[64][4];
    Rng r(seed);
    for (int s = 0; s < 64; s++) {
        double w[4], tot = 0;
        for (int j = 0; j < 4; j++) {
            w[j] = 0;
            for (int g = 0; g < 4; g++) w[j] += -std::log(1.0 - r.uniform());
            tot += w[j];
        }
        double acc = 0;
        for (int j = 0; j < 4; j++) {
            acc += w[j] / tot;
            cum[s][j] = acc;
        }
        cum[s][3] = 1.0;
    }
    const uint64_t chunks = (n + CHUNK - 1) / CHUNK;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < (int64_t)chunks; c++) {
        Rng g(seed * 7919ull + 17ull + (uint64_t)c);
        const uint64_t lo = (uint64_t)c * CHUNK, hi = std::min(n, lo + CHUNK);
        uint32_t state = (uint32_t)(g.next() & 63);
        for (uint64_t i = lo; i < hi; i++) {
            const double u = g.uniform();
            uint32_t x = 0;
            while (x < 3 && u > cum[state][x]) x++;
            out[i] = DNA[x];
            state = ((state << 2) | x) & 63;
        }
    }
}

// Overwrites about frac*n positions with copies of earlier segments whose
// lengths are log-uniform in [lmin, lmax]; each copied char is substituted by a
// different base with probability sub.  Returns the number of copied chars.
uint64_t tg_repeats(uint8_t* out, uint64_t n, double frac, uint64_t lmin, uint64_t lmax, double sub,
                    uint64_t seed) {
    Rng r(seed ^ 0x5EEDull);
    const uint64_t target = (uint64_t)(frac * (double)n);
    uint64_t covered = 0;
    if (n < 2 * lmin) return 0;
    while (covered < target) {
        const double lg = std::log((double)lmin) + r.uniform() * (std::log((double)lmax) - std::log((double)lmin));
        uint64_t len = (uint64_t)std::exp(lg);
        len = std::min(len, n / 2);
        const uint64_t dst = len + r.below(n - 2 * len + 1);
        const uint64_t src = r.below(dst - len + 1);
        for (uint64_t i = 0; i < len; i++) {
            uint8_t ch = out[src + i];
            if (r.uniform() < sub) {
                uint8_t alt;
                do alt = DNA[r.next() & 3]; while (alt == ch);
                ch = alt;
            }
            out[dst + i] = ch;
        }
        covered += len;
    }
    return covered;
}

// Pangenome-like text: i.i.d. base of base_len, then mutated copies joined by '$'.
void tg_pangenome(uint8_t* out, uint64_t n, uint64_t base_len, double sub, double indel, uint64_t seed) {
    std::vector<uint8_t> base(base_len);
    tg_iid(base.data(), base_len, DNA, 4, seed);
    Rng r(seed ^ 0xC0FFEEull);
    uint64_t pos = 0;
    while (pos < n) {
        for (uint64_t i = 0; i < base_len && pos < n; i++) {
            const double u = r.uniform();
            if (u < sub) {
                uint8_t alt;
                do alt = DNA[r.next() & 3]; while (alt == base[i]);
                out[pos++] = alt;
            } else if (u < sub + indel * 0.5) {
                i += 1 + r.below(10);  // deletion of 1..10 chars
            } else if (u < sub + indel) {
                uint64_t k = 1 + r.below(10);  // insertion of 1..10 chars
                for (uint64_t j = 0; j < k && pos < n; j++) out[pos++] = DNA[r.next() & 3];
                if (pos < n) out[pos++] = base[i];
            } else {
                out[pos++] = base[i];
            }
        }
        if (pos < n) out[pos++] = '$';
    }
}

// i.i.d. Zipf(s) over byte values 0..255 (rank k+1 has weight (k+1)^-s; rank 1 = byte 0)
void tg_zipf(uint8_t* out, uint64_t n, double s, uint64_t seed) {
    double cum[256];
    double tot = 0;
    for (int k = 0; k < 256; k++) {
        tot += std::pow((double)(k + 1), -s);
        cum[k] = tot;
    }
    for (int k = 0; k < 256; k++) cum[k] /= tot;
    cum[255] = 1.0;
    const uint64_t chunks = (n + CHUNK - 1) / CHUNK;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < (int64_t)chunks; c++) {
        Rng g(seed * 104729ull + 3ull + (uint64_t)c);
        const uint64_t lo = (uint64_t)c * CHUNK, hi = std::min(n, lo + CHUNK);
        for (uint64_t i = lo; i < hi; i++) {
            const double u = g.uniform();
            out[i] = (uint8_t)(std::lower_bound(cum, cum + 256, u) - cum);
        }
    }
}

// Log-uniform lengths in [lmin, lmax].
void tg_loguniform_lengths(uint64_t* out, uint64_t count, uint64_t lmin, uint64_t lmax, uint64_t seed) {
    Rng r(seed ^ 0x1E9ull);
    const double a = std::log((double)lmin), b = std::log((double)lmax);
    for (uint64_t i = 0; i < count; i++) out[i] = (uint64_t)std::exp(a + r.uniform() * (b - a));
}

int tg_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
