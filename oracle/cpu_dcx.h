/* C interface of the CPU restatement of lightweight_dcx's PDCX (oracle).
 * TEST INFRASTRUCTURE ONLY: called by tests, the smoke check and bench.py's
 * CPU-baseline leg; never by the GPU product. */
#ifndef CPU_DCX_H
#define CPU_DCX_H
#include <stdint.h>

#define CPU_DCX_ERR_ARG (-1)
#define CPU_DCX_ERR_ALPHABET (-2)

typedef struct cpu_dcx_trace {
    /* level-0 observations */
    uint64_t m;            /* number of DC samples incl. the dummy sample */
    uint64_t last_rank;    /* highest lexicographic name (== m iff all distinct) */
    uint64_t sample_chars; /* chars per phase-1 sample key */
    uint64_t merge_chars;  /* chars per phase-4 tuple */
    int recursion;         /* 0 none, 1 direct, 2 with discarding */
    int max_depth;         /* recursion levels entered (1 = level 0 only) */
    int base_case;         /* 1 if level 0 was solved by the sequential base case */
    double reduction;      /* discarding reduction at level 0 */
    /* optional outputs in sample text order (slot = (i/X)*D + NEXT_RANK[i%X]) */
    uint64_t capacity;
    uint64_t* names;
    uint8_t* unique;
} cpu_dcx_trace;

int cpu_dcx_table(uint32_t X, uint32_t* D_out, uint32_t* dc_out, uint8_t* in_dc_out,
                  uint32_t* next_rank_out, uint32_t* cmp_out);
int cpu_compress_alphabet(uint8_t* text, uint64_t n, uint32_t* sigma_out);
void cpu_packing_for_sigma(uint32_t X, uint32_t sigma, uint32_t* bits, uint32_t* words);
int cpu_dcx_sa(const uint8_t* text, uint64_t n, uint32_t X, int pack_samples, int pack_merging,
               double discarding_threshold, uint64_t base_case_threshold, uint32_t sigma,
               uint64_t* sa_out, cpu_dcx_trace* trace);
int cpu_slow_sa(const uint8_t* text, uint64_t n, uint64_t* sa_out);
int cpu_dcx_threads(void);
#endif
