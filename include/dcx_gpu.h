/*
 * dcx_gpu.h -- C ABI of the B200 DCX suffix-array builder.
 *
 * The reference (lightweight_dcx of distributed_suffix_sorting_evaluation)
 * exposes its construction path through two surfaces, and this ABI covers both:
 *   - the library call  PDCX<char,index,DC>::compute_sa(std::vector<char>&)
 *     -> std::vector<index>   (lightweight_dcx/src/pdcx/pdcx.hpp:529), wrapped
 *     by run_pdcx / compute_sa (lightweight_dcx/src/executables/cli.cpp:465-472,655-689);
 *   - the `cli` process (cli.cpp:747-820), rebuilt on top of this ABI as
 *     `dcx_cli` with the same flags.
 * Its error model follows libsais64 (libsais/include/libsais64.h:61): 0 on
 * success, a negative code otherwise.  The library never exits the process and
 * never falls back to the CPU.
 *
 * Threading: a context serves one host thread for dcx_build_* calls.
 * dcx_serve_* calls are thread-safe (internal queue and worker thread).
 * Ownership: callers own every buffer they pass; a context never retains a
 * caller pointer beyond the call that received it.
 */
#ifndef DCX_GPU_H
#define DCX_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
#define DCX_OK 0
#define DCX_ERR_ARG (-1)      /* invalid argument (size, DC, width, null pointer) */
#define DCX_ERR_ALPHABET (-2) /* 256 distinct byte values with packing requested (cli.cpp:440-446) */
#define DCX_ERR_OOM (-3)      /* device allocation failed */
#define DCX_ERR_BUDGET (-4)   /* projected HBM footprint above the context budget */
#define DCX_ERR_TIMEOUT (-5)  /* a bounded device-side wait gave up (kernel returned cleanly) */
#define DCX_ERR_CUDA (-6)     /* CUDA runtime error */
#define DCX_ERR_INTERNAL (-7) /* internal consistency check failed */
#define DCX_ERR_BUSY (-8)     /* serving queue full or request not finished */
#define DCX_ERR_NOTFOUND (-9) /* unknown serving request id */
#define DCX_ERR_IO (-10)      /* a file could not be opened, read or written */

/* ---- flags for dcx_build_sa / dcx_build_sa_batch ---------------------------- */
#define DCX_HOST_PTRS 0u        /* text / sa_out are host pointers (pinned or pageable) */
#define DCX_DEVICE_PTRS 1u      /* text / sa_out are device pointers on the context's GPU */
#define DCX_NO_PACKING 2u       /* level-0 keys use X chars instead of the packed word width */
#define DCX_NO_REMAP 4u         /* text is already remapped to 1..sigma (skip compress_alphabet) */

/* SA output widths: 32 (uint32 LE), 40 (uint40 LE: low uint32 then high uint8,
 * the reference's on-disk format, util/uint_types.hpp:49-269 + mpi/io.hpp:80-98),
 * 64 (uint64 LE). */

typedef struct dcx_ctx dcx_ctx;

/* Per-build statistics (phase names follow pdcx.hpp:544,659,741,778). */
typedef struct dcx_stats {
    double ms_total;          /* device time of the whole build (CUDA events) */
    double ms_phase0;         /* preparation: alphabet remap, key materialisation */
    double ms_phase12;        /* phase 1 + 2: sample sort, naming */
    double ms_phase3;         /* recursion */
    double ms_phase4;         /* merge: tie-group sort and SA emission */
    double ms_h2d;            /* host->device copies (host-pointer calls) */
    double ms_d2h;            /* device->host copies (host-pointer calls) */
    uint64_t bytes_alg;       /* algorithmic bytes of all kernels (read + write, logical) */
    uint64_t bytes_radix;     /* algorithmic bytes of the radix-sort passes alone */
    double ms_radix;          /* device time of the radix-sort passes alone */
    uint64_t radix_passes;    /* radix passes executed (all levels) */
    uint64_t radix_keys;      /* sum over passes of keys moved */
    uint64_t kernel_launches; /* kernels launched by the build */
    uint64_t peak_bytes;      /* device memory high-water mark of the build */
    uint32_t levels;          /* recursion levels entered (1 = no recursion) */
    uint32_t sigma;           /* alphabet size after remapping */
    uint64_t level0_samples;  /* m at level 0 */
    uint64_t level0_last_rank;/* highest level-0 name (== m iff all distinct) */
    int level0_recursion;     /* 0 none, 1 direct, 2 discarding */
    double level0_reduction;  /* discarding reduction at level 0 */
    uint64_t tie_groups;      /* phase-4 tie groups (all levels) */
    uint64_t tie_elements;    /* elements in phase-4 tie groups (all levels) */
    uint64_t lookback_gave_up;/* radix-pass CTAs whose bounded look-back wait ran out */
    uint64_t pool_growth_bytes;/* device memory the allocation pool had to add during the build */
} dcx_stats;

/* ---- context --------------------------------------------------------------- */
/* Creates a context on `device` whose builds may hold at most hbm_budget_bytes
 * of device memory (0 = 90% of the free memory at creation). */
int dcx_ctx_create(dcx_ctx** out, int device, uint64_t hbm_budget_bytes);
int dcx_ctx_destroy(dcx_ctx* ctx);

/* Tuning knobs (pdcx/config.hpp:34-60 names where one exists):
 *   "discarding_threshold" (double, default 0.7),
 *   "recursion_dc"         (X used below level 0; 0 = same as level 0; default 3),
 *   "small_threshold"      (texts up to this length are solved by the in-CTA
 *                           base case; default 2048, max 2048),
 *   "prefix_chars"         (chars in the first radix sort; 0 = auto),
 *   "rec_prefix_words"     (key words of the first radix sort at recursion levels: 2 or 3;
 *                           default 3),
 *   "radix_tile"           (elements per tile of every radix pass: 4096, the default,
 *                           or 3072),
 *   "batch_tune_tiles"     (1 = dcx_autotune_batch also chooses the radix tile per class;
 *                           default 1),
 *   "trace"                (1 = keep level-0 names/unique flags for dcx_get_trace),
 *   "spin_limit"           (polls of a radix pass's look-back wait before it gives
 *                           up: the build then returns DCX_ERR_TIMEOUT and the
 *                           contents of its output buffer are undefined; default 2^24),
 *   "lookback_hold_tile"   (failure-detection test hook: this tile of every radix
 *                           pass never publishes its look-back status, so the next
 *                           tile's wait runs out; negative = off, the default). */
int dcx_set_option(dcx_ctx* ctx, const char* name, double value);

/* ---- single text ----------------------------------------------------------- */
/* PDCX::compute_sa for one text of n bytes.  `dc` is X in {3,7,13,21,31,39,57,73,
 * 91,95,133}.  Unless DCX_NO_REMAP, bytes are remapped to 1..sigma first (the
 * reference cli's compress_alphabet).  A text that uses all 256 byte values is
 * accepted and built with 257-symbol keys (the reference refuses it);
 * dcx_build_sa_strict reproduces the refusal.  sa_out receives n entries of
 * sa_width bits.  n must be < 2^32 - 1. */
int dcx_build_sa(dcx_ctx* ctx, const uint8_t* text, uint64_t n, int dc, int sa_width,
                 void* sa_out, uint32_t flags);
/* Same as dcx_build_sa but refuses a 256-symbol alphabet (cli.cpp:440-446). */
int dcx_build_sa_strict(dcx_ctx* ctx, const uint8_t* text, uint64_t n, int dc, int sa_width,
                        void* sa_out, uint32_t flags);

/* Checks on the GPU that sa (n entries of sa_width bits) is the suffix array of
 * text: a permutation of 0..n-1 whose adjacent entries i, j satisfy
 * (T[i], ISA[i+1]) < (T[j], ISA[j+1]) -- the conditions check_suffixarray
 * establishes with distributed sorts (lightweight_dcx/src/sa_check.hpp:56-184,
 * wired to `cli --check`, cli.cpp:700-727).  *ok = 1 if correct, 0 if not. */
int dcx_check_sa(dcx_ctx* ctx, const uint8_t* text, uint64_t n, const void* sa, int sa_width,
                 uint32_t flags, int* ok);

/* ---- SA files ---------------------------------------------------------------- */
/* The reference writes an SA as its entries back to back, little endian, no
 * header (write_data, lightweight_dcx/src/mpi/io.hpp:80-98; uint40 entries,
 * util/uint_types.hpp:49-269).  These move such a file between the disk and
 * device memory without a host copy of the whole SA: two pinned buffers of
 * chunk_bytes (0 = 64 MiB), the device<->host copy of one chunk overlapping the
 * file access of the other.  dcx_read_sa_file returns DCX_ERR_ARG for a file
 * shorter than n entries (longer files are read from the start);
 * DCX_ERR_IO when the file cannot be opened, read or written. */
int dcx_write_sa_file(dcx_ctx* ctx, const char* path, const void* sa_dev, uint64_t n, int sa_width,
                      uint64_t chunk_bytes);
int dcx_read_sa_file(dcx_ctx* ctx, const char* path, void* sa_dev, uint64_t n, int sa_width,
                     uint64_t chunk_bytes);
/* dcx_check_sa for an SA stored in such a file (e.g. the --output of the
 * reference's cli): the file is streamed to the device and checked there; the
 * text is a host or device pointer per flags.  *ok as for dcx_check_sa. */
int dcx_check_sa_file(dcx_ctx* ctx, const uint8_t* text, uint64_t n, const char* path, int sa_width,
                      uint32_t flags, int* ok);

/* ---- LCP ------------------------------------------------------------------- */
/* Longest-common-prefix array of a text and its suffix array (sa_width 32, 40
 * or 64 bits per entry): lcp_out[k] = lcp(SA[k], SA[k-1]), lcp_out[0] = 0, as
 * libsais64_plcp + libsais64_lcp (libsais/include/libsais64.h:236-263) compute
 * it; with DCX_LCP_PERMUTED the permuted array PLCP[i] = LCP[ISA[i]] instead.
 * lcp_width is 32 or 64.  No counterpart in lightweight_dcx, whose SA is the
 * usual input of this step.  Host or device pointers as for dcx_build_sa. */
#define DCX_LCP_PERMUTED 16
/* With DCX_LCP_GSA, sa is a generalized SA of a 0-separated string set
 * (dcx_build_gsa) and every separator is its own symbol: no common prefix runs
 * through one, as libsais64_plcp_gsa computes it (libsais/include/libsais64.h:
 * 245-253).  DCX_ERR_ARG unless text[n-1] = 0. */
#define DCX_LCP_GSA 32
int dcx_build_lcp(dcx_ctx* ctx, const uint8_t* text, uint64_t n, const void* sa, int sa_width,
                  void* lcp_out, int lcp_width, uint32_t flags);

/* ---- generalized SA ----------------------------------------------------------- */
/* Generalized suffix array of a string set, in the convention of
 * libsais64_gsa (libsais/include/libsais64.h:63-72): text holds the strings,
 * each followed by a 0 byte (text[n-1] = 0; no empty string, except that the
 * set may be the single byte 0), and sa_out receives all n suffixes ordered as
 * if every separator were its own symbol below every character, separators in
 * string order.  (The reference tree's other generalized-SA construction,
 * psac's prefix doubling over a distributed string set,
 * psac/include/suffix_array.hpp:283-380, needs MPI.)  `dc` and `sa_width` as for dcx_build_sa;
 * DCX_ERR_ARG for a set libsais64_gsa refuses.  Host or device pointers. */
int dcx_build_gsa(dcx_ctx* ctx, const uint8_t* text, uint64_t n, int dc, int sa_width, void* sa_out,
                  uint32_t flags);

/* ---- BWT ------------------------------------------------------------------- */
/* Burrows-Wheeler transform of a text from its SA, in the convention of
 * libsais64_bwt (libsais/include/libsais64.h:125-135): bwt_out[0..n) is the last
 * column of the sorted rotations of T$ without the sentinel's row
 * (bwt_out[0] = T[n-1], then T[SA[k]-1] for every SA[k] != 0 in SA order) and
 * *primary_index = 1 + the k with SA[k] = 0, where that row would stand (0 for
 * n = 0).  No counterpart in lightweight_dcx.  DCX_ERR_ARG when an SA entry is
 * >= n or the SA has not exactly one 0 (a permutation is not checked:
 * dcx_check_sa does that).  Host or device pointers as for dcx_build_sa. */
int dcx_build_bwt(dcx_ctx* ctx, const uint8_t* text, uint64_t n, const void* sa, int sa_width,
                  uint8_t* bwt_out, uint64_t* primary_index, uint32_t flags);
/* The same BWT straight from the text, as libsais64_bwt(T, U, A, n, 0, NULL)
 * returns it: the SA is built on the GPU with difference cover `dc` and not
 * returned.  Host or device pointers as for dcx_build_sa; DCX_NO_PACKING and
 * DCX_NO_REMAP act on the SA build as they do there. */
int dcx_bwt(dcx_ctx* ctx, const uint8_t* text, uint8_t* bwt_out, uint64_t n, int dc, uint64_t* primary_index,
            uint32_t flags);

/* The CUDA stream (cudaStream_t) every kernel of this context runs on, so a
 * caller can time builds with events recorded on it. */
int dcx_get_stream(dcx_ctx* ctx, void** stream_out);

/* Statistics of the last build on this context. */
int dcx_get_stats(dcx_ctx* ctx, dcx_stats* out);

/* Level-0 observations of the last build with option "trace" = 1: names and
 * unique flags of the m level-0 samples in sample text order
 * (slot = (i/X)*D + NEXT_RANK[i%X], pdcx/merge_samples.hpp:181-188). */
int dcx_get_trace(dcx_ctx* ctx, uint64_t* m_out, uint32_t* names, uint8_t* unique, uint64_t capacity);

/* ---- building blocks of the multi-GPU single-text build --------------------- */
/* The reference distributes one text over MPI ranks and sorts with a
 * distributed sample sort (lightweight_dcx/src/sorters/sample_sort.hpp:36-171,
 * mpi/alltoall.hpp:106-137); distributed.py does the same over
 * torch.distributed with these two device calls as its local steps.
 * dcx_sort_u32 sorts n pairs in place, stable, by kw (1..3) little-endian
 * uint32 key words (keys_dev[kw-1] most significant) carrying one uint32
 * value: the onesweep radix passes of every sort in this library (the local
 * sort that replaces ips4o in SortingWrapper::sort, sorters/sorting_wrapper.hpp:57-94).
 * Every array is a device buffer, 16-byte aligned; n < 2^32 - 1. */
int dcx_sort_u32(dcx_ctx* ctx, uint32_t* const* keys_dev, uint32_t kw, uint32_t* vals_dev, uint64_t n);
/* Suffix array of a device string of n uint32 symbols, each in [1, sigma]
 * (no 0: it marks the end), into the device buffer sa_out_dev (sa_width 32,
 * 40 or 64): the recursive call on the names of the samples
 * (PDCX::handle_recursive_call, pdcx/pdcx.hpp:146-180) when the recursion
 * string is gathered onto one GPU.  dc as for dcx_build_sa. */
int dcx_build_sa_u32(dcx_ctx* ctx, const uint32_t* text_dev, uint64_t n, uint64_t sigma, int dc, int sa_width,
                     void* sa_out_dev);

/* ---- batch ----------------------------------------------------------------- */
/* Builds one SA per text.  texts is the concatenation, offsets[num_texts+1] the
 * text boundaries (offsets[0] = 0).  sa_out receives, per text, its SA with
 * text-local indices, concatenated in the same layout as texts.  dc_or_auto = 0
 * takes X per size class from the table below (dcx_set_batch_dc_table /
 * dcx_autotune_batch; DC39 without one).  Every text must be < 2^32 - 1 bytes;
 * the concatenation may be larger than one build fits: it is split into rounds. */
int dcx_build_sa_batch(dcx_ctx* ctx, const uint8_t* texts, const uint64_t* offsets,
                       uint32_t num_texts, int dc_or_auto, int sa_width, void* sa_out,
                       uint32_t flags);

/* Size-class table of dcx_build_sa_batch with dc_or_auto = 0: a text longer
 * than the in-CTA base case uses dc[i] for the first i with length <=
 * max_len[i] (max_len ascending), DC39 when no class holds it; count = 0
 * restores DC39 for all.  The texts of each X are built as one group.  Any X
 * gives the same SAs; the table only changes the speed.  Serving lanes take the
 * table in force at the first dcx_serve_submit. */
int dcx_set_batch_dc_table(dcx_ctx* ctx, const uint64_t* max_len, const int* dc, uint32_t count);
/* Copies up to `capacity` entries of the table; *count = its length. */
int dcx_get_batch_dc_table(dcx_ctx* ctx, uint64_t* max_len, int* dc, uint32_t capacity, uint32_t* count);
/* Radix tile (elements per tile: 4096 or 3072) of every class of that table,
 * as the autotuner chose it; dcx_set_batch_dc_table resets every class to the
 * context's tile (option "radix_tile").  *count = the table's length. */
int dcx_get_batch_tile_table(dcx_ctx* ctx, uint32_t* tile_elems, uint32_t capacity, uint32_t* count);
/* Autotuner of that table.  The texts of a sample batch in HOST memory (layout
 * of dcx_build_sa_batch) are split into size classes (length in
 * (class_max_len[i-1], class_max_len[i]]); each class is built as one batch
 * with every candidate X, device-resident, one warm-up then `repeats` timed
 * runs (device time, median), and the fastest X of each class is installed as
 * the table.  chosen_dc[num_classes] receives the choices (0 for a class
 * without sample texts, which keeps DC39); ms_out[num_classes *
 * num_candidates] (may be null) the medians in ms (-1 for such a class).  With
 * the option "batch_tune_tiles" (default 1) the chosen X of each class is also
 * timed with the other radix tile (3072 against 4096 elements), and the faster
 * tile is installed beside it (dcx_get_batch_tile_table).  No counterpart in
 * the reference, whose cli takes --dcx per run. */
int dcx_autotune_batch(dcx_ctx* ctx, const uint8_t* texts, const uint64_t* offsets, uint32_t num_texts,
                       const uint64_t* class_max_len, uint32_t num_classes, const int* candidates,
                       uint32_t num_candidates, uint32_t repeats, int* chosen_dc, double* ms_out);

/* Splits a batch of independent texts over `world` GPUs, one process per GPU.
 * The reference splits its single text into equal blocks per rank
 * (lightweight_dcx/src/mpi/io.hpp:33-65); independent texts need no
 * exchange, so each rank takes whole texts instead.  Size-balanced, longest
 * first: texts in order of decreasing length (equal lengths: lower index
 * first) each go to the rank with the least text so far (equal loads: lower
 * rank).  owner[i] receives the rank of text i and load_out[r] (may be null)
 * the bytes of rank r.  The assignment depends only on the lengths, so every
 * rank computes the same split without a collective; the largest load is at
 * most 4/3 of the best possible (Graham's bound for longest-first
 * scheduling).  Host-only, needs no GPU.  DCX_ERR_ARG for world = 0 or null
 * owner / lengths with num_texts > 0. */
int dcx_shard_texts(const uint64_t* lengths, uint32_t num_texts, uint32_t world, uint32_t* owner,
                    uint64_t* load_out);

/* ---- serving (continuous batching) ----------------------------------------- */
/* No counterpart in the reference (its cli builds one SA per run,
 * cli.cpp:747-820).  A request loop on the context's GPU: requests are copied
 * at submission and queued in arrival order; `serve_lanes` worker lanes (each
 * its own stream) take the queued requests of one (dc, sa_width) class, first
 * come first served, while their projected HBM footprint fits the serving
 * budget, and build them as one batch (dcx_build_sa_batch semantics).  A lane
 * that finishes takes whatever has arrived meanwhile, so new requests overlap
 * on the device with the batches of the other lanes.  Results stay on the
 * device (and count against the budget) until released.  Every result equals
 * the SA of its text built alone.  All dcx_serve_* calls are thread-safe. */
typedef struct dcx_serve_stats {
    uint32_t lanes;
    uint64_t budget_bytes;        /* serving HBM budget */
    uint64_t reserved_bytes;      /* projected bytes of running batches + unreleased results */
    uint64_t peak_reserved_bytes; /* high-water mark of reserved_bytes */
    uint64_t peak_lane_bytes;     /* largest scratch high-water mark a lane measured in one batch */
    uint64_t submitted, done, failed;
    uint64_t done_bytes;          /* text bytes of finished requests */
    uint64_t batches;             /* batches started */
    uint64_t max_batch_texts;     /* most requests in one batch */
    uint64_t queued;              /* requests waiting now */
    uint32_t running_batches;     /* batches on the GPU now */
    double ms_upload;             /* summed over batches: host -> device copies of the texts */
    double ms_build;              /* summed over batches: the builds */
} dcx_serve_stats;

/* Queues an SA request (dc = 0: DC39; sa_width 32, 40 or 64).  Returns
 * DCX_ERR_BUDGET if its projected footprint can never fit the budget.  The
 * serving budget is the option "serve_budget" (bytes; 0 = the context budget),
 * read when the first request starts the server, as are "serve_lanes"
 * (default 1), "serve_batch_bytes" (text bytes per batch, default 1 GiB) and
 * "serve_batch_texts" (requests per batch, default 65536),
 * "serve_host_bytes" (pinned host memory for request copies, default 8 GiB;
 * requests that do not fit it are copied to pageable memory) and
 * "serve_express_bytes" (default 4 MiB): lane 0 serves the requests longer
 * than this (all requests when it is the only lane), uploading its next batch
 * while it builds the current one; the other lanes, on high-priority streams,
 * serve the shorter ones in batches of at most 4x it.  A text of 32 MiB or more
 * is always built in a batch of its own.  Each class is served in
 * arrival order, long builds run one at a time and short requests do not wait
 * behind them. */
int dcx_serve_submit(dcx_ctx* ctx, const uint8_t* text, uint64_t n, int dc, int sa_width,
                     uint64_t* req_id);
/* dcx_serve_submit with flags: DCX_SERVE_BORROW skips the copy at submission --
 * the caller keeps `text` valid and unchanged until the request is done (or
 * failed); with DCX_SERVE_BORROW | DCX_DEVICE_PTRS the text is a device buffer. */
#define DCX_SERVE_BORROW 8
int dcx_serve_submit_ex(dcx_ctx* ctx, const uint8_t* text, uint64_t n, int dc, int sa_width,
                        uint32_t flags, uint64_t* req_id);
/* Polls a request: *status = 0 queued, 1 running, 2 done, <0 failed (error code).
 * When done and sa_host is non-null, copies the SA (n entries of sa_width bits)
 * into sa_host.  latency_ms (optional) receives the submit -> done time (done =
 * SA complete in device memory). */
int dcx_serve_poll(dcx_ctx* ctx, uint64_t req_id, void* sa_host, int* status, double* latency_ms);
/* Device address of a finished request's SA (valid until released). */
int dcx_serve_result_device(dcx_ctx* ctx, uint64_t req_id, const void** sa_dev);
/* Frees a finished (or failed) request and its result; DCX_ERR_BUSY while it
 * is queued or running, DCX_ERR_NOTFOUND for unknown ids. */
int dcx_serve_release(dcx_ctx* ctx, uint64_t req_id);
/* Blocks until no request is queued or running.  Returns DCX_ERR_BUDGET instead
 * of waiting forever when nothing runs and the first queued request cannot be
 * admitted until results are released. */
int dcx_serve_drain(dcx_ctx* ctx);
int dcx_serve_get_stats(dcx_ctx* ctx, dcx_serve_stats* out);

/* ---- allocation-free entry point ----------------------------------------- */
/* No counterpart in the reference.  Suffix array of a device-resident text of
 * at most 32768 bytes, written as uint32 indices to the device buffer sa_dev,
 * launched on `stream` (a cudaStream_t; 0 = legacy default stream) and
 * returning without waiting for it.  It never allocates: it is meant for
 * callers that cannot call cudaMalloc where they need the result (inside stream
 * capture, inside an allocator, or with all device memory already reserved by
 * another pool).  All working memory is one 512 KiB device array that every GPU
 * loading this library holds until the process exits.  The first call on a
 * device looks that array's address up (cudaGetSymbolAddress) with the device
 * current, so make it before any stream capture.  Every call reuses the same
 * array: calls whose kernels overlap on the GPU race, so serialise them (one
 * stream, or events).  Returns DCX_ERR_ARG for n > 32768 or null pointers. */
int dcx_build_sa_noalloc(const uint8_t* text_dev, uint64_t n, uint32_t* sa_dev, void* stream);

/* ---- misc ------------------------------------------------------------------ */
const char* dcx_strerror(int code);
/* Difference-cover tables generated in closed form (pdcx/difference_cover.hpp):
 * fills D, DC[D], NEXT_RANK[X] and cmpDepthRanks[X][X][3]; returns DCX_ERR_ARG
 * for an unsupported X.  Host-only, needs no GPU. */
int dcx_dc_table(int X, uint32_t* D, uint32_t* dc, uint32_t* next_rank, uint32_t* cmp_depth_ranks);
/* Library version string. */
const char* dcx_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DCX_GPU_H */
