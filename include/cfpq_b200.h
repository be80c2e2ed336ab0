/*
 * cfpq_b200.h -- C ABI of the B200 CFPQ closure engine (libcfpq_b200.so).
 *
 * The reference crosses from its C++ driver to the GPU through C++ namespaces
 * (gpu_lib:: in cuda/naive-gpu/Multiplication.h:7-28, gpu_m4ri:: in
 * cuda/methodOf4RusBooleanSemiringGpu/gpuMemoryManagement.h:7-33 and
 * methodOf4RusBooleanSemiringGpu.h:53-54) behind the Matrix / MatricesEnv
 * plug-in interface (cfpq-cpp/Matrix.h:7-37).  This header replaces that
 * boundary with plain C entry points: opaque handles, plain pointers and sizes,
 * integer status codes.  Each entry point names the reference function it
 * replaces.
 *
 * Matrices are n x n Boolean matrices that live on the device for their whole
 * life.  The host exchange format ("row bits") is row-major, ceil(n/64) 64-bit
 * words per row, column c of a row at bit c % 64 of word c / 64 (LSB first).
 *
 * Errors: every entry point returns CFPQ_OK (0) or a cfpq_status code and never
 * exits the process or writes to stderr (the reference prints and calls exit(),
 * cuda/naive-gpu/Multiplication.cu:10-17).  cfpq_last_error() returns a
 * description of the last failure on the calling thread.
 *
 * Threading: a context may be used by one host thread at a time.  All work of
 * a context is issued on its own CUDA stream.
 */
#ifndef CFPQ_B200_H
#define CFPQ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFPQ_B200_ABI_VERSION 2

typedef enum cfpq_status {
    CFPQ_OK = 0,
    CFPQ_ERR_INVALID = 1,      /* bad argument (null handle, index out of range, size mismatch) */
    CFPQ_ERR_CUDA = 2,         /* a CUDA runtime call or a kernel failed */
    CFPQ_ERR_OOM = 3,          /* device or pinned host allocation failed */
    CFPQ_ERR_UNSUPPORTED = 4,  /* requested variant or size not supported */
    CFPQ_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
    CFPQ_ERR_IO = 6            /* a file could not be read or written */
} cfpq_status;

/* Product variants (kernels) for one rule product C |= A * B. */
typedef enum cfpq_variant {
    CFPQ_VARIANT_AUTO = 0,   /* the engine's selector picks per product */
    CFPQ_VARIANT_PLAIN = 1,  /* dense word-level kernel, no tiles, no skipping */
    CFPQ_VARIANT_LOP3 = 2,   /* tiled word-level AND/OR kernel with bulk-copy staged panels */
    CFPQ_VARIANT_M4R = 3,    /* Four Russians with 8-bit lookup tables in shared memory */
    CFPQ_VARIANT_TC = 4,     /* exact tensor-core product (0/1 operands, int accumulators > 0) */
    CFPQ_VARIANT_NTSET = 5   /* cfpq_closure only: the whole closure as one n x n matrix of
                                nonterminal sets squared until it stops changing (the
                                formulation of the reference's single-matrix CUTLASS backend,
                                cuda/cutlass/CutlassMatrix.cu:290-316, rule encoding
                                cfpq-cpp/Grammar.cpp:63-75); at most 32 nonterminals (one
                                byte per cell up to 8) and n <= 16384 (<= 8192 above 8) */
} cfpq_variant;

/* Closure drivers. */
typedef enum cfpq_driver {
    CFPQ_DRIVER_ENGINE = 0,   /* device-resident semi-naive iterations, tile skipping,
                                 no host round trip per iteration */
    CFPQ_DRIVER_WORKLIST = 1  /* the reference's host worklist (cfpq-cpp/Grammar.h:58-69):
                                 one add_mul at a time, changed flag read back each time */
} cfpq_driver;

typedef struct cfpq_ctx cfpq_ctx;
typedef struct cfpq_matrix cfpq_matrix;

/* One CNF binary rule head -> body1 body2, as indices into the matrix array
 * passed to cfpq_closure (the reference's rules vector, cfpq-cpp/Grammar.h:98). */
typedef struct cfpq_rule {
    uint32_t head;
    uint32_t body1;
    uint32_t body2;
} cfpq_rule;

#define CFPQ_LOOP_HOST 0
#define CFPQ_LOOP_DEVICE 1
#define CFPQ_LOOP_GRAPH 2

typedef struct cfpq_closure_opts {
    int32_t driver;          /* cfpq_driver */
    int32_t variant;         /* cfpq_variant used for every product, or AUTO */
    int32_t max_iterations;  /* 0 = until the fixpoint */
    int32_t use_graph;       /* ENGINE driver, how the iterations are sequenced:
                                0 (CFPQ_LOOP_HOST)   kernels launched from a host loop
                                1 (CFPQ_LOOP_DEVICE) no host round trip: one persistent
                                   cooperative kernel for the whole fixpoint when every
                                   product is word-level, else the CUDA-graph loop
                                2 (CFPQ_LOOP_GRAPH)  one CUDA graph with a device-side
                                   while condition, one node per kernel */
    int32_t log_products;    /* CFPQ_LOG_* flags (cfpq_last_kernel_profile, cfpq_product_log) */
    int32_t wait_limit;      /* persistent kernel: polls of each bounded device wait (work-item
                                wait, grid barrier) before it gives up and the closure returns
                                CFPQ_ERR_TIMEOUT; 0 = default (about one second) */
    int32_t test_flags;      /* CFPQ_TEST_* hooks for testing the failure paths; 0 in normal use */
    int32_t reserved[1];
} cfpq_closure_opts;

/* Test hook: the persistent kernel's first grid barrier waits for one arrival
 * more than there are CTAs, so its bounded wait runs out.  The closure then
 * returns CFPQ_ERR_TIMEOUT with the matrices holding a subset of the fixpoint
 * (every bit set is a true result) and the context stays usable.  Nothing
 * faults: the wait is a bounded poll. */
#define CFPQ_TEST_STALL_BARRIER 1

typedef struct cfpq_closure_stats {
    uint32_t iterations;        /* ENGINE: device iterations run; WORKLIST: 0 */
    uint32_t reserved0;
    uint64_t products;          /* rule products launched (ENGINE: non-empty product terms) */
    uint64_t tile_triples;      /* 64x64x64 bit tile products executed */
    uint64_t work_items;        /* output blocks processed by product kernels */
    uint64_t dense_bitops;      /* sum over products of n^3 (dense-equivalent bit-MACs) */
    double device_ms;           /* device time of the closure (CUDA events) */
    uint64_t kernel_launches;   /* kernels launched by this call */
    uint64_t variant_items[5];  /* work items per cfpq_variant */
    uint64_t bytes_staged;      /* operand bytes staged global -> shared by product kernels */
    uint64_t out_words;         /* non-zero 64-bit result words merged into heads */
    uint64_t new_words;         /* result words that carried new bits */
} cfpq_closure_stats;

/* Measured device rates, the denominators of the word-level rooflines: a
 * register-only kernel of independent 3-input logic chains (the LOP3 pipe)
 * timed with CUDA events on the context's stream.  No reference counterpart. */
typedef struct cfpq_calibration {
    double logic_ops_per_s;       /* 32-bit logic instructions per second, whole GPU */
    double logic_ops_per_clk_sm;  /* the same per SM per clock at the nominal clock */
    double bitmac_per_s;          /* Boolean AND-OR pairs per second = 32 x logic_ops_per_s */
    double ms;                    /* duration of the timed kernel */
} cfpq_calibration;
int cfpq_calibrate(cfpq_ctx *ctx, cfpq_calibration *out);

/* Per-kernel device times of the last closure run with
 * opts->log_products & CFPQ_LOG_KERNELS (every launch bracketed by CUDA events
 * on the context's stream; the iteration loop then runs from the host instead
 * of a CUDA graph).  The delta clear and the iteration end are one kernel
 * (advance_*); iter_end_* stay zero. */
#define CFPQ_LOG_KERNELS 1
#define CFPQ_LOG_PRODUCTS 2
#define CFPQ_LOG_SELECTION 4 /* AUTO closures: keep the selector's features and choices (cfpq_product_log) */
typedef struct cfpq_kernel_profile {
    double plan_ms, product_ms, advance_ms, iter_end_ms;
    uint64_t plan_launches, product_launches, advance_launches, iter_end_launches;
} cfpq_kernel_profile;
int cfpq_last_kernel_profile(cfpq_ctx *ctx, cfpq_kernel_profile *out);

/* ---- context ------------------------------------------------------------ */

/* Replaces the implicit per-process CUDA state of the reference backends
 * (static gpuMatrix::N / tmp_matrix, cuda/naive-gpu/GpuMatrix.h:15-16;
 * MethodOf4RusMatricesEnv, methodOf4RusBooleanSemiringMatrix.h:11-26). */
int cfpq_ctx_create(int device, cfpq_ctx **out);
int cfpq_ctx_destroy(cfpq_ctx *ctx);
/* Waits for all work issued on the context's stream. */
int cfpq_ctx_synchronize(cfpq_ctx *ctx);
/* Number of SMs of the context's device. */
int cfpq_ctx_num_sms(const cfpq_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * work or timing events with the library's. */
void *cfpq_ctx_stream(const cfpq_ctx *ctx);
/* Description of the last error on this thread ("" if none). */
const char *cfpq_last_error(void);
/* Library ABI version (CFPQ_B200_ABI_VERSION). */
int cfpq_abi_version(void);

/* ---- vertex orders -------------------------------------------------------- */

/* A relabeling of the n vertices of one query, shared by its matrices:
 * perm[v] is the internal index of vertex v (perm is a permutation of 0..n-1).
 * A matrix created with an order stores bit (perm[r], perm[c]) for (r, c);
 * every entry point that takes or returns coordinates, row bits, hashes or
 * counts still works in original vertex ids, so results are identical to an
 * unordered matrix.  Products and closures need all operands to share one
 * order.  The order exists so that the bits of sparse results cluster into
 * few 64x64 tiles, which the engine skips when empty.  No reference
 * counterpart (the reference stores vertex v at index v,
 * cuda/naive-gpu/GpuMatrix.cpp:15-18). */
typedef struct cfpq_order cfpq_order;
int cfpq_order_create(cfpq_ctx *ctx, uint32_t n, const uint32_t *perm, cfpq_order **out);
int cfpq_order_destroy(cfpq_ctx *ctx, cfpq_order *order);
/* Host-side heuristic: suggests perm for a graph given as an edge list.  Keeps
 * the identity when most edges already join nearby vertex ids; otherwise
 * groups vertices by the set of labels on their incoming and outgoing edges
 * and orders each group breadth-first (seeds by decreasing degree). */
int cfpq_order_suggest(uint32_t n, const uint32_t *from, const uint32_t *label, const uint32_t *to,
                       size_t nedges, uint32_t *perm_out);

/* ---- graph files ----------------------------------------------------------- */

/* Edge list of a graph file in the reference's format: "from label to"
 * triples separated by whitespace, read until the first triple whose vertex
 * tokens are not decimal numbers of at most 4294967295 (the stream extraction
 * loop of cfpq-cpp/Graph.cpp:15 stops there too; a vertex token with a sign
 * or with trailing non-digits, such as "-2" or "2.0", ends the list here,
 * while the stream would still take its leading part); nvertices = max id + 1.
 * Labels are numbered by first appearance in the file. */
typedef struct cfpq_edge_list {
    uint32_t *from;       /* nedges source vertices */
    uint32_t *label;      /* nedges label ids, indices into labels */
    uint32_t *to;         /* nedges target vertices */
    size_t nedges;
    uint32_t nvertices;
    uint32_t nlabels;
    const char **labels;  /* nlabels NUL-terminated names (then a NULL) */
} cfpq_edge_list;
/* Parses a graph file with `threads` host threads (0 = all cores): the file is
 * cut at line starts and the chunks parsed in parallel (a layout with triples
 * across lines falls back to one sequential pass).  Replaces the iostream
 * loop of Graph::Graph (cfpq-cpp/Graph.cpp:11-20).  *out is freed with
 * cfpq_edge_list_free.  No GPU needed. */
int cfpq_graph_load(const char *path, int threads, cfpq_edge_list **out);
void cfpq_edge_list_free(cfpq_edge_list *e);

/* ---- matrices ----------------------------------------------------------- */

/* Allocates a zero n x n matrix on the device.  Replaces
 * gpu_lib::device_matrix_alloc + host_matrix_calloc
 * (cuda/naive-gpu/Multiplication.cu:103-119) and
 * gpu_m4ri::allocate_matrix_device (gpuMemoryManagement.cu:51-55). */
int cfpq_matrix_create(cfpq_ctx *ctx, uint32_t n, cfpq_matrix **out);
/* Same with a vertex order (order->n must equal n; order may be NULL). */
int cfpq_matrix_create_ordered(cfpq_ctx *ctx, uint32_t n, cfpq_order *order, cfpq_matrix **out);
int cfpq_matrix_destroy(cfpq_ctx *ctx, cfpq_matrix *m);
uint32_t cfpq_matrix_size(const cfpq_matrix *m);

/* Sets bits (rows[i], cols[i]) from host arrays; the arrays are copied to the
 * device and scattered there.  Replaces the per-bit Matrix::set_bit calls of the
 * driver's initialisation (cfpq-cpp/Grammar.h:41-45, gpuMatrix::set_bit
 * cuda/naive-gpu/GpuMatrix.cpp:15-18) followed by the H2D transfer of
 * environment_preprocessing (cuda/naive-gpu/GpuMatrix.cpp:56-64). */
int cfpq_matrix_set_bits(cfpq_ctx *ctx, cfpq_matrix *m, const uint32_t *rows,
                         const uint32_t *cols, size_t count);
/* Same, with the coordinate arrays already in device memory. */
int cfpq_matrix_set_bits_device(cfpq_ctx *ctx, cfpq_matrix *m, const uint32_t *d_rows,
                                const uint32_t *d_cols, size_t count);
/* Initialises all nonterminal matrices of a query from its edge list in one
 * host->device copy and one scatter kernel: edge e (from[e], label[e], to[e])
 * sets bit (from[e], to[e]) in every matrix listed for its label, where the
 * matrices of label l are label_mats[label_offsets[l] .. label_offsets[l+1]-1]
 * (indices into mats).  Labels >= nlabels are ignored, like graph labels that
 * no terminal rule derives.  Replaces the edge loop of
 * Grammar::intersection_with_graph (cfpq-cpp/Grammar.h:41-45) and the H2D
 * upload of environment_preprocessing (cuda/naive-gpu/GpuMatrix.cpp:56-64). */
int cfpq_load_edges(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, const uint32_t *from,
                    const uint32_t *label, const uint32_t *to, size_t nedges, const uint32_t *label_offsets,
                    const uint32_t *label_mats, uint32_t nlabels);
/* Same as cfpq_load_edges with from / label / to already in device memory
 * (label_offsets and label_mats stay host arrays).  Asynchronous on the
 * context's stream; out-of-range coordinates are reported by the next
 * synchronising call of the context. */
int cfpq_load_edges_device(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, const uint32_t *d_from,
                           const uint32_t *d_label, const uint32_t *d_to, size_t nedges,
                           const uint32_t *label_offsets, const uint32_t *label_mats, uint32_t nlabels);
/* Sets the diagonal (epsilon nonterminals, cfpq-cpp/Grammar.h:47-51). */
int cfpq_matrix_set_diagonal(cfpq_ctx *ctx, cfpq_matrix *m);
/* Clears all bits. */
int cfpq_matrix_clear(cfpq_ctx *ctx, cfpq_matrix *m);
/* Clear `count` matrices with one kernel that zeroes only their occupied
 * tiles (the occupancy invariant holds at every API boundary), so the cost
 * follows the number of set tiles, not n^2. */
int cfpq_matrices_clear(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t count);
/* Copies all bits of src into dst (same n). */
int cfpq_matrix_copy(cfpq_ctx *ctx, cfpq_matrix *dst, const cfpq_matrix *src);

/* Host row-bits exchange: n * ceil(n/64) words.  Replaces
 * gpu_lib::cpu_to_gpu_transfer_async / gpu_to_cpu_transfer_async
 * (cuda/naive-gpu/Multiplication.cu:125-131) and the host mirror that
 * Matrix::get_bit reads (cuda/naive-gpu/GpuMatrix.cpp:20-23). */
int cfpq_matrix_upload_rows(cfpq_ctx *ctx, cfpq_matrix *m, const uint64_t *host_rows);
int cfpq_matrix_download_rows(cfpq_ctx *ctx, const cfpq_matrix *m, uint64_t *host_rows);

/* Reference result line for one matrix: the polynomial row hash (bases 11 and
 * 13 modulo 1e9+7) and the number of set bits, computed on the device.
 * Replaces the O(n^2) get_bit loop of Grammar::print_results
 * (cfpq-cpp/Grammar.cpp:81-100). */
int cfpq_matrix_hash_count(cfpq_ctx *ctx, const cfpq_matrix *m, uint64_t *hash,
                           uint64_t *count);
/* Number of set bits only. */
int cfpq_matrix_count(cfpq_ctx *ctx, const cfpq_matrix *m, uint64_t *count);

/* Result line (hash, count) of an n x n answer matrix that the caller keeps in
 * its own device memory as row bits (n rows of ceil(n/64) words, column c at
 * bit c % 64 of word c / 64), without allocating any memory.  No counterpart
 * in the reference.  It is for callers that cannot call cudaMalloc: hosts
 * whose own pool allocator owns the device memory, and latency-sensitive loops
 * that cannot take the device synchronisation an allocation may cause.  The
 * caller passes the input rows and d_out, a device buffer of two 64-bit words
 * that receives (hash, count).  Asynchronous on `stream` (a cudaStream_t, NULL
 * = the default stream) of `device`.  Scratch memory is a fixed device array
 * in the library sized for n <= CFPQ_NOALLOC_MAX_N; larger n is rejected with
 * CFPQ_ERR_UNSUPPORTED.  The first call on a device looks that array up (and
 * so does the first call in another CUDA context of the device, e.g. after
 * cudaDeviceReset), so make it before any stream capture.  All calls on a device share the array:
 * calls that overlap on the GPU race and must be ordered by the caller.
 * Errors are described by cfpq_noalloc_last_error(). */
#define CFPQ_NOALLOC_MAX_N 65536u
int cfpq_hash_count_rows_noalloc(int device, const uint64_t *d_rows, uint32_t n, unsigned long long *d_out,
                                 void *stream);
const char *cfpq_noalloc_last_error(void);
/* Diagnostics: the matrix's 64x64-bit tile statistics as the engine keeps
 * them.  occ_out: T*ceil(T/32) words (bit tj of row ti = tile occupied);
 * nnz_out: T*T counts (set bits per tile), T = ceil(n/64).  Either may be NULL.
 * No reference counterpart (tile statistics are this engine's own). */
int cfpq_matrix_tile_stats(cfpq_ctx *ctx, const cfpq_matrix *m, uint32_t *occ_out, uint32_t *nnz_out);
/* hash/count of several matrices with one synchronisation. */
int cfpq_hash_count_many(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, uint64_t *hashes,
                         uint64_t *counts);

/* ---- products and closure ----------------------------------------------- */

/* c |= a * b over the Boolean semiring; *changed = 1 if any bit of c changed.
 * a and/or b may be c: the product then uses their values from before the
 * call.  Replaces Matrix::add_mul (cfpq-cpp/Matrix.h:17) as implemented by
 * gpu_lib::matrix_product_add_wrapper (cuda/naive-gpu/Multiplication.cu:145-166)
 * and gpu_m4ri::wrapper_method_of_4rus_bool_semiring
 * (cuda/methodOf4RusBooleanSemiringGpu/methodOf4RusBooleanSemiringGpu.cu:133-178).
 * Synchronous: returns after the product is done and the flag is read. */
int cfpq_add_mul(cfpq_ctx *ctx, cfpq_matrix *c, const cfpq_matrix *a, const cfpq_matrix *b,
                 int variant, int *changed);

/* ---- row blocks: the multi-GPU row-block closure ---------------------------
 * A single large query can be closed by several processes (one per GPU), each
 * owning a contiguous block of rows of every matrix and holding full copies of
 * all matrices: per iteration every rank runs the products of its rows, and
 * the changed row blocks are exchanged (all-gather) between iterations.  The
 * exchange itself is the caller's (the package's rowblock.py uses
 * torch.distributed).  Row ranges [row_begin, row_end) start and end on
 * multiples of 64 (the end may be n).  None of these has a reference
 * counterpart: the reference runs one query on one GPU per process
 * (cuda/naive-gpu/main.cpp:9-10). */

/* c[rows] |= a[rows] * b over the Boolean semiring for the rows in
 * [row_begin, row_end) only (the other rows of c are untouched); *changed = 1
 * if a bit of c changed.  Variant LOP3, M4R or AUTO (= LOP3); matrices without
 * a vertex order.  Aliasing as in cfpq_add_mul.  Synchronous. */
int cfpq_add_mul_rows(cfpq_ctx *ctx, cfpq_matrix *c, const cfpq_matrix *a, const cfpq_matrix *b, int variant,
                      uint32_t row_begin, uint32_t row_end, int *changed);
/* Bytes of the packed form of a row block: the 64x64-bit tiles of its
 * tile-rows, then their occupancy words, then their tile populations (0 for
 * an invalid range). */
size_t cfpq_matrix_block_bytes(const cfpq_matrix *m, uint32_t row_begin, uint32_t row_end);
/* Copies a row block into (export) or out of (import: overwrites those rows)
 * a packed buffer of cfpq_matrix_block_bytes bytes, device or host memory.
 * Asynchronous on the context's stream. */
int cfpq_matrix_export_block(cfpq_ctx *ctx, const cfpq_matrix *m, uint32_t row_begin, uint32_t row_end, void *dst);
int cfpq_matrix_import_block(cfpq_ctx *ctx, cfpq_matrix *m, uint32_t row_begin, uint32_t row_end, const void *src);
/* delta = cur AND NOT prev, then prev = cur (three different matrices of the
 * same n): the bits an iteration added, for semi-naive products.
 * Asynchronous. */
int cfpq_matrix_delta(cfpq_ctx *ctx, cfpq_matrix *delta, const cfpq_matrix *cur, cfpq_matrix *prev);

/* Runs the whole fixpoint "mats[head] |= mats[body1] * mats[body2] for every
 * rule until nothing changes" on the device.  Replaces the worklist loop of
 * Grammar::intersection_with_graph (cfpq-cpp/Grammar.h:58-69).  All matrices
 * must have the same n.  opts and stats may be NULL. */
int cfpq_closure(cfpq_ctx *ctx, const cfpq_rule *rules, size_t nrules, cfpq_matrix *const *mats,
                 size_t nmats, const cfpq_closure_opts *opts, cfpq_closure_stats *stats);

/* cfpq_closure followed by the result line (hash, count) of every matrix,
 * as cfpq_hash_count_many gives them, with one host synchronisation for both
 * (the hashes are computed on the device right after the closure).  Replaces
 * the worklist loop plus the print_results pass of the reference
 * (cfpq-cpp/Grammar.h:58-69, cfpq-cpp/Grammar.cpp:81-100) for callers that
 * want the answer lines of a query. */
int cfpq_closure_hash(cfpq_ctx *ctx, const cfpq_rule *rules, size_t nrules, cfpq_matrix *const *mats,
                      size_t nmats, const cfpq_closure_opts *opts, cfpq_closure_stats *stats, uint64_t *hashes,
                      uint64_t *counts);

/* A labelled graph for cfpq_intersection: edge e goes from[e] -> to[e] with
 * terminal label[e], and label l sets its bit in the matrices
 * label_mats[label_offsets[l] .. label_offsets[l+1]) (the terminal's
 * nonterminals, cfpq-cpp/Grammar.h:41-45).  from/label/to are device
 * pointers when on_device is nonzero; label_offsets and label_mats are host
 * arrays. */
typedef struct cfpq_edges {
    const uint32_t *from;
    const uint32_t *label;
    const uint32_t *to;
    size_t count;
    const uint32_t *label_offsets;  /* nlabels + 1 entries */
    const uint32_t *label_mats;
    uint32_t nlabels;
    int32_t on_device;
} cfpq_edges;

/* One whole query, the work of Grammar::intersection_with_graph
 * (cfpq-cpp/Grammar.h:24-69): clears mats, scatters the edges, sets the
 * diagonal of the `nepsilon` matrices listed in `epsilon` (indices into
 * mats; Grammar.h:47-51), runs the closure and, when hashes and counts are
 * non-NULL, computes every matrix's result line -- all enqueued back to back
 * with ONE synchronisation at the end (the separate calls cost one host
 * round trip each).  Host edge arrays in pinned memory that the device can
 * map (cudaMallocHost / cudaHostAlloc, or registered) are read in place by
 * the scatter kernel, with no copy; other host arrays are copied first.  An
 * edge whose vertex id is >= a matrix's n makes the call return
 * CFPQ_ERR_INVALID after the closure; the matrices then hold the closure of
 * the in-range edges. */
int cfpq_intersection(cfpq_ctx *ctx, const cfpq_rule *rules, size_t nrules, cfpq_matrix *const *mats,
                      size_t nmats, const cfpq_edges *edges, const uint32_t *epsilon, size_t nepsilon,
                      const cfpq_closure_opts *opts, cfpq_closure_stats *stats, uint64_t *hashes,
                      uint64_t *counts);

/* One independent query of a batch: its rules index into its own matrices. */
typedef struct cfpq_query {
    const cfpq_rule *rules;
    size_t nrules;
    cfpq_matrix *const *mats;
    size_t nmats;
} cfpq_query;

/* Closes many independent queries (matrices of different n allowed) together:
 * every iteration runs the products of all unfinished queries in one grouped
 * launch.  iterations_out[q] (optional) receives the iteration after which
 * query q stopped changing, done_ms_out[q] (optional) the device time from the
 * start of the batch until the end of that iteration.  No reference
 * counterpart (the reference runs one query per process, runners.py:22-30). */
int cfpq_closure_batch(cfpq_ctx *ctx, const cfpq_query *queries, size_t nqueries,
                       const cfpq_closure_opts *opts, cfpq_closure_stats *stats,
                       uint32_t *iterations_out, double *done_ms_out);

/* Per-product log of the last cfpq_closure / cfpq_closure_batch call run with
 * opts->log_products & CFPQ_LOG_PRODUCTS (engine driver): one record per
 * (iteration, product term).  In that mode the iterations run from the host;
 * after the selection, every term runs alone with every candidate variant,
 * term after term, so each timing sees the operands the selection saw plus
 * what the terms timed before it added (as in a sequential pass; the
 * candidates are real products, bits only ever get added), then the
 * iteration runs with the selected variants: usec[v] is the device time of
 * variant v (CUDA events around its plan and product launches), or < 0 where
 * v was not timed.  These
 * records are the cost model's training data and the ground truth of its
 * regret.  Returns the number of records available; copies at most cap.
 * No reference counterpart (the reference only times the whole closure,
 * cfpq-cpp/Grammar.h:53-80). */
#define CFPQ_SEL_FEATURES 16
#define CFPQ_SEL_OUTPUTS 3 /* LOP3, M4R, TC */
typedef struct cfpq_product_record {
    uint32_t iteration;
    uint32_t query;
    uint32_t rule;
    uint32_t term;          /* 0: delta(body1) * body2, 1: body1 * delta(body2) */
    uint32_t n;
    uint32_t variant;       /* variant that did the real work (the selector's choice) */
    uint32_t flags;         /* bit 8: the MLP chose; bit 9: the MLP ran but was not confident */
    uint32_t reserved;
    float features[CFPQ_SEL_FEATURES];  /* the selector's feature vector (kernel_select.cu) */
    float predicted[CFPQ_SEL_OUTPUTS];  /* MLP prediction, log microseconds (0 if it did not run) */
    float usec[5];                      /* index = cfpq_variant */
} cfpq_product_record;
size_t cfpq_product_log(cfpq_ctx *ctx, cfpq_product_record *out, size_t cap);

/* ---- Variant selector -------------------------------------------------------
 * With opts->variant = CFPQ_VARIANT_AUTO the engine chooses, on the device and
 * for every product term in every iteration, which exact variant runs it
 * (LOP3, M4R or TC).  The choice never changes a result.  No reference
 * counterpart: the reference binds one Matrix implementation per executable
 * (cfpq-cpp/Grammar.h:23). */
#define CFPQ_SELECT_FIXED 0     /* AUTO behaves like LOP3 */
#define CFPQ_SELECT_HEURISTIC 1 /* autotuned density thresholds */
#define CFPQ_SELECT_MLP 2       /* cost model, heuristic when it is not confident */
typedef struct cfpq_selector_config {
    int32_t mode;
    uint32_t allowed;       /* bit v set: variant v may be chosen (bits 2, 3, 4) */
    uint32_t tc_min_tiles;  /* tensor cores only for n >= 64 * tc_min_tiles */
    float tc_min_occ;       /* TC: minimum occupied-tile fraction of P */
    float tc_min_dense;     /* TC: minimum fraction of dense P tiles (population > 96): the
                               word-level kernels pay a dense tile's full cost whatever its
                               population, the tensor cores pay it for every tile */
    float m4r_min_dense;    /* M4R: minimum fraction of dense P tiles (population > 96) */
    float conf_margin;      /* MLP: best prediction ahead of the second by this (log us) */
    float range_margin;     /* MLP: features within the training range widened by this fraction */
    uint32_t min_tiles;     /* a single-query closure selects only if it has a term of
                               n >= 64 * min_tiles (smaller ones are latency-bound and run
                               LOP3 throughout); batches of queries always select */
} cfpq_selector_config;
int cfpq_selector_configure(cfpq_ctx *ctx, const cfpq_selector_config *cfg);
int cfpq_selector_get_config(cfpq_ctx *ctx, cfpq_selector_config *cfg);

/* Cost model weights: W1[16][64], b1[64], W2[64][64], b2[64], W3[64][3], b3[3]
 * (row-major, input index first), then the training range of the features
 * (lo[16], hi[16]).  cfpq_selector_weight_count() floats in total. */
size_t cfpq_selector_weight_count(void);
int cfpq_selector_set_weights(cfpq_ctx *ctx, const float *w, size_t count);
int cfpq_selector_get_weights(cfpq_ctx *ctx, float *w, size_t count); /* CFPQ_ERR_INVALID if untrained */

/* Train the cost model on the GPU (hand-written forward/backward kernels,
 * full-batch Adam) from product records: targets log(usec[v]) of the timed
 * variants, loss = mean squared error over timed entries.  Sets the weights
 * and the feature ranges; does not change the mode. */
typedef struct cfpq_train_opts {
    int32_t epochs;         /* default 2000 */
    float learning_rate;    /* default 3e-3 */
    float weight_decay;     /* default 1e-4 */
    uint32_t seed;          /* weight initialisation */
    int32_t keep_weights;   /* 1: continue from the current weights */
} cfpq_train_opts;
typedef struct cfpq_train_report {
    float loss_first, loss_last;
    uint32_t samples, epochs;
    double ms;
} cfpq_train_report;
int cfpq_selector_train(cfpq_ctx *ctx, const cfpq_product_record *recs, size_t count, const cfpq_train_opts *opts,
                        cfpq_train_report *report);

/* The training kernels' loss and gradient for explicit weights (count =
 * cfpq_selector_weight_count() - 32 floats, no feature ranges) on samples
 * x[n][16], targets y[n][3], mask m[n][3] (host arrays): the gradient check. */
int cfpq_selector_loss_grad(cfpq_ctx *ctx, const float *weights, const float *x, const float *y, const float *m,
                            size_t n, float *loss, float *grad);
/* Predictions of the current weights for x[n][16] (host), out[n][3]. */
int cfpq_selector_predict(cfpq_ctx *ctx, const float *x, size_t n, float *out);

/* Autotuner: times C |= A * B with LOP3, M4R and TC on seeded random
 * matrices (every tile populated) for the given sizes and densities, finds the
 * crossovers and stores them in the context's selector thresholds (and in
 * *result).  timings (optional, [nsizes][ndensities][3] ms, < 0 = not run). */
typedef struct cfpq_autotune_opts {
    const uint32_t *sizes;
    size_t nsizes;
    const float *densities;
    size_t ndensities;
    uint32_t reps;
    uint32_t seed;
} cfpq_autotune_opts;
int cfpq_autotune(cfpq_ctx *ctx, const cfpq_autotune_opts *opts, cfpq_selector_config *result, float *timings);

/* Phase timestamps of the last closure that ran as one persistent kernel
 * (use_graph = CFPQ_LOOP_DEVICE, every product word-level): per iteration
 * three %globaltimer values in ns taken by CTA 0 -- iteration start, CTA 0
 * done with its share of the plan (other CTAs' items may already run), and
 * the iteration's grid barrier passed (all products done).  Copies
 * min(cap, 3 * iterations) values and returns the number of iterations logged
 * (at most 4096; 0 when the last closure did not run persistently). */
size_t cfpq_last_phase_log(cfpq_ctx *ctx, uint64_t *out, size_t cap);

/* Work-item trace of the last persistent closure run with
 * opts->log_products & CFPQ_LOG_ITEMS: one record per processed work item
 * (the first 65536), in no particular order.  `item` is the item's encoding
 * (bits 48-63 product index in the closure, 37-47 tile-row, 28-36 block of 16
 * output tiles, 16-27 first k-tile, 4-15 end k-tile), `list` 0 for the LOP3
 * inner loop and 1 for Four Russians; times are %globaltimer ns taken by the
 * CTA around the item.  Records with list 2 (item 0) are the CTA's plan and
 * delta-clear span of the iteration, from its start to the moment the CTA
 * published its items (results of the iteration's items merge only after
 * every CTA has).  Copies min(cap, count) records and returns the count
 * (0 when the last closure was not traced). */
#define CFPQ_LOG_ITEMS 8
typedef struct cfpq_item_record {
    uint64_t item;
    uint32_t iteration;
    uint16_t cta, list;
    uint64_t start_ns, end_ns;
    /* item sub-phases, ns after start_ns: k-list built, first staged k-tile
     * arrived, last k-tile done, results allowed to merge (0 for list 2) */
    uint32_t klist_ns, staged_ns, computed_ns, gate_ns;
} cfpq_item_record;
size_t cfpq_item_log(cfpq_ctx *ctx, cfpq_item_record *out, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* CFPQ_B200_H */
