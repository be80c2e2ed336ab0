// Internal host-side state of libcfpq_b200.so: the context, matrix and
// order handles behind the opaque C types, device buffers, error reporting.
// Shared by the C-ABI sources (capi.cu, capi_select.cu).
#pragma once

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "cfpq_b200.h"
#include "launch.h"

using namespace cfpq;

// ---------------------------------------------------------------------------
// errors

// Records the message for cfpq_last_error() and returns code.
int set_error(int code, const char *fmt, ...);

#define CUDA_TRY(call)                                                                                \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return set_error(e_ == cudaErrorMemoryAllocation ? CFPQ_ERR_OOM : CFPQ_ERR_CUDA,          \
                             "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);    \
    } while (0)

#define TRY(call)                   \
    do {                            \
        int r_ = (call);            \
        if (r_ != CFPQ_OK) return r_; \
    } while (0)

// ---------------------------------------------------------------------------
// types

namespace cfpq_host {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes) {
        if (bytes <= cap) return CFPQ_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        want = (want + 4095) & ~(size_t)4095;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            p = nullptr;
            return set_error(CFPQ_ERR_OOM, "device allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
        }
        cap = want;
        return CFPQ_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

struct PowTables {
    uint32_t *d_pow11 = nullptr;
    uint32_t *d_pow13 = nullptr;
    uint32_t *d_nib11 = nullptr;  // per tile column and nibble: the 16 subset sums of pow11 (launch_pow_nibbles)
};

struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    std::vector<uint64_t> key;
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        key.clear();
    }
};

}  // namespace cfpq_host

using namespace cfpq_host;

struct cfpq_order {
    uint32_t n = 0;
    uint32_t *d_perm = nullptr;
    PowTables pow;  // hash powers indexed by internal id
};

struct cfpq_matrix {
    cfpq_ctx *ctx;
    DevMat d;
    cfpq_order *order = nullptr;
};

struct PlanCache;

struct cfpq_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // small device scratch
    IterState *d_st = nullptr;
    uint32_t *d_flag = nullptr;
    unsigned long long *d_hash = nullptr;  // 2 per matrix for hash_count_many (when h_hash is not mapped)
    size_t d_hash_cap = 0;
    unsigned long long *d_hash_part = nullptr;  // 2 per hash block (tile-row)
    size_t d_hash_part_cap = 0;                 // in blocks
    uint32_t *d_hash_ticket = nullptr;          // blocks done of the running hash launch (0 between launches)
    uint32_t *d_bad = nullptr;
    // pinned host scratch
    IterState *h_st = nullptr;
    IterState *h_st_dev = nullptr;  // h_st as the device sees it (pinned, mapped)
    uint32_t *h_flag_dev = nullptr; // h_flag as the device sees it
    uint32_t *h_flag = nullptr;
    unsigned long long *h_hash = nullptr;
    unsigned long long *h_hash_dev = nullptr;  // h_hash as the device sees it (null: not mapped)
    size_t h_hash_cap = 0;
    // growable device scratch
    DevBuf stage, items, prods, slots, qtrack, prod_seen, mats_desc, edge_buf, clear_desc, diag_desc;
    std::unordered_map<uint32_t, PowTables> pow;
    std::vector<cfpq_matrix *> pool;  // zeroed spare matrices (deltas, alias copies)
    GraphCache gcache;
    PlanCache *pcache = nullptr;  // created by the first closure
    uint64_t plan_ids = 0;
    uint64_t tables_owner = 0;  // plan id whose slot / product tables are in `slots` / `prods`
    int lop3_grid = 0, m4r_grid = 0, tc_grid = 0;  // tc_grid 0: tensor-core variant unavailable
    int persist_grid[2] = {0, 0};  // persistent closure CTAs [with M4R items]; 0: unavailable
    DevBuf phase_log;              // persistent closure: 3 timestamps per iteration
    DevBuf qranges;                // persistent closure of a batch: QueryRange per query
    DevBuf item_trace;             // CFPQ_LOG_ITEMS: ItemTrace records, then the record count
    uint32_t item_trace_n = 0;     // records of the last closure
    uint32_t phase_log_iters = 0;  // iterations logged by the last closure
    std::vector<cfpq_product_record> log;
    cudaEvent_t kev[5] = {};
    cfpq_kernel_profile prof = {};
    void *h_small = nullptr;
    size_t h_small_cap = 0;
    std::vector<unsigned char> edge_tables_key;  // small tables of the last edge load still in edge_buf
    std::vector<unsigned char> clear_desc_key;   // matrix list of the last cfpq_matrices_clear in clear_desc
    std::vector<unsigned char> diag_desc_key;    // epsilon matrices of the last cfpq_intersection in diag_desc
    void *items_clean_ptr = nullptr;  // items buffer whose first items_clean_words words are zero
    size_t items_clean_words = 0;
    void *h_query = nullptr;  // pinned: per-query results of a closure (done_ns, last_iter)
    size_t h_query_cap = 0;
    // variant selector
    SelectorParams sel;            // host copy of the device parameters
    bool sel_dirty = true;         // host copy changed since the last upload
    DevBuf d_sel, cnts, choice, tc_ok, sel_log, tc_rows;
    uint32_t sel_log_iters = 0, sel_log_prods = 0;
    bool cnts_on = false;          // the current closure keeps buffer counters
    std::vector<cudaEvent_t> tev;  // product timing events (CFPQ_LOG_PRODUCTS)
    DevBuf mlp_w, mlp_x, mlp_y, mlp_m, mlp_grad, mlp_m1, mlp_v2, mlp_loss, mlp_out;
    // nonterminal-set variant: cell matrix, matrix descriptors, rules, counters
    DevBuf nt_cells, nt_mats, nt_rules, nt_ctr;
};

// Selector defaults (before cfpq_autotune or cfpq_selector_configure).
void selector_defaults(SelectorParams *sp);
// Upload the selector parameters if they changed.
int selector_sync(cfpq_ctx *ctx);

