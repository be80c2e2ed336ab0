// Host-side launch wrappers for the kernels of libcfpq_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "input_device.cuh"

namespace cfpq {

// Layout / initialisation
cudaError_t launch_set_bits(const DevMat &m, const uint32_t *d_rows, const uint32_t *d_cols, size_t count,
                            uint32_t *d_bad, cudaStream_t s);
// dependent: launched right after k_input_first as a programmatic dependent
// launch (its loads of edges and tables overlap that kernel).
cudaError_t launch_load_edges(const DevMat *d_mats, uint32_t nmats, const uint32_t *d_from, const uint32_t *d_label,
                              const uint32_t *d_to, size_t ne, const uint32_t *d_off, const uint32_t *d_lm,
                              uint32_t nlabels, uint32_t nlm, uint32_t *d_bad, cudaStream_t s, bool dependent = false);
cudaError_t launch_set_diag(const DevMat &m, cudaStream_t s);
cudaError_t launch_occ_rebuild(const DevMat &m, cudaStream_t s);
// delta = cur & ~prev, then prev = cur; tile statistics of both rebuilt.
cudaError_t launch_delta_snapshot(const DevMat &delta, const DevMat &cur, const DevMat &prev, cudaStream_t s);

// Nonterminal-set closure (kernel_ntset.cu): one n x n matrix of cells holding
// sets of nonterminals (1-byte cells for <= 8 nonterminals, 4-byte for <= 32),
// row stride `stride` cells (n rounded up to 64).  d_rules: nrules records of
// 4 bytes (head, body1, body2, 0); counters: [0] row counter, [1] changed
// flag, zero before each squaring pass.
size_t ntset_cell_bytes(uint32_t nmats);
size_t ntset_max_n(uint32_t nmats);
cudaError_t launch_ntset_pack(void *cells, uint32_t stride, uint32_t nmats, const DevMat *d_mats, int num_sms,
                              cudaStream_t s);
cudaError_t launch_ntset_unpack(const void *cells, uint32_t stride, uint32_t nmats, const DevMat *d_mats, int num_sms,
                                cudaStream_t s);
cudaError_t launch_ntset_square(void *cells, uint32_t n, uint32_t stride, uint32_t nmats, const void *d_rules,
                                uint32_t nrules, uint32_t ymask, uint32_t *counters, int num_sms, cudaStream_t s);
cudaError_t launch_rows_to_tiles(const DevMat &m, const uint64_t *d_rows, cudaStream_t s);
cudaError_t launch_tiles_to_rows(const DevMat &m, uint64_t *d_rows, cudaStream_t s);
cudaError_t launch_copy_matrix(const DevMat &dst, const DevMat &src, cudaStream_t s);
cudaError_t launch_clear_matrix(const DevMat &m, cudaStream_t s);
// Seeded random matrix with the given bit density (not for ordered matrices).
cudaError_t launch_random_fill(const DevMat &m, double density, uint64_t seed, cudaStream_t s);
// Clear the matrices of d_tab (occupied tiles only; relies on the occupancy invariant).
cudaError_t launch_clear_rows(const MatRows *d_tab, uint32_t nmats, uint32_t total_rows, cudaStream_t s);

// Result hash / count (cfpq-cpp/Grammar.cpp:81-100 on the device) of up to
// kHashBatch matrices in one launch: one block per tile-row (matrix i owns
// blocks [start[i], start[i+1])), partial sums in d_partial (2 words per
// block), and the last block writes out[2i] = hash, out[2i+1] = bit count.
// d_ticket must be 0 before the first launch (every launch leaves it 0);
// out may be mapped host memory.  start[count] must be > 0.
constexpr uint32_t kHashBatch = 16;
struct HashBatch {
    DevMat m[kHashBatch];
    const uint32_t *nib11[kHashBatch];  // nibble tables of the column powers (launch_pow_nibbles)
    const uint32_t *pow13[kHashBatch];
    uint32_t start[kHashBatch + 1];  // prefix sums of the matrices' tile-rows (one block each)
    uint32_t count;
};
cudaError_t launch_hash_lines(const HashBatch &hb, unsigned long long *d_partial, uint32_t *d_ticket,
                              unsigned long long *out, cudaStream_t s);
// sub[tj * 256 + p * 16 + v] = sum over the set bits b of v of pow11[64 tj + 4 p + b]
// (mod 1e9+7) for the T tile columns: a row's column term is the sum of 16
// entries, one per nibble of its tile word.
cudaError_t launch_pow_nibbles(const uint32_t *d_pow11, uint32_t T, uint32_t *d_sub, cudaStream_t s);

// Plain dense product (variant PLAIN): mode 0 ORs into c and sets *d_flag on
// change; mode 1 writes the product into c (c must not alias a or b).
cudaError_t launch_plain_product(const DevMat &a, const DevMat &b, const DevMat &c, int mode, uint32_t *d_flag,
                                 cudaStream_t s);
// dst |= src, *d_flag set on change.
cudaError_t launch_merge_or(const DevMat &dst, const DevMat &src, uint32_t *d_flag, cudaStream_t s);

// Closure iteration
// A tensor-core-capable product of a closure and where its groups of 4
// tile-rows start in the grouped tensor-core plan (k_plan_tc).
struct TcRows {
    uint32_t prod, row_start, pref, pad;
};
cudaError_t launch_plan_tc(const ProdDesc *d_prods, uint32_t nprods, const TcRows *d_tc, uint32_t ntc,
                           uint32_t total_groups, const MatSlot *d_slots, IterState *d_st, uint64_t *d_items,
                           size_t list_cap, int tiles_per_block, uint32_t *d_prod_seen, const uint8_t *d_choice,
                           cudaStream_t s, const uint32_t *d_q_last = nullptr);
cudaError_t launch_plan(const ProdDesc *d_prods, uint32_t nprods, uint32_t row_begin, uint32_t row_end,
                        const MatSlot *d_slots, IterState *d_st, uint64_t *d_items, size_t list_cap,
                        int tiles_per_block, uint32_t *d_prod_seen, int tc_mode, const uint8_t *d_choice,
                        cudaStream_t s, const PlanSelect *sel = nullptr, const uint32_t *d_q_last = nullptr);
// (tc_mode 0 plans the word-level products of the row range, 1 the tensor-core
// ones; the variant of product p is d_choice[p], or its descriptor's when
// null; with sel, the word-level plan decides the variants, PlanSelect.)
// Tiled product over item list `m4r` (0: LOP3 inner loop, 1: Four Russians
// inner loop); items of list l start at d_items + l * list_cap.
cudaError_t launch_product_tiled(int m4r, const ProdDesc *d_prods, const MatSlot *d_slots, IterState *d_st,
                                 const uint64_t *d_items, size_t list_cap, uint32_t *d_qchanged, int grid,
                                 BufCounters *d_cnts, cudaStream_t s);
// Tensor-core product over item list 2 (d_items + 2 * list_cap): packed
// operand tiles staged by bulk copies and expanded to 0/1 bytes in shared
// memory; one CTA per SM (it owns all 512 TMEM columns).
cudaError_t launch_product_tc(const ProdDesc *d_prods, const MatSlot *d_slots, IterState *d_st,
                              const uint64_t *d_items, size_t list_cap, uint32_t *d_qchanged, int grid,
                              BufCounters *d_cnts, cudaStream_t s);
int product_tc_blocks_per_sm();
// Closes a tensor-core product's item list (counts it, resets the counters).
cudaError_t launch_reset_list(IterState *st, int list, cudaStream_t s);
int product_lop3_tiles_per_block();
int product_lop3_max_tiles();
// Called once per context before any capture: sets kernel attributes, returns
// resident CTAs per SM of the given inner loop.
int product_tiled_blocks_per_sm(int m4r);
// Clears the deltas read in this iteration, then (last block) ends the
// iteration: changed flag, iteration index, loop condition, per-query records.
cudaError_t launch_advance_end(const MatSlot *d_slots, uint32_t nslots, uint32_t total_rows, IterState *d_st,
                               const QueryTrack &qt, cudaGraphConditionalHandle handle, int use_handle,
                               BufCounters *d_cnts, cudaStream_t s);

// Closure prologue (one launch): zero[r][0 .. nwords[r]) = 0, choice[0 ..
// nchoice) = choice_value, *st = a fresh iteration state (active, max_iter,
// nqueries, start stamp).
struct ClosureBegin {
    static constexpr int kRanges = 3;
    uint32_t *zero[kRanges];
    size_t nwords[kRanges];
    uint8_t *choice;
    size_t nchoice;
    uint8_t choice_value;
    IterState *st;
    uint32_t max_iter, nqueries;
};
cudaError_t launch_closure_begin(const ClosureBegin &a, int num_sms, cudaStream_t s);
// A query's input phase as stand-alone kernels: clear (with in.bad set to 0
// and, when begin is given, the closure prologue in the same launch), edge
// scatter, diagonals.
cudaError_t launch_closure_input(const ClosureInput &in, int num_sms, cudaStream_t s,
                                 const ClosureBegin *begin = nullptr);
// Persistent closure (word-level variants only): the whole fixpoint in one
// cooperative launch of `grid` CTAs (at most persistent_blocks_per_sm() per
// SM); items: 4 lists of list_cap; phase_log: 3 timestamps per iteration.
int persistent_blocks_per_sm(int has_m4r);
cudaError_t launch_closure_persistent(int has_m4r, int grid, const ProdDesc *prods, uint32_t nprods,
                                      uint32_t prod_rows, const MatSlot *slots, uint32_t nslots, uint32_t slot_rows,
                                      IterState *st, uint64_t *items, size_t list_cap, uint32_t *prod_seen,
                                      const QueryTrack &qt, int tpb, unsigned long long *phase_log,
                                      uint32_t phase_log_iters, BufCounters *cnts, uint8_t *choice,
                                      const SelectorParams *sel, SelLogRow *sel_log, uint32_t sel_log_iters,
                                      const QueryRange *qr, ItemTrace *trace, uint32_t *trace_count,
                                      int direct_merge, int prefetch, uint32_t spin_limit, int stall_barrier,
                                      IterState *host_st, const uint32_t *flag_src, uint32_t *flag_dst,
                                      cudaStream_t s);
// (spin_limit 0: the default of about a second of polling per wait;
// trace non-null: one ItemTrace per processed item, counted in *trace_count)
// (direct_merge: result words go to their atomic OR without reading C first)
// (prefetch: a CTA takes its next item index while it processes one)
// (qr non-null: per-query ranges of a batch of 2..kMaxActiveQueries queries,
// whose iterations then plan and clear only the queries still changing; the
// query-changed flags are then 3 * nqueries words, rotated per iteration)
// (sel non-null: every iteration starts with a selection phase writing choice[];
// else choice[] is fixed for the closure)

// Variant selection (kernel_select.cu): one warp per product per iteration.
cudaError_t launch_select(const ProdDesc *d_prods, uint32_t nprods, const BufCounters *d_cnts, const IterState *d_st,
                          const SelectorParams *d_params, uint8_t *d_choice, const uint8_t *d_tc_ok,
                          SelLogRow *d_log, uint32_t log_iters, cudaStream_t s);
// Buffer counters at closure start (current matrices measured, deltas zero).
cudaError_t launch_counters_init(const MatSlot *d_slots, uint32_t nslots, BufCounters *d_cnts, cudaStream_t s);
cudaError_t launch_fill_choice(uint8_t *d_choice, uint32_t n, uint8_t v, cudaStream_t s);

// Cost-model training and inference (kernel_mlp.cu); weights: kSelWeights floats.
cudaError_t mlp_loss_grad(const float *d_w, const float *d_x, const float *d_y, const float *d_m, uint32_t n,
                          float inv_msum, float *d_grad, float *d_loss, cudaStream_t s);
cudaError_t mlp_adam_step(float *d_w, float *d_grad, float *d_m, float *d_v, float lr, float wd, uint32_t step,
                          cudaStream_t s);
cudaError_t mlp_predict(const float *d_w, const float *d_x, uint32_t n, float *d_out, cudaStream_t s);
// Calibration: logic instructions per second of the whole GPU (d_out: 8*256*num_sms words).
cudaError_t measure_logic_rate(int num_sms, uint32_t *d_out, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1,
                               double *ops_per_s, double *ms_out);

}  // namespace cfpq
