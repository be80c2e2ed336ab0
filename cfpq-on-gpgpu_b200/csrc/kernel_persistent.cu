// Persistent closure kernel: the whole semi-naive fixpoint of a closure whose
// products all use the word-level variants (LOP3 / M4R) in ONE cooperative
// launch (every CTA resident), one grid barrier per iteration instead of
// kernel boundaries.
//
// Iteration t (parity par = t & 1), every CTA:
//   plan     warps take units round-robin: the product tile-rows (plan::plan_row
//            appends the iteration's work items to the item list of parity
//            par, Four Russians items marked by bit 0; AUTO closures: the
//            planner also chooses each term's variant, select_device.cuh) and,
//            for t >= 1, the slot tile-rows of the delta read in iteration t-1
//            (dlt[par ^ 1], cleared: the products of iteration t write their
//            new bits there).  CTA 0 also folds the counters of parity par ^ 1
//            (iteration t-1) into the statistics and zeroes them.  Batches of
//            at most kMaxActive queries plan only the queries that changed in
//            iteration t-1 and clear only those that changed in t-2 (the
//            deltas of the others are empty): every CTA compacts the
//            per-query changed flags into its own active lists first, so
//            converged queries cost nothing in the tail of a batch.  The CTA
//            then counts itself in the plan word pplan[par] (high half;
//            the low half counts the items written).
//   products the CTA takes items from the list as soon as they are written
//            (no barrier after the plan) and runs tiled::process_item; an
//            item merges its results only once every CTA is done planning
//            and clearing (plan-done half == grid).  New bits set
//            changed[par] and the query's flag in qt.changed[t % 3] (three
//            rotating flag arrays: iteration t reads those of t-1 and t-2;
//            CTA 0 zeroes those of t+1 after the barrier of t).
//   barrier
//   decision every CTA reads changed[par] (final after the barrier) and the
//            error word: continue while something changed, no wait gave up
//            and the iteration limit is not reached.  CTA 0 records the
//            per-query convergence data.
// After the loop the delta read in the last iteration is cleared, so the
// delta buffers go back to the pool zeroed.
//
// Overlapping the plan with the products is exact: an item's operands only
// grow after its planner read them (its k-tile range is a fixed part of
// [0, T) and the item re-reads the occupancy), so it covers at least the
// semi-naive terms of its planner, and bits it finds beyond those are true
// and recorded in the delta like any other.
//
// The same plan and item code as the multi-kernel iteration runs here; only
// the sequencing differs.  Every wait is bounded: a CTA that gives up sets
// the error word and leaves the loop, and every other wait then gives up too.
#include "launch.h"
#include "plan_device.cuh"
#include "product_tiled.cuh"

namespace cfpq {

namespace {

using tiled::ItemCounters;

// 8 warps per CTA: an item's 16 output tiles are spread 2 per warp (twice the
// threads of the product kernels on one item: most iterations of a single
// closure have fewer items than CTAs, so item latency is the phase length).
constexpr int kPW = 8;
constexpr uint32_t kThreads = 32 * kPW;

constexpr uint32_t kBarrierSpinLimit = 1u << 25;  // default limit of the waits below: ~1 s of polling
constexpr uint32_t kNoIndex = 0xFFFFFFFFu;

// Word-level products only: output blocks of 16 tiles, at most 128 per
// tile-row.  The planner areas do not alias the product layout (its mbarriers
// live across phases).
constexpr uint32_t kWordBlocks = 128;

// Slot and product tables are copied into shared memory when they fit (one
// query or a small batch), saving two dependent global loads per item.
constexpr uint32_t kTableBytes = 8192;

constexpr uint32_t kMaxActive = kMaxActiveQueries;
constexpr uint32_t kActivePerThread = kMaxActive / kThreads;
static_assert(kMaxActive % kThreads == 0, "active-list build: whole queries per thread");

// Queries of one phase-A unit set with the prefix sum of their row counts:
// unit u belongs to q[i] for the last i with pref[i] <= u.
struct ActiveList {
    uint32_t n;
    uint32_t pref[kMaxActive + 1];
    uint16_t q[kMaxActive];
};

// Phase-A scratch.  It lives in the Q staging buffers of the product layout:
// no bulk copy is in flight outside phase B (every item waits for all the
// k-tiles it staged), and the mbarriers lie outside the staging buffers.
struct PlanScratch {
    plan::WarpArea<kWordBlocks> plan[kPW];
    ActiveList act_plan, act_clear;
    uint32_t wtot[kPW][2];
};

// (8 staged k-tiles instead of 4 for LOP3-only closures measured no faster
// on the same-generation N=8192 closure: 0.2714 vs 0.2715 ms.)
template <bool kM4R>
struct PersistSmem {
    tiled::TiledSmem<kM4R> prod;
    alignas(16) unsigned char tables[kTableBytes];
    __device__ PlanScratch &scratch() { return *reinterpret_cast<PlanScratch *>(&prod.q[0][0]); }
};
static_assert(sizeof(PlanScratch) <= sizeof(tiled::TiledSmem<false>::q), "phase-A scratch fits the staging buffers");

struct PersistArgs {
    const ProdDesc *prods;
    uint32_t nprods, prod_rows;
    const MatSlot *slots;
    uint32_t nslots, slot_rows;
    IterState *st;
    uint64_t *items;  // 4 lists: (parity, list) at items + (2 * parity + list) * list_cap
    size_t list_cap;
    uint32_t *prod_seen;
    QueryTrack qt;
    int tpb;
    unsigned long long *phase_log;  // 3 %globaltimer stamps per iteration (may be null)
    uint32_t phase_log_iters;
    BufCounters *cnts;              // 3 per slot
    uint8_t *choice;                // variant of every product in the current iteration
    const SelectorParams *sel;      // non-null: choose per iteration (selection phase)
    SelLogRow *sel_log;
    uint32_t sel_log_iters;
    const QueryRange *qr;           // non-null (batches of 2..kMaxActive queries): active-query phase A
    ItemTrace *trace;               // non-null: one record per processed item (first kItemTraceCap)
    int direct_merge;               // items merge without reading C first (small single closures)
    int prefetch;                   // take the next item index while processing one (batches)
    uint32_t *trace_count;
    uint32_t spin_limit;            // polls of the item wait and of the grid barrier before they give up
    uint32_t stall_barrier;         // test hook: the first grid barrier waits for one arrival more than
                                    // there are CTAs, so that its bounded wait runs out
    IterState *host_st;             // non-null: the last CTA to exit writes the final state here
    const uint32_t *flag_src;       // and (non-null) this word to *flag_dst (both mapped host memory)
    uint32_t *flag_dst;
};

// Records one processed item (thread 0 of the CTA); sub: the item's
// sub-phase stamps (process_item), null for plan spans.
__device__ __forceinline__ void trace_item(const PersistArgs &a, uint64_t it, uint32_t iter, uint32_t list,
                                           unsigned long long t0, const unsigned long long *sub = nullptr) {
    const uint32_t k = atomicAdd(a.trace_count, 1u);
    if (k >= kItemTraceCap) return;
    auto rel = [&](int i) { return sub ? (uint32_t)(sub[i] - t0) : 0u; };
    a.trace[k] = ItemTrace{it, iter, (uint16_t)blockIdx.x, (uint16_t)list, t0, globaltimer_ns(), rel(0), rel(1),
                           rel(2), rel(3)};
}

// Block-wide compaction of the queries whose flag is set (every query when
// flags is null) into L, with the prefix sum of their plan rows (slot rows
// when srows).  Called by all threads; ends synchronised.
__device__ void build_active(ActiveList &L, const uint32_t *flags, const QueryRange *qr, uint32_t nq, bool srows,
                             uint32_t (*wtot)[2]) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t q0 = tid * kActivePerThread;
    uint32_t rows[kActivePerThread], c = 0, r = 0;
#pragma unroll
    for (uint32_t k = 0; k < kActivePerThread; ++k) {
        const uint32_t q = q0 + k;
        const bool on = q < nq && (!flags || __ldcg(flags + q) != 0);
        rows[k] = on ? (srows ? qr[q].nsrow : qr[q].nprow) : 0xFFFFFFFFu;
        c += on;
        r += on ? rows[k] : 0;
    }
    uint32_t ic = c, ir = r;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t xc = __shfl_up_sync(tiled::kFull, ic, o), xr = __shfl_up_sync(tiled::kFull, ir, o);
        if (lane >= (uint32_t)o) {
            ic += xc;
            ir += xr;
        }
    }
    if (lane == 31) {
        wtot[warp][0] = ic;
        wtot[warp][1] = ir;
    }
    __syncthreads();
    uint32_t ec = ic - c, er = ir - r;
    for (uint32_t w = 0; w < warp; ++w) {
        ec += wtot[w][0];
        er += wtot[w][1];
    }
#pragma unroll
    for (uint32_t k = 0; k < kActivePerThread; ++k) {
        if (rows[k] == 0xFFFFFFFFu) continue;
        L.q[ec] = (uint16_t)(q0 + k);
        L.pref[ec] = er;
        ++ec;
        er += rows[k];
    }
    if (tid == kThreads - 1) {
        L.n = ec;
        L.pref[ec] = er;
    }
    __syncthreads();
}

// Index i of the last pref[i] <= u in L (u below the list's total).
__device__ __forceinline__ uint32_t active_find(const ActiveList &L, uint32_t u) {
    uint32_t lo = 0, hi = L.n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (L.pref[mid] <= u) lo = mid; else hi = mid;
    }
    return lo;
}

// Grid barrier of an iteration (all CTAs of the cooperative launch) on the
// 64-bit word w: every CTA adds one arrival to the low half and polls the
// word until the count reaches `target`; the high half, final by then, comes
// with the same load.  Returns false when the wait gave up; *flags receives
// the high half.
__device__ __forceinline__ bool grid_barrier(unsigned long long *w, uint32_t target, bool abort, uint32_t *flags,
                                             uint32_t spin_limit) {
    __shared__ uint32_t s_ok, s_flags;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ok = 1;
        if (abort) atomicOr(reinterpret_cast<uint32_t *>(w) + 1, kBarAbort);
        // release: the CTA's writes (ordered by the __syncthreads above) are
        // visible before the arrival; acquire: other CTAs' writes before theirs
        unsigned long long v = atom_add_acq_rel_u64(w, 1ull) + 1ull;
        uint32_t i = 0;
        while ((uint32_t)v < target) {
            if (++i > spin_limit) {
                ok = 0;
                break;
            }
            v = ld_acquire_u64(w);
        }
        s_ok = ok;
        s_flags = (uint32_t)(v >> 32);
    }
    __syncthreads();
    *flags = s_flags;
    return s_ok != 0;
}

template <bool kHasM4R>
__global__ void __launch_bounds__(kThreads, 2) k_closure_persistent(PersistArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    PersistSmem<kHasM4R> &S = *reinterpret_cast<PersistSmem<kHasM4R> *>(smem_raw);
    PlanScratch &X = S.scratch();
    IterState *st = a.st;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t gwarp = blockIdx.x * (kThreads / 32) + warp, nwarps = gridDim.x * (kThreads / 32);
    __shared__ uint32_t s_stop;
    __shared__ unsigned long long s_item;

    if (tid == 0) {
        for (uint32_t i = 0; i < decltype(S.prod)::kNumStages; ++i) mbar_init(&S.prod.bar[i], 1);
        fence_mbar_init();
    }
    const size_t slot_bytes = (size_t)a.nslots * sizeof(MatSlot), prod_bytes = (size_t)a.nprods * sizeof(ProdDesc);
    const bool cached = slot_bytes + prod_bytes <= kTableBytes;
    const MatSlot *slots = a.slots;
    const ProdDesc *prods = a.prods;
    if (cached) {
        uint32_t *dst = reinterpret_cast<uint32_t *>(S.tables);
        const uint32_t *s0 = reinterpret_cast<const uint32_t *>(a.slots);
        const uint32_t *p0 = reinterpret_cast<const uint32_t *>(a.prods);
        for (size_t i = tid; i < slot_bytes / 4; i += kThreads) dst[i] = s0[i];
        for (size_t i = tid; i < prod_bytes / 4; i += kThreads) dst[slot_bytes / 4 + i] = p0[i];
        slots = reinterpret_cast<const MatSlot *>(S.tables);
        prods = reinterpret_cast<const ProdDesc *>(S.tables + slot_bytes);
    }
    __syncthreads();
    const PlanSelect psel = {a.sel && a.cnts ? a.sel : nullptr, a.cnts, nullptr, a.choice, a.sel_log, a.sel_log_iters};
    uint32_t phase = 0, bar_uses[2] = {0, 0};
    bool timed_out = false;
    ItemCounters ctr;
    const uint32_t iter0 = st->iter, max_iter = st->max_iter;
    uint32_t t = iter0;

    for (;; ++t) {
        const uint32_t par = t & 1;
        uint64_t *const items = a.items + (size_t)(2 * par) * a.list_cap;  // one list per parity
        if (blockIdx.x == 0 && tid == 0) {
            if (a.phase_log && t - iter0 < a.phase_log_iters) a.phase_log[3 * (t - iter0)] = globaltimer_ns();
            // flags of this iteration's barrier word (last read before the
            // barrier of t-1; next set after every CTA's plan of t)
            if (t > iter0 + 1) reinterpret_cast<uint32_t *>(&st->pbar[par])[1] = 0;
            if (t > iter0) {  // counters of iteration t-1 -> statistics, then reset for iteration t+1
                const uint32_t q = par ^ 1;
                const uint32_t c0 = (uint32_t)st->pplan[q], m4r = st->pitem_m4r[q];
                st->items_total += c0;
                st->items_by_variant[2] += c0 - m4r;
                st->items_by_variant[3] += m4r;
                st->pplan[q] = 0;
                st->pitem_next[q][0] = st->pitem_next[q][1] = 0;
                st->pitem_m4r[q] = 0;
            }
        }
        // plan word halves: the planners' item count (list 0: every
        // word-level item, Four Russians ones marked) and the plan-done count
        uint32_t *const item_count = reinterpret_cast<uint32_t *>(&st->pplan[par]);
        uint32_t *const plan_done = item_count + 1;
        // ---- plan of iteration t + clear of the delta read in t-1 ----
        const unsigned long long plan_t0 = a.trace && tid == 0 ? globaltimer_ns() : 0ull;
        if (a.cnts && blockIdx.x == 0 && t > 0)  // that delta's counters restart at zero
            for (uint32_t sl = tid; sl < a.nslots; sl += kThreads) a.cnts[3 * sl + 1 + (par ^ 1)] = BufCounters{0, 0, 0};
        if (a.qr) {
            // plan: queries that changed in t-1 (all in iteration 0); clear:
            // queries that changed in t-2 (all in iteration 1, none in 0)
            const uint32_t nq = st->nqueries;
            build_active(X.act_plan, t > 0 ? a.qt.changed + ((t - 1) % 3) * nq : nullptr, a.qr, nq, false, X.wtot);
            if (t > 0)
                build_active(X.act_clear, t > 1 ? a.qt.changed + ((t - 2) % 3) * nq : nullptr, a.qr, nq, true,
                             X.wtot);
            const uint32_t np = X.act_plan.pref[X.act_plan.n], ns = t > 0 ? X.act_clear.pref[X.act_clear.n] : 0u;
            for (uint32_t u = gwarp; u < np + ns; u += nwarps) {
                if (u < np) {
                    const uint32_t i = active_find(X.act_plan, u);
                    const QueryRange qr = a.qr[X.act_plan.q[i]];
                    plan::plan_row(qr.prow0 + (u - X.act_plan.pref[i]), prods, a.nprods, slots, t, st,
                                   item_count, items, a.list_cap, a.tpb, a.prod_seen, 0, psel,
                                   X.plan[warp].cnt, X.plan[warp].bnd, qr.prod0, qr.prod0 + qr.nprod,
                                   &st->pitem_m4r[par]);
                } else {
                    const uint32_t i = active_find(X.act_clear, u - np);
                    const QueryRange qr = a.qr[X.act_clear.q[i]];
                    clear_delta_row(slots, a.nslots, qr.srow0 + (u - np - X.act_clear.pref[i]), par ^ 1, qr.slot0,
                                    qr.slot0 + qr.nslot);
                }
                __syncwarp();
            }
        } else {
            const uint32_t clear_rows = t > 0 ? a.slot_rows : 0u;
            const uint32_t units = a.prod_rows + clear_rows;
            for (uint32_t u = gwarp; u < units; u += nwarps) {
                if (u < a.prod_rows) {
                    plan::plan_row(u, prods, a.nprods, slots, t, st, item_count, items, a.list_cap, a.tpb,
                                   a.prod_seen, 0, psel, X.plan[warp].cnt, X.plan[warp].bnd, 0u, 0xFFFFFFFFu,
                                   &st->pitem_m4r[par]);
                } else {
                    clear_delta_row(slots, a.nslots, u - a.prod_rows, par ^ 1);
                }
                __syncwarp();
            }
        }
        fence_proxy_async_smem();  // the scratch writes come before the next bulk copies into the same bytes
        __syncthreads();
        if (tid == 0) {  // this CTA's items, clears and counter resets are all published
            red_add_release_u32(plan_done, 1u);
            if (blockIdx.x == 0 && a.phase_log && t - iter0 < a.phase_log_iters)
                a.phase_log[3 * (t - iter0) + 1] = globaltimer_ns();
            if (a.trace) trace_item(a, 0, t, 2, plan_t0);
        }

        // ---- products: items as the planners publish them ----
        // A CTA takes the next list index and waits (bounded) until that item
        // is written or every CTA is done planning with fewer items; it
        // zeroes the slot again for the iteration after next.  Items may run
        // while other CTAs still plan (operands only grow: an item sees at
        // least what its planner saw) but their results wait for every
        // CTA's delta clear (the gate before the epilogue).
        uint32_t *const qchanged = a.qt.changed ? a.qt.changed + (t % 3) * st->nqueries : nullptr;
        uint32_t *const changed = reinterpret_cast<uint32_t *>(&st->pbar[par]) + 1;  // kBarChanged
        const uint32_t *gate = plan_done;  // cleared by the first item that passes it
        uint32_t next_idx = kNoIndex;  // (thread 0) list index taken ahead
        while (!timed_out) {
            if (tid == 0) {
                const uint32_t idx = next_idx != kNoIndex ? next_idx : atomicAdd(&st->pitem_next[par][0], 1u);
                next_idx = kNoIndex;
                volatile uint64_t *slot = items + idx;
                unsigned long long v = 0;
                uint32_t stop = 0, spins = 0;
                for (;;) {
                    // the slot and the plan word load together (one round
                    // trip); a slot read empty is read again once the plan
                    // word (acquire) says that every planner is done and the
                    // item exists
                    v = idx < a.list_cap ? *slot : 0ull;
                    const unsigned long long pw = ld_acquire_u64(&st->pplan[par]);
                    if (v) break;
                    if ((uint32_t)(pw >> 32) == gridDim.x) {
                        if (idx >= (uint32_t)pw) {
                            stop = 1;
                            break;
                        }
                        if (idx < a.list_cap && (v = *slot) != 0) break;
                    }
                    if (++spins > a.spin_limit) {
                        stop = 2;
                        break;
                    }
                    __nanosleep(32);
                }
                if (v) {
                    *slot = 0;
                    // batches: take the next index now, its round trip
                    // overlaps this item (a single closure keeps items for
                    // the CTAs that are free first)
                    if (a.prefetch) next_idx = atomicAdd(&st->pitem_next[par][0], 1u);
                }
                s_item = v;
                s_stop = stop;
            }
            __syncthreads();
            const unsigned long long v = s_item;
            const uint32_t stop = s_stop;
            __syncthreads();
            if (stop) {
                if (stop == 2) timed_out = true;
                break;
            }
            const unsigned long long t0 = a.trace ? globaltimer_ns() : 0ull;
            unsigned long long sub[4] = {t0, t0, t0, t0};
            const uint64_t item = v & ~1ull;
            bool m4r_item = false;
            if constexpr (kHasM4R) m4r_item = (v & 1ull) != 0;
            if constexpr (kHasM4R) {
                if (m4r_item)
                    tiled::process_item<true, kPW>(S.prod, item, prods, slots, t, changed, qchanged,
                                                   phase, timed_out, ctr, a.cnts, &gate, gridDim.x,
                                                a.direct_merge != 0, a.trace ? sub : nullptr);
            }
            if (!m4r_item)
                tiled::process_item<false, kPW>(S.prod, item, prods, slots, t, changed, qchanged, phase,
                                                timed_out, ctr, a.cnts, &gate, gridDim.x,
                                                a.direct_merge != 0, a.trace ? sub : nullptr);
            if (a.trace && tid == 0) trace_item(a, item, t, (uint32_t)(v & 1ull), t0, sub);
        }
        uint32_t flags = 0;
        const uint32_t target = ++bar_uses[par] * gridDim.x + (a.stall_barrier && t == iter0 ? 1u : 0u);
        if (!grid_barrier(&st->pbar[par], target, timed_out, &flags, a.spin_limit)) timed_out = true;
        if (flags & kBarAbort) timed_out = true;
        if (timed_out) break;

        // ---- decision (the same on every CTA: the flags are final) ----
        const bool go = (flags & kBarChanged) && (max_iter == 0 || t + 1 < max_iter);
        if (blockIdx.x == 0) {
            if (tid == 0 && a.phase_log && t - iter0 < a.phase_log_iters)
                a.phase_log[3 * (t - iter0) + 2] = globaltimer_ns();
            if (qchanged) {
                const unsigned long long now = globaltimer_ns();
                // flags of iteration t+1: last read by the plan of t, next
                // written after this CTA's plan of t+1 is published
                uint32_t *next = a.qt.changed + ((t + 1) % 3) * st->nqueries;
                for (uint32_t q = tid; q < st->nqueries; q += kThreads) {
                    if (__ldcg(qchanged + q)) {
                        a.qt.last_iter[q] = t + 1;
                        a.qt.done_ns[q] = now;
                    }
                    next[q] = 0;
                }
            }
        }
        if (!go) break;
    }

    // ---- exit: clear the delta read in the last iteration; final state ----
    if (!timed_out) {
        const uint32_t par = t & 1;
        if (a.qr) {  // queries planned in iteration t
            const uint32_t nq = st->nqueries;
            build_active(X.act_clear, t > 0 ? a.qt.changed + ((t - 1) % 3) * nq : nullptr, a.qr, nq, true, X.wtot);
            const uint32_t ns = X.act_clear.pref[X.act_clear.n];
            for (uint32_t u = gwarp; u < ns; u += nwarps) {
                const uint32_t i = active_find(X.act_clear, u);
                const QueryRange qr = a.qr[X.act_clear.q[i]];
                clear_delta_row(slots, a.nslots, qr.srow0 + (u - X.act_clear.pref[i]), par, qr.slot0,
                                qr.slot0 + qr.nslot);
                __syncwarp();
            }
        } else {
            for (uint32_t u = gwarp; u < a.slot_rows; u += nwarps) {
                clear_delta_row(slots, a.nslots, u, par);
                __syncwarp();
            }
        }
    }
    unsigned long long triples = ctr.triples, outw = ctr.outw, neww = ctr.neww;
    for (int o = 16; o > 0; o >>= 1) {
        triples += __shfl_down_sync(tiled::kFull, triples, o);
        outw += __shfl_down_sync(tiled::kFull, outw, o);
        neww += __shfl_down_sync(tiled::kFull, neww, o);
    }
    if (lane == 0) {
        if (triples) atomicAdd(&st->tile_triples, triples);
        if (outw) atomicAdd(&st->out_words, outw);
        if (neww) atomicAdd(&st->new_words, neww);
    }
    if (tid == 0 && ctr.staged) atomicAdd(&st->bytes_staged, ctr.staged);
    if (tid == 0 && timed_out) atomicExch(&st->error, (uint32_t)5);
    if (blockIdx.x == 0 && tid == 0 && !timed_out) {
        const uint32_t par = t & 1;
        const uint32_t c0 = (uint32_t)st->pplan[par], m4r = st->pitem_m4r[par];
        st->items_total += c0;
        st->items_by_variant[2] += c0 - m4r;
        st->items_by_variant[3] += m4r;
        st->last_changed = (uint32_t)(st->pbar[par] >> 32) & kBarChanged;
        st->iter = t + 1;
        st->active = 0;
    }
    // the final state to the host without a copy after the kernel: the last
    // CTA past this point (every other CTA's statistics and block 0's final
    // writes are then performed) writes it into mapped host memory
    if (a.host_st) {
        __shared__ uint32_t s_last;
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            s_last = atomicAdd(&st->exit_count, 1u) == gridDim.x - 1 ? 1u : 0u;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            const uint32_t *src = reinterpret_cast<const uint32_t *>(st);
            uint32_t *dst = reinterpret_cast<uint32_t *>(a.host_st);
            for (uint32_t i = tid; i < sizeof(IterState) / 4; i += kThreads) dst[i] = __ldcg(src + i);
            if (tid == 0 && a.flag_src) *a.flag_dst = __ldcg(a.flag_src);
        }
    }
}

template <bool kHasM4R>
int persistent_blocks_per_sm_impl() {
    const int smem = (int)sizeof(PersistSmem<kHasM4R>);
    if (cudaFuncSetAttribute(k_closure_persistent<kHasM4R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_closure_persistent<kHasM4R>, kThreads, smem) !=
        cudaSuccess)
        return 0;
    return nb;
}

}  // namespace

int persistent_blocks_per_sm(int has_m4r) {
    return has_m4r ? persistent_blocks_per_sm_impl<true>() : persistent_blocks_per_sm_impl<false>();
}

cudaError_t launch_closure_persistent(int has_m4r, int grid, const ProdDesc *prods, uint32_t nprods,
                                      uint32_t prod_rows, const MatSlot *slots, uint32_t nslots, uint32_t slot_rows,
                                      IterState *st, uint64_t *items, size_t list_cap, uint32_t *prod_seen,
                                      const QueryTrack &qt, int tpb, unsigned long long *phase_log,
                                      uint32_t phase_log_iters, BufCounters *cnts, uint8_t *choice,
                                      const SelectorParams *sel, SelLogRow *sel_log, uint32_t sel_log_iters,
                                      const QueryRange *qr, ItemTrace *trace, uint32_t *trace_count,
                                      int direct_merge, int prefetch, uint32_t spin_limit, int stall_barrier,
                                      IterState *host_st, const uint32_t *flag_src, uint32_t *flag_dst,
                                      cudaStream_t s) {
    PersistArgs a;
    a.prods = prods;
    a.nprods = nprods;
    a.prod_rows = prod_rows;
    a.slots = slots;
    a.nslots = nslots;
    a.slot_rows = slot_rows;
    a.st = st;
    a.items = items;
    a.list_cap = list_cap;
    a.prod_seen = prod_seen;
    a.qt = qt;
    a.tpb = tpb;
    a.phase_log = phase_log;
    a.phase_log_iters = phase_log_iters;
    a.cnts = cnts;
    a.choice = choice;
    a.sel = sel;
    a.sel_log = sel_log;
    a.sel_log_iters = sel_log_iters;
    a.qr = qr;
    a.trace = trace;
    a.trace_count = trace_count;
    a.direct_merge = direct_merge;
    a.prefetch = prefetch;
    a.spin_limit = spin_limit ? spin_limit : kBarrierSpinLimit;
    a.stall_barrier = stall_barrier ? 1u : 0u;
    a.host_st = host_st;
    a.flag_src = flag_src;
    a.flag_dst = flag_dst;
    void *args[] = {&a};
    if (has_m4r)
        return cudaLaunchCooperativeKernel((const void *)k_closure_persistent<true>, dim3(grid), dim3(kThreads), args,
                                           sizeof(PersistSmem<true>), s);
    return cudaLaunchCooperativeKernel((const void *)k_closure_persistent<false>, dim3(grid), dim3(kThreads), args,
                                       sizeof(PersistSmem<false>), s);
}

}  // namespace cfpq
