// Closure plan: per (product, tile-row) the work items of one iteration.
// Used by the plan kernel (kernels_core.cu) and the persistent closure kernel
// (kernel_persistent.cu).
#pragma once

#include "common.cuh"
#include "select_device.cuh"

namespace cfpq {
namespace plan {

constexpr unsigned kFull = 0xffffffffu;

// One warp per (product, output tile-row ti) (a group of 4 tile-rows for
// tensor-core products).  For every block of `tpb` output tiles the warp counts
// the contributing k-tiles tk (occupied P tile (ti, tk) and a non-empty Q
// block (tk, block)) in increasing tk order and cuts them into chunks of E
// (item_entries of the row's occupied P tile count, so at most
// kMaxChunksPerBlock chunks; tensor-core items take one chunk).  Chunk j of a
// block becomes the item with k-tile range [first tk of chunk j, first tk of
// chunk j+1), the first range starting at 0 and the last ending at T: the
// ranges partition [0, T).  Skipping is exact: a tile pair contributes only if
// both tiles are occupied.
// The k-tiles of one P occupancy word go to the lanes (lane l takes the l-th
// set bit), so the Q occupancy loads of a word are issued together; per-block
// counts and chunk boundaries live in shared memory (one region per warp).
__device__ __forceinline__ DevMat resolve_operand(const MatSlot &s, uint8_t use_delta, uint32_t iter) {
    if (!use_delta || iter == 0) return s.cur;
    return s.dlt[iter & 1];
}

// Position of the n-th (0-based) set bit of x (x has more than n set bits).
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t x, uint32_t n) {
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t s = 16; s > 0; s >>= 1) {
        const uint32_t c = __popc(x & ((1u << s) - 1));
        if (n >= c) {
            n -= c;
            x >>= s;
            pos += s;
        }
    }
    return pos;
}

constexpr uint32_t kPlanMaxBlocks = 512;  // T <= 2048 tiles, blocks of >= 4 tiles

// Per-warp shared memory of the planner for up to kBlocks output blocks per
// tile-row (512: any product; 128: word-level products, blocks of 16 tiles).
template <uint32_t kBlocks>
struct WarpArea {
    uint32_t cnt[kBlocks];
    uint16_t bnd[kBlocks][kMaxChunksPerBlock - 1];
};

// Plan product row gw (one warp): items go to list 0 (LOP3 inner loop), 1
// (Four Russians) or 2 (tensor cores) by the product's variant, list l at
// items_all + l * list_cap, counted in item_count[l]; st receives the
// product statistics.  tc_mode 0 plans word-level products, 1 tensor-core ones.
// unified_m4r non-null: every word-level item goes to list 0, Four Russians
// items marked by bit 0 of the item and also counted in *unified_m4r.
__device__ __forceinline__ void plan_row(uint32_t gw, const ProdDesc *__restrict__ prods, uint32_t nprods,
                                         const MatSlot *__restrict__ slots, uint32_t iter, IterState *st,
                                         uint32_t *item_count, uint64_t *__restrict__ items_all, size_t list_cap,
                                         int tpb, uint32_t *prod_seen, int tc_mode, const PlanSelect &ps,
                                         uint32_t *cnt, uint16_t (*bnd)[kMaxChunksPerBlock - 1],
                                         uint32_t plo = 0, uint32_t phi = 0xFFFFFFFFu,
                                         uint32_t *unified_m4r = nullptr) {
    const uint32_t lane = threadIdx.x & 31;
    // product: last p with row_start <= gw, searched in [plo, phi) (a query's
    // products when the caller knows the query)
    uint32_t lo = plo, hi = phi < nprods ? phi : nprods;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (prods[mid].row_start <= gw) lo = mid; else hi = mid;
    }
    const ProdDesc pd = prods[lo];
    if (pd.term == 1 && iter == 0) return;  // first iteration: delta(A) = A, one term covers A*B
    if (ps.q_last && iter > 0 && ps.q_last[pd.query] != iter) return;  // both terms read an empty delta
    uint32_t variant;  // this iteration's variant of the product
    if (ps.sel && !tc_mode) {
        float f[kSelFeatures], pred[kSelOutputs] = {0.f, 0.f, 0.f};
        uint32_t flags = 0;
        variant = sel::select_product(pd, ps.cnts, iter, ps.sel, ps.tc_ok && ps.tc_ok[lo], f, pred, &flags);
        if (gw == pd.row_start && (threadIdx.x & 31) == 0) {
            ps.choice[lo] = (uint8_t)variant;
            if (ps.log && iter < ps.log_iters) {
                SelLogRow &r = ps.log[(size_t)iter * nprods + lo];
                for (int i = 0; i < kSelFeatures; ++i) r.f[i] = f[i];
                for (int o = 0; o < kSelOutputs; ++o) r.pred[o] = pred[o];
                r.choice = variant | flags;
            }
        }
    } else {
        variant = ps.choice ? ps.choice[lo] : pd.variant;
    }
    const bool tc = variant == 4;                                // CFPQ_VARIANT_TC
    if (tc != (tc_mode != 0)) return;  // word-level and tensor-core products are planned by separate launches
    const bool m4r = !tc && variant == 3;                        // CFPQ_VARIANT_M4R
    const uint32_t list = tc ? 2u : (m4r && !unified_m4r ? 1u : 0u);
    const uint64_t vbit = m4r && unified_m4r ? 1u : 0u;
    if (tc) tpb = 4;
    const uint32_t rows_per_item = tc ? 4u : 1u;
    uint64_t *items = items_all + list * list_cap;
    const uint32_t ti = gw - pd.row_start;  // tile-row, or group of 4 tile-rows for tc
    const DevMat P = resolve_operand(slots[pd.pslot], pd.p_delta, iter);
    const DevMat Q = resolve_operand(slots[pd.qslot], pd.q_delta, iter);
    const uint32_t T = pd.T, ow = P.ow;
    const uint32_t bpw = 32 / tpb;  // blocks per occupancy word
    const uint32_t bmask = tpb == 32 ? 0xffffffffu : ((1u << tpb) - 1);
    const uint32_t nblocks = (T + tpb - 1) / tpb;
    auto prow_word = [&](uint32_t w) {
        uint32_t bits = 0;
        for (uint32_t g = 0; g < rows_per_item && ti * rows_per_item + g < T; ++g)
            bits |= P.occ[(size_t)(ti * rows_per_item + g) * ow + w];
        return bits;
    };
    // occupied P tiles of the row (group); the first 32 occupancy words stay
    // in registers (one per lane) for the main loop
    const uint32_t first = lane < ow ? prow_word(lane) : 0u;
    uint32_t np = __reduce_add_sync(kFull, (uint32_t)__popc(first));
    for (uint32_t base = 32; base < ow; base += 32)
        np += __reduce_add_sync(kFull, base + lane < ow ? (uint32_t)__popc(prow_word(base + lane)) : 0u);
    if (!np) return;
    const uint32_t E = tc ? T : item_entries(np);
    for (uint32_t b = lane; b < nblocks; b += 32) cnt[b] = 0;
    __syncwarp();
    // Q occupancy words m[0..3] (words w0.. of Q row tk, tk the lane's
    // candidate) -> per output block b the count of candidate k-tiles and the
    // chunk boundaries
    auto scan = [&](uint32_t w0, const uint32_t (&m)[4], uint32_t tk) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (w0 + u >= ow) break;
            if (!__ballot_sync(kFull, m[u] != 0)) continue;
            for (uint32_t h = 0; h < bpw; ++h) {
                const unsigned bal = __ballot_sync(kFull, ((m[u] >> (h * tpb)) & bmask) != 0);
                if (!bal) continue;
                const uint32_t b = (w0 + u) * bpw + h, c = __popc(bal), cb = cnt[b];
                // chunk boundaries: ranks j*E (j >= 1) among this ballot's ranks cb .. cb+c-1
                for (uint32_t j = (cb + E - 1) / E; j < kMaxChunksPerBlock && j * E < cb + c; ++j) {
                    if (j == 0) continue;
                    const uint32_t src = nth_set_bit(bal, j * E - cb);
                    const uint32_t tkj = __shfl_sync(kFull, tk, src);
                    if (lane == 0) bnd[b][j - 1] = (uint16_t)tkj;
                }
                __syncwarp();
                if (lane == 0) cnt[b] = cb + c;
                __syncwarp();
            }
        }
    };
    if (ow <= 4) {
        // at most 128 tiles: the Q words of every candidate load together
        // (one round trip), lane l holding the l-th candidate of each P word
        uint32_t pre[4][4], tks[4];
#pragma unroll
        for (int pw = 0; pw < 4; ++pw) {
            const uint32_t bits = __shfl_sync(kFull, first, pw);  // 0 beyond ow
            const bool valid = lane < (uint32_t)__popc(bits);
            tks[pw] = valid ? pw * 32 + nth_set_bit(bits, lane) : 0u;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                pre[pw][u] = (valid && (uint32_t)u < ow) ? Q.occ[(size_t)tks[pw] * ow + u] : 0u;
        }
#pragma unroll
        for (int pw = 0; pw < 4; ++pw)
            if (__shfl_sync(kFull, first, pw)) scan(0, pre[pw], tks[pw]);
    } else {
        uint32_t mine = first;
        for (uint32_t pw = 0; pw < ow; ++pw) {
            // P occupancy words come 32 at a time, one per lane
            if (pw > 0 && (pw & 31) == 0) mine = pw + lane < ow ? prow_word(pw + lane) : 0u;
            const uint32_t bits = __shfl_sync(kFull, mine, pw & 31);  // warp-uniform
            if (!bits) continue;
            const bool valid = lane < (uint32_t)__popc(bits);
            const uint32_t tk = valid ? pw * 32 + nth_set_bit(bits, lane) : 0u;  // increasing with the lane
            const uint32_t *qrow = Q.occ + (size_t)tk * ow;
            for (uint32_t w0 = 0; w0 < ow; w0 += 4) {
                uint32_t m[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) m[u] = (valid && w0 + u < ow) ? qrow[w0 + u] : 0u;
                scan(w0, m, tk);
            }
        }
    }

    auto nchunks = [&](uint32_t c) { return c ? (c + E - 1) / E : 0u; };
    uint32_t total = 0;
    for (uint32_t base = 0; base < nblocks; base += 32) {
        const uint32_t b = base + lane;
        total += __reduce_add_sync(kFull, b < nblocks ? nchunks(cnt[b]) : 0u);
    }
    if (!total) return;
    uint32_t pos0 = 0;
    if (lane == 0) {
        pos0 = atomicAdd(&item_count[list], total);
        if (vbit) atomicAdd(unified_m4r, total);
    }
    pos0 = __shfl_sync(kFull, pos0, 0);
    for (uint32_t base = 0; base < nblocks; base += 32) {
        const uint32_t b = base + lane;
        const uint32_t nitem = b < nblocks ? nchunks(cnt[b]) : 0u;
        uint32_t pre = nitem;  // inclusive scan over lanes
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, pre, o);
            if (lane >= (uint32_t)o) pre += v;
        }
        for (uint32_t j = 0; j < nitem; ++j) {
            const uint32_t klo = j ? bnd[b][j - 1] : 0u, khi = j + 1 < nitem ? bnd[b][j] : T;
            items[pos0 + pre - nitem + j] = make_item(lo, ti, b, klo, khi) | vbit;
        }
        pos0 += __shfl_sync(kFull, pre, 31);
    }
    if (lane == 0 && prod_seen) {
        if (atomicExch(&prod_seen[lo], iter + 1) != iter + 1) {
            atomicAdd(&st->products, 1ULL);
            atomicAdd(&st->dense_bitops, (unsigned long long)pd.n * pd.n * pd.n);
        }
    }
}

}  // namespace plan
}  // namespace cfpq
