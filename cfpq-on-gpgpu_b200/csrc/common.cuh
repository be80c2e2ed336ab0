// Internal definitions shared by the CUDA sources of libcfpq_b200.so.
//
// Device matrix layout ("tiled bits"): an n x n Boolean matrix is padded to
// np = ceil(n/64)*64 and split into T x T tiles of 64 x 64 bits, T = np/64.
// Tile (ti, tj) is 64 consecutive uint64 words at word offset (ti*T + tj)*64;
// word r of the tile holds row ti*64 + r, columns tj*64 .. tj*64+63, column
// tj*64 + b at bit b.  A tile is 512 contiguous bytes, so a block of tiles along
// a tile-row is one contiguous range that a single bulk copy can stage.
//
// Occupancy bitmap: one bit per tile, row ti of the bitmap is `ow` uint32
// words (ow = ceil(T/32)), tile (ti, tj) at bit tj % 32 of word ti*ow + tj/32.
// Invariant at every API boundary and at every kernel boundary of the closure:
// a tile that holds a set bit has its occupancy bit set.  (A set occupancy bit
// does not promise a non-zero tile.)  Bits of padding rows/columns (>= n) are
// always zero.
//
// Tile population: nnz[ti*T + tj] counts the set bits of tile (ti, tj).  It is
// exact at API boundaries and at the kernel boundaries of the closure; product
// kernels only use it to choose between the dense and the sparse inner loop,
// never to decide which bits exist.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cfpq {

constexpr int kTileBits = 64;   // tile side
constexpr int kTileWords = 64;  // uint64 words per tile

struct DevMat {
    uint64_t *bits;   // T*T*64 words
    uint32_t *occ;    // T*ow words
    uint32_t *nnz;    // T*T tile populations
    const uint32_t *perm;  // vertex order: internal index of vertex v (null = identity)
    uint32_t T;       // tiles per side
    uint32_t ow;      // occupancy words per tile-row
    uint32_t n;       // logical size
    uint32_t pad;
};

// One nonterminal matrix of a closure: the current matrix and two delta
// buffers used alternately (bits added in the previous / current iteration).
struct MatSlot {
    DevMat cur;
    DevMat dlt[2];
    uint32_t query;
    uint32_t row_start;  // prefix sum of T over slots (advance grid mapping)
};

// One product term of a closure iteration: C |= P * Q, new bits also into the
// head's "next" delta.  Operands are slots; p_delta / q_delta select the
// slot's previous-iteration delta instead of its current matrix.
struct ProdDesc {
    uint32_t head, pslot, qslot;
    uint8_t p_delta, q_delta, term, variant;
    uint32_t query, rule;
    uint32_t T;
    uint32_t n;
    uint32_t row_start;  // prefix sum of T over products (plan grid mapping)
};

// Device-resident iteration state of a closure (one per context).
struct IterState {
    uint32_t iter;          // iteration index (parity selects delta buffers)
    uint32_t item_count[3]; // work items written by the plan kernel, per list
                            // (list 0: LOP3 inner loop, 1: Four Russians, 2: tensor cores)
    uint32_t item_next[3];  // work-stealing counters of the product kernels
    uint32_t changed;       // set when any new bit appeared in this iteration
    uint32_t last_changed;  // copy of `changed` at the end of the iteration
    uint32_t error;         // nonzero: a bounded wait gave up (cfpq_status)
    uint32_t max_iter;      // 0 = unbounded
    uint32_t active;        // loop condition mirror (1 while iterating)
    uint32_t nqueries;
    uint32_t blocks_done;   // blocks of the advance kernel that finished (the last one ends the iteration)
    // persistent closure kernel: per-parity iteration counters
    uint32_t pitem_m4r[2];       // Four Russians items among the items counted in pplan[.]
    // polled by every CTA of the persistent kernel: own cache lines
    // plan word of the iterations of parity p: the low 32 bits count the work
    // items written (the planners' item_count[0]), the high 32 bits the CTAs
    // done with their plan/clear units; one load returns both
    alignas(128) unsigned long long pplan[2];
    alignas(128) uint32_t pitem_next[2][2];
    // grid barrier of the iterations of parity p: low 32 bits count the CTAs'
    // arrivals (cumulative over the closure), high 32 bits are the
    // iteration's flags (kBarChanged, kBarAbort), read with the count
    alignas(128) unsigned long long pbar[2];
    unsigned long long tile_triples;
    unsigned long long items_total;
    unsigned long long products;      // non-empty product terms over all iterations
    unsigned long long dense_bitops;  // sum of n^3 over those products
    unsigned long long t_start_ns;    // %globaltimer at the first plan
    unsigned long long items_by_variant[5];
    unsigned long long bytes_staged;  // operand bytes copied global -> shared by product kernels
    unsigned long long out_words;     // non-zero accumulator words merged into heads
    unsigned long long new_words;     // words that received new bits
    uint32_t exit_count;              // persistent kernel: CTAs past their exit statistics
};

// A matrix and the prefix sum of tile-rows over a list of matrices (kernels
// with one warp per (matrix, tile-row)).
struct MatRows {
    DevMat m;
    uint32_t row_start;
    uint32_t pad;
};

// Statistics of one buffer of a closure (a slot's current matrix or one of
// its two deltas), kept exact by the product epilogues and reset when a delta
// is cleared: population, occupied tiles (occupancy bits), dense tiles
// (population > kDenseTilePop).  Buffer b of slot s is counters[3*s + b]
// (b = 0: current matrix, 1 + d: delta d).  They are the selector's features.
struct BufCounters {
    unsigned long long nnz;
    uint32_t occ_tiles;
    uint32_t dense_tiles;
};
constexpr uint32_t kDenseTilePop = 96;

// Variant selector (device-resident).  Feature vector of a product term,
// predicted log-microseconds per candidate variant (LOP3, M4R, TC).
constexpr int kSelFeatures = 16;
constexpr int kSelHidden = 64;
constexpr int kSelOutputs = 3;
constexpr int kSelWeights = kSelFeatures * kSelHidden + kSelHidden + kSelHidden * kSelHidden + kSelHidden +
                            kSelHidden * kSelOutputs + kSelOutputs;
struct SelectorParams {
    int32_t mode;           // 0 fixed, 1 heuristic, 2 MLP with heuristic fallback
    uint32_t allowed;       // bit v: variant v may be chosen
    uint32_t tc_min_tiles;  // tensor cores only for products with T >= tc_min_tiles
    float tc_min_occ, tc_min_dense, m4r_min_dense;
    float conf_margin, range_margin;
    uint32_t min_tiles;     // closures whose largest term has fewer tile-rows run LOP3 throughout
    int32_t has_weights;
    float feat_lo[kSelFeatures], feat_hi[kSelFeatures];  // training range of every feature
    float w[kSelWeights];   // W1 [F][H], b1 [H], W2 [H][H], b2 [H], W3 [H][O], b3 [O]
};

// One row of the selection log: the features of (iteration, product), the
// MLP's predictions (if it ran) and the choice (bits 0-7 variant, bit 8: the
// MLP decided, bit 9: the MLP ran but fell back to the heuristic).
struct SelLogRow {
    float f[kSelFeatures];
    float pred[kSelOutputs];
    uint32_t choice;
};

// Variant source of the planner.  sel non-null: the planner's warps decide
// every word-level plan's variant themselves from the buffer counters (every
// row of a product gets the same answer; the warp of tile-row 0 stores it in
// choice[] and the selection log), and the tensor-core plan reads choice[].
// sel null: choice[] (or, if null too, the product's own variant).
struct PlanSelect {
    const SelectorParams *sel;
    const BufCounters *cnts;
    const uint8_t *tc_ok;
    uint8_t *choice;
    SelLogRow *log;
    uint32_t log_iters;
    // non-null (multi-kernel iterations): per query the last iteration
    // (1-based) in which it changed; a query that did not change in the
    // previous iteration has empty deltas and is not planned
    const uint32_t *q_last;
};

constexpr uint32_t kBarChanged = 1u;  // some product set a new bit
constexpr uint32_t kBarAbort = 2u;    // a CTA gave up a bounded wait

// Rows, slots and products of one query of a closure (all contiguous): plan
// rows [prow0, prow0 + nprow), slot tile-rows [srow0, srow0 + nsrow), slots
// [slot0, slot0 + nslot), products [prod0, prod0 + nprod).
struct QueryRange {
    uint32_t prow0, nprow, srow0, nsrow, slot0, nslot, prod0, nprod;
};

// One traced work item of a persistent closure (layout of cfpq_item_record).
struct ItemTrace {
    uint64_t item;
    uint32_t iteration;
    uint16_t cta, list;
    unsigned long long start_ns, end_ns;
    uint32_t klist_ns, staged_ns, computed_ns, gate_ns;  // after start_ns
};
constexpr uint32_t kItemTraceCap = 65536;

// Largest batch whose persistent closure plans over active queries only.
constexpr uint32_t kMaxActiveQueries = 512;

// Per-query bookkeeping of a batched closure (device arrays of nqueries).
struct QueryTrack {
    uint32_t *changed;              // set by product kernels in the current iteration
    uint32_t *last_iter;            // last iteration (1-based) in which the query changed
    unsigned long long *done_ns;    // %globaltimer at the end of that iteration
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
#ifdef __CUDA_ARCH__
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
#else
    return 0;
#endif
}

// Work item: (product, output tile-row ti, output tile-column block tjb,
// inner-dimension range [klo, khi)).  The item processes the k-tiles tk in its
// range that contribute to the block (occupied P tile (ti, tk) and a non-empty
// Q block (tk, tjb)).  The ranges of one block partition [0, T), so every
// k-tile present when the iteration started is processed exactly once (a
// k-tile that appears during the iteration may be processed or not: its bits
// are also in the next delta).  Items of the same output block are
// independent: their partial products are OR-ed into the head atomically.
// Fields: p 16 bits, ti 11, tjb 9, klo 12, khi 12 (T <= 2048).
constexpr uint32_t kMaxItemProducts = 1u << 16;
__host__ __device__ inline uint64_t make_item(uint32_t p, uint32_t ti, uint32_t tjb, uint32_t klo, uint32_t khi) {
    return ((uint64_t)p << 48) | ((uint64_t)ti << 37) | ((uint64_t)tjb << 28) | ((uint64_t)klo << 16) |
           ((uint64_t)khi << 4);
}
__host__ __device__ inline uint32_t item_prod(uint64_t it) { return (uint32_t)(it >> 48); }
__host__ __device__ inline uint32_t item_ti(uint64_t it) { return (uint32_t)((it >> 37) & 0x7FF); }
__host__ __device__ inline uint32_t item_tjb(uint64_t it) { return (uint32_t)((it >> 28) & 0x1FF); }
__host__ __device__ inline uint32_t item_klo(uint64_t it) { return (uint32_t)((it >> 16) & 0xFFF); }
__host__ __device__ inline uint32_t item_khi(uint64_t it) { return (uint32_t)((it >> 4) & 0xFFF); }

// Chunk length of the word-level items of a tile-row whose P operand has `np`
// occupied tiles: at most kMaxChunksPerBlock chunks per output block (short
// chains keep the per-item latency low when an iteration has few blocks; each
// chunk re-does the block's epilogue).  (Finer chunking of small closures,
// more and shorter items, measured slower: the planner's boundary work and
// the extra items outweigh the shorter longest item.)
constexpr uint32_t kMaxChunksPerBlock = 8;

// Bits of occupancy word w (tiles 32w .. 32w+31) that lie in [lo, hi).
__host__ __device__ inline uint32_t range_word_mask(uint32_t w, uint32_t lo, uint32_t hi) {
    const int a = (int)lo - (int)(w * 32), z = (int)hi - (int)(w * 32);
    uint32_t m = 0xffffffffu;
    if (a > 0) m = a >= 32 ? 0u : (m & (0xffffffffu << a));
    if (z < 32) m = z <= 0 ? 0u : (m & (0xffffffffu >> (32 - z)));
    return m;
}
__host__ __device__ inline uint32_t item_entries(uint32_t np) {
    const uint32_t e = (np + kMaxChunksPerBlock - 1) / kMaxChunksPerBlock;
    return e < 1 ? 1 : e;
}
// Tensor-core items keep the whole inner dimension ([0, T), one chunk): their
// TMEM epilogue is amortised over every k-tile of the 256 x 256 block.

__host__ __device__ inline size_t tile_offset(uint32_t T, uint32_t ti, uint32_t tj) {
    return ((size_t)ti * T + tj) * kTileWords;
}

#ifdef __CUDACC__

// ---- mbarrier + bulk copy (TMA engine, 1D) helpers -------------------------

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// GPU-scope acquire / release accesses (a release publishes every write that
// happens before it, including the CTA's writes ordered by a preceding
// __syncthreads; an acquire orders every later access after it).
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long atom_add_acq_rel_u64(unsigned long long *p, unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}
__device__ __forceinline__ void red_add_release_u32(uint32_t *p, uint32_t v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global to this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait: each try_wait suspends for a hardware-defined time slice; the
// iteration limit bounds the wait to well under a minute.  Returns false when
// the limit is hit.
constexpr uint32_t kWaitLimit = 1u << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase) {
    for (uint32_t i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// Lanes 0..3 of a warp, lane j for tile tj0 + j (add[j] new bits, 0: none):
// tile populations and occupancy bits of m, then (cnt non-null) the buffer
// counters, aggregated over the 4 tiles into one update per counter.
__device__ __forceinline__ void tiles_gain(const DevMat &m, uint32_t ti, uint32_t tj0, uint32_t add,
                                           BufCounters *cnt) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t tj = tj0 + lane;
    uint32_t gained = 0, dense = 0;
    if (lane < 4 && add) {
        const size_t t = (size_t)ti * m.T + tj;
        const uint32_t bit = 1u << (tj & 31);
        if (cnt) {
            const uint32_t old_pop = atomicAdd(m.nnz + t, add);
            const uint32_t old_occ = atomicOr(m.occ + (size_t)ti * m.ow + (tj >> 5), bit);
            gained = (old_occ & bit) ? 0u : 1u;
            dense = (old_pop <= kDenseTilePop && old_pop + add > kDenseTilePop) ? 1u : 0u;
        } else {
            atomicAdd(m.nnz + t, add);
            atomicOr(m.occ + (size_t)ti * m.ow + (tj >> 5), bit);
        }
    }
    if (!cnt) return;
    const uint32_t sum_add = __reduce_add_sync(0xffffffffu, lane < 4 ? add : 0u);
    const uint32_t sum_gained = __reduce_add_sync(0xffffffffu, gained);
    const uint32_t sum_dense = __reduce_add_sync(0xffffffffu, dense);
    if (lane == 0) {
        if (sum_add) atomicAdd(&cnt->nnz, sum_add);
        if (sum_gained) atomicAdd(&cnt->occ_tiles, sum_gained);
        if (sum_dense) atomicAdd(&cnt->dense_tiles, sum_dense);
    }
}

// One warp: clear tile-row ti of D -- zero every occupied tile and its
// population, then the occupancy row (tiles without an occupancy bit hold no
// bit and have population 0).  The occupancy words come 32 at a time, one per
// lane, so a row costs one load round trip; the zeroing stores are not
// waited for.
__device__ __forceinline__ void clear_tile_row(const DevMat &D, uint32_t ti) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t *orow = D.occ + (size_t)ti * D.ow;
    for (uint32_t base = 0; base < D.ow; base += 32) {
        const uint32_t mine = base + lane < D.ow ? orow[base + lane] : 0u;
        unsigned todo = __ballot_sync(0xffffffffu, mine != 0);
        while (todo) {
            const uint32_t src = __ffs(todo) - 1;
            todo &= todo - 1;
            uint32_t bits = __shfl_sync(0xffffffffu, mine, src);
            while (bits) {
                const uint32_t tj = (base + src) * 32 + (__ffs(bits) - 1);
                bits &= bits - 1;
                uint4 *tile = reinterpret_cast<uint4 *>(D.bits + tile_offset(D.T, ti, tj));
                tile[lane] = make_uint4(0, 0, 0, 0);
                if (lane == 0) D.nnz[(size_t)ti * D.T + tj] = 0;
            }
        }
        __syncwarp();
        if (mine) orow[base + lane] = 0;
    }
}

// One warp: clear tile-row `row` (over all slots, slot tile-rows in order) of
// the delta buffer dlt[parity].
__device__ __forceinline__ void clear_delta_row(const MatSlot *__restrict__ slots, uint32_t nslots, uint32_t row,
                                                uint32_t parity, uint32_t slo = 0, uint32_t shi = 0xFFFFFFFFu) {
    uint32_t lo = slo, hi = shi < nslots ? shi : nslots;  // slot search range (a query's slots if known)
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (slots[mid].row_start <= row) lo = mid; else hi = mid;
    }
    clear_tile_row(slots[lo].dlt[parity], row - slots[lo].row_start);
}

#endif  // __CUDACC__

}  // namespace cfpq
