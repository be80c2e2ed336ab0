// Tiled Boolean product C |= P * Q over the work items of one closure
// iteration (or one add_mul), with two dense inner loops:
//   variant LOP3  (item list 0): word-level AND/OR with LOP3
//   variant M4R   (item list 1): Four Russians with 4-bit tables in shared memory
//
// Work item = (product, output tile-row ti, block of kBJ output tiles, chunk of
// contributing k-tiles).  A CTA of 4 warps owns the 64 x (64*kBJ) output block
// in registers: warp w owns tiles 4w..4w+3 of the block, lane l owns rows 2l
// and 2l+1, so every thread keeps 2 rows x 4 tiles x 64 bits = 16 uint32
// accumulators.
//
// Inner dimension: the contributing k-tiles tk (occupied P tile (ti, tk) and a
// non-empty Q block (tk, block)) of the item's k-tile range, in increasing tk
// order.  One elected thread stages,
// per k-tile, the P tile (512 B) and the Q tiles with bulk copies
// (cp.async.bulk, the TMA engine) completing on an mbarrier, four k-tiles in flight,
// and the CTA runs one of three inner loops on the staged tiles, chosen by the
// population of the P tile:
//   dense  (population > kSparseMax), all kBJ Q tiles staged (one contiguous
//          range of the tiled layout, empty tiles are zeros):
//          LOP3: per row and inner index k, mask = -(P[row] bit k) (2 ALU
//          ops), then acc |= mask & Q[k] on 8 uint32 words (one LOP3 each); Q
//          rows k, k+1 of a tile come in one 16-byte shared load read by all
//          lanes of the warp at the same address (broadcast).
//          M4R: the CTA first builds, for each of the 16 four-bit slabs of the
//          k-tile and each of the kBJ Q tiles, the 16 ORs of the slab's Q rows
//          (a table row per key, padded to 17 words so that lanes reading
//          different keys hit different banks); each row then ORs one table
//          word per slab and tile: 16 loads instead of 64 masked LOP3s.
//   sparse (population <= kSparseMax), only the range of occupied Q tiles
//          staged: a thread walks up to kLaneBits set bits k of each of its
//          two P rows and ORs row k of each occupied Q tile of its warp from
//          shared memory; the bits left in rows of hub vertices are spread
//          over the warp's lanes one row at a time and OR-reduced.
// A warp skips its empty Q tiles (all of them: no inner loop at all).
//
// Epilogue: for each non-zero accumulator word, new = acc & ~old via a 64-bit
// atomicOr (several products of one iteration may write the same head); new
// bits also go to the head's next-delta matrix D; occupancy bits and tile
// populations of C and D are updated.  Concurrent reads of matrices that other
// CTAs are OR-ing into are safe: every bit only goes 0 -> 1, so a read sees a
// subset of the final value and a superset of the iteration-start value.
#include "launch.h"
#include "product_tiled.cuh"

namespace cfpq {

namespace {

using namespace tiled;

template <bool kM4R>
__global__ void __launch_bounds__(kThreads, 4)
    k_product_tiled(const ProdDesc *__restrict__ prods, const MatSlot *__restrict__ slots, IterState *st,
                    const uint64_t *__restrict__ items_all, size_t list_cap, uint32_t *qchanged, BufCounters *cnts) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TiledSmem<kM4R> &S = *reinterpret_cast<TiledSmem<kM4R> *>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    const uint32_t list = kM4R ? 1u : 0u;
    const uint64_t *items = items_all + list * list_cap;

    if (tid == 0) {
        for (uint32_t i = 0; i < tiled::kStages; ++i) mbar_init(&S.bar[i], 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;  // bit s = next parity to wait for on stage s
    const uint32_t iter = st->iter;
    const uint32_t nitems = st->item_count[list];
    ItemCounters ctr;
    bool timed_out = false;

    for (;;) {
        if (tid == 0) S.item = atomicAdd(&st->item_next[list], 1u);
        __syncthreads();
        const uint32_t idx = S.item;
        if (idx >= nitems) break;
        process_item<kM4R, kThreads / 32>(S, items[idx], prods, slots, iter, &st->changed, qchanged, phase, timed_out, ctr, cnts);
    }
    // per-CTA counters (warp-reduced) for statistics and the roofline report
    unsigned long long triples = ctr.triples, outw = ctr.outw, neww = ctr.neww;
    for (int o = 16; o > 0; o >>= 1) {
        triples += __shfl_down_sync(kFull, triples, o);
        outw += __shfl_down_sync(kFull, outw, o);
        neww += __shfl_down_sync(kFull, neww, o);
    }
    if (lane == 0) {
        if (triples) atomicAdd(&st->tile_triples, triples);
        if (outw) atomicAdd(&st->out_words, outw);
        if (neww) atomicAdd(&st->new_words, neww);
    }
    if (tid == 0 && ctr.staged) atomicAdd(&st->bytes_staged, ctr.staged);
    if (timed_out && tid == 0) atomicExch(&st->error, 5u);
}

}  // namespace

int product_lop3_tiles_per_block() { return kBJ; }
int product_lop3_max_tiles() { return kMaxTiles; }

int product_tiled_blocks_per_sm(int m4r) {
    int nb = 0;
    if (m4r) {
        cudaFuncSetAttribute(k_product_tiled<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TiledSmem<true>));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_product_tiled<true>, kThreads, sizeof(TiledSmem<true>));
    } else {
        cudaFuncSetAttribute(k_product_tiled<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TiledSmem<false>));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_product_tiled<false>, kThreads,
                                                      sizeof(TiledSmem<false>));
    }
    return nb > 0 ? nb : 1;
}

cudaError_t launch_product_tiled(int m4r, const ProdDesc *d_prods, const MatSlot *d_slots, IterState *d_st,
                                 const uint64_t *d_items, size_t list_cap, uint32_t *d_qchanged, int grid,
                                 BufCounters *d_cnts, cudaStream_t s) {
    if (m4r)
        k_product_tiled<true><<<grid, kThreads, sizeof(TiledSmem<true>), s>>>(d_prods, d_slots, d_st, d_items, list_cap,
                                                                              d_qchanged, d_cnts);
    else
        k_product_tiled<false><<<grid, kThreads, sizeof(TiledSmem<false>), s>>>(d_prods, d_slots, d_st, d_items,
                                                                                list_cap, d_qchanged, d_cnts);
    return cudaGetLastError();
}

}  // namespace cfpq
