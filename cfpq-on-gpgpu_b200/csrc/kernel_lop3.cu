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
// (cp.async.bulk, the TMA engine) completing on an mbarrier, double-buffered,
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
//          staged: a thread walks the set bits k of its two P rows and ORs
//          row k of each occupied Q tile of its warp from shared memory.
// A warp whose 4 Q tiles are all empty skips the inner loop.
//
// Epilogue: for each non-zero accumulator word, new = acc & ~old via a 64-bit
// atomicOr (several products of one iteration may write the same head); new
// bits also go to the head's next-delta matrix D; occupancy bits and tile
// populations of C and D are updated.  Concurrent reads of matrices that other
// CTAs are OR-ing into are safe: every bit only goes 0 -> 1, so a read sees a
// subset of the final value and a superset of the iteration-start value.
#include "launch.h"

namespace cfpq {

namespace {

constexpr int kBJ = 16;              // output tiles per work item (1024 columns)
constexpr int kThreads = 128;        // 4 warps
constexpr int kMaxTiles = 2048;      // k-list capacity (n <= 131072)
constexpr uint32_t kSparseMax = 96;  // P-tile population up to which the sparse loop runs
constexpr int kTabRow = kBJ + 1;     // padded table row (uint64 words)
constexpr unsigned kFull = 0xffffffffu;

template <bool kM4R>
struct __align__(128) TiledSmem {
    uint64_t q[2][kBJ * 64];     // 2 x 8 KiB
    uint64_t p[2][64];           // 2 x 512 B
    uint64_t tab[kM4R ? 16 * 16 * kTabRow : 1];  // M4R tables [slab][key][tile], 34 KiB
    uint64_t bar[2];
    uint16_t cand[kMaxTiles];    // occupied P tiles of the item's tile-row
    uint16_t cmask[kMaxTiles];   // their Q block occupancy
    uint32_t rball[kMaxTiles / 32], roff[kMaxTiles / 32];  // per-round ballots and rank offsets
    uint16_t ktile[kMaxTiles];   // the item's k-tiles, increasing; bit 15: dense P tile
    uint16_t kmask[kMaxTiles];   // their Q block occupancy
    uint32_t nc, nk;
    uint32_t item;
};

__device__ __forceinline__ DevMat resolve_operand(const MatSlot &s, uint8_t use_delta, uint32_t iter) {
    if (!use_delta || iter == 0) return s.cur;
    return s.dlt[iter & 1];
}

__device__ __forceinline__ uint32_t bitmask(uint32_t word, int b) {
    // all-ones if bit b of word is set, else zero
    return (uint32_t)((int32_t)(word << (31 - b)) >> 31);
}

__device__ __forceinline__ void or64(uint2 &a, uint64_t v) {
    a.x |= (uint32_t)v;
    a.y |= (uint32_t)(v >> 32);
}

template <bool kM4R>
__global__ void __launch_bounds__(kThreads, 4)
    k_product_tiled(const ProdDesc *__restrict__ prods, const MatSlot *__restrict__ slots, IterState *st,
                    const uint64_t *__restrict__ items_all, size_t list_cap, uint32_t *qchanged) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TiledSmem<kM4R> &S = *reinterpret_cast<TiledSmem<kM4R> *>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t list = kM4R ? 1u : 0u;
    const uint64_t *items = items_all + list * list_cap;

    if (tid == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;  // bit s = next parity to wait for on stage s
    const uint32_t iter = st->iter;
    const uint32_t nitems = st->item_count[list];
    unsigned long long triples = 0, staged = 0, outw = 0, neww = 0;
    bool timed_out = false;

    for (;;) {
        if (tid == 0) S.item = atomicAdd(&st->item_next[list], 1u);
        __syncthreads();
        const uint32_t idx = S.item;
        if (idx >= nitems) break;
        const uint64_t it = items[idx];
        const ProdDesc pd = prods[item_prod(it)];
        const uint32_t ti = item_ti(it), tjb = item_tjb(it), klo = item_klo(it), khi = item_khi(it);
        const DevMat P = resolve_operand(slots[pd.pslot], pd.p_delta, iter);
        const DevMat Q = resolve_operand(slots[pd.qslot], pd.q_delta, iter);
        const DevMat C = slots[pd.head].cur;
        const DevMat D = slots[pd.head].dlt[(iter & 1) ^ 1];
        const uint32_t T = pd.T, ow = P.ow;
        const uint32_t tj0 = tjb * kBJ;
        const uint32_t nblk = min((uint32_t)kBJ, T - tj0);
        const uint32_t qword = tj0 >> 5, qshift = tj0 & 31;

        // ---- k-list: warp 0 compacts the occupied P tiles of row ti in
        // [klo, khi) into a candidate list, then all threads classify the
        // candidates in parallel ----
        if (warp == 0) {
            uint32_t nc = 0;
            const uint32_t *prow = P.occ + (size_t)ti * ow;
            for (uint32_t base = 0; base < ow; base += 32) {
                uint32_t bits = (base + lane < ow) ? prow[base + lane] & range_word_mask(base + lane, klo, khi) : 0u;
                const uint32_t cnt = __popc(bits);
                uint32_t pre = cnt;  // inclusive scan over lanes
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(kFull, pre, o);
                    if (lane >= (uint32_t)o) pre += v;
                }
                uint32_t pos = nc + pre - cnt;
                while (bits) {
                    S.cand[pos++] = (uint16_t)((base + lane) * 32 + (__ffs(bits) - 1));
                    bits &= bits - 1;
                }
                nc += __shfl_sync(kFull, pre, 31);
            }
            if (lane == 0) S.nc = nc;
        }
        __syncthreads();
        // rank the candidates with a non-empty Q block in increasing tk order
        // (ballot per round of 32)
        const uint32_t nc = S.nc, rounds = (nc + 31) / 32;
        for (uint32_t r = warp; r < rounds; r += kThreads / 32) {
            const uint32_t c = r * 32 + lane;
            uint32_t mask = 0;
            if (c < nc) mask = (Q.occ[(size_t)S.cand[c] * ow + qword] >> qshift) & ((1u << kBJ) - 1);
            const unsigned ball = __ballot_sync(kFull, mask != 0);
            if (c < nc) S.cmask[c] = (uint16_t)mask;
            if (lane == 0) S.rball[r] = ball;
        }
        __syncthreads();
        if (warp == 0) {  // exclusive prefix of the per-round counts
            uint32_t carry = 0;
            for (uint32_t base = 0; base < rounds; base += 32) {
                const uint32_t r = base + lane;
                const uint32_t cnt = r < rounds ? __popc(S.rball[r]) : 0;
                uint32_t pre = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(kFull, pre, o);
                    if (lane >= (uint32_t)o) pre += v;
                }
                if (r < rounds) S.roff[r] = carry + pre - cnt;
                carry += __shfl_sync(kFull, pre, 31);
            }
        }
        __syncthreads();
        for (uint32_t c = tid; c < nc; c += kThreads) {
            const uint32_t mask = S.cmask[c];
            if (!mask) continue;
            const uint32_t rank = S.roff[c >> 5] + __popc(S.rball[c >> 5] & ((1u << (c & 31)) - 1));
            const uint32_t tk = S.cand[c];
            triples += __popc(mask);
            const bool dense = P.nnz[(size_t)ti * T + tk] > kSparseMax;
            S.ktile[rank] = (uint16_t)(tk | (dense ? 0x8000u : 0u));
            S.kmask[rank] = (uint16_t)mask;
        }
        if (tid == 0) S.nk = rounds ? S.roff[rounds - 1] + __popc(S.rball[rounds - 1]) : 0u;
        __syncthreads();
        const uint32_t nk = S.nk;

        uint2 acc0[4], acc1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) acc0[j] = acc1[j] = make_uint2(0, 0);

        // ---- staged k-tiles ----
        auto issue = [&](uint32_t e, uint32_t stage) -> uint32_t {
            const uint32_t kt = S.ktile[e], tk = kt & 0x7FFFu, mask = S.kmask[e];
            // dense: the whole block (its empty tiles read as zeros); sparse:
            // the range of occupied tiles only
            const uint32_t lo = (kt & 0x8000u) ? 0u : (uint32_t)(__ffs(mask) - 1);
            const uint32_t hi = (kt & 0x8000u) ? nblk - 1 : 31u - __clz(mask);
            const uint32_t qbytes = (hi - lo + 1) * 512u;
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&S.bar[stage], 512u + qbytes);
            bulk_g2s(S.p[stage], P.bits + tile_offset(T, ti, tk), 512u, &S.bar[stage]);
            bulk_g2s(&S.q[stage][lo * 64], Q.bits + tile_offset(T, tk, tj0 + lo), qbytes, &S.bar[stage]);
            return 512u + qbytes;
        };
        if (tid == 0 && nk > 0) staged += issue(0, 0);
        uint32_t stage = 0;
        for (uint32_t e = 0; e < nk; ++e) {
            if (tid == 0 && e + 1 < nk) staged += issue(e + 1, stage ^ 1);
            if (!timed_out && !mbar_wait_bounded(&S.bar[stage], (phase >> stage) & 1u)) timed_out = true;
            phase ^= 1u << stage;
            const bool dense = (S.ktile[e] & 0x8000u) != 0;
            const uint32_t wmask = ((uint32_t)S.kmask[e] >> (4 * warp)) & 0xFu;
            const uint4 pp = *reinterpret_cast<const uint4 *>(&S.p[stage][2 * lane]);
            if (!dense) {
                // sparse P tile: walk the set bits of rows 2l and 2l+1; only
                // the occupied Q tiles of this warp were staged and are read
                if (wmask && !timed_out) {
                    const uint64_t *q = &S.q[stage][(4 * warp) * 64];
                    uint64_t xa = ((uint64_t)pp.y << 32) | pp.x;
                    uint64_t xb = ((uint64_t)pp.w << 32) | pp.z;
                    while (xa | xb) {
                        if (xa) {
                            const int k = __ffsll((long long)xa) - 1;
                            xa &= xa - 1;
#pragma unroll
                            for (int j = 0; j < 4; ++j)
                                if ((wmask >> j) & 1u) or64(acc0[j], q[j * 64 + k]);
                        }
                        if (xb) {
                            const int k = __ffsll((long long)xb) - 1;
                            xb &= xb - 1;
#pragma unroll
                            for (int j = 0; j < 4; ++j)
                                if ((wmask >> j) & 1u) or64(acc1[j], q[j * 64 + k]);
                        }
                    }
                }
            } else if constexpr (kM4R) {
                // build: (slab s, tile j) pairs over the CTA; 16 keys each
                for (uint32_t pr = tid; pr < 16 * kBJ; pr += kThreads) {
                    const uint32_t s = pr / kBJ, j = pr % kBJ;
                    const uint64_t *qr = &S.q[stage][j * 64 + 4 * s];
                    const uint64_t q0 = qr[0], q1 = qr[1], q2 = qr[2], q3 = qr[3];
                    uint64_t *t = &S.tab[(s * 16) * kTabRow + j];
                    const uint64_t a01 = q0 | q1, a23 = q2 | q3;
                    t[0 * kTabRow] = 0;
                    t[1 * kTabRow] = q0;
                    t[2 * kTabRow] = q1;
                    t[3 * kTabRow] = a01;
                    t[4 * kTabRow] = q2;
                    t[5 * kTabRow] = q0 | q2;
                    t[6 * kTabRow] = q1 | q2;
                    t[7 * kTabRow] = a01 | q2;
                    t[8 * kTabRow] = q3;
                    t[9 * kTabRow] = q0 | q3;
                    t[10 * kTabRow] = q1 | q3;
                    t[11 * kTabRow] = a01 | q3;
                    t[12 * kTabRow] = a23;
                    t[13 * kTabRow] = q0 | a23;
                    t[14 * kTabRow] = q1 | a23;
                    t[15 * kTabRow] = a01 | a23;
                }
                __syncthreads();
                if (wmask && !timed_out) {
                    const uint64_t pa = ((uint64_t)pp.y << 32) | pp.x;  // row 2l
                    const uint64_t pb = ((uint64_t)pp.w << 32) | pp.z;  // row 2l+1
#pragma unroll
                    for (int s = 0; s < 16; ++s) {
                        const uint64_t *ta = &S.tab[(s * 16 + (uint32_t)((pa >> (4 * s)) & 15u)) * kTabRow + 4 * warp];
                        const uint64_t *tb = &S.tab[(s * 16 + (uint32_t)((pb >> (4 * s)) & 15u)) * kTabRow + 4 * warp];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            or64(acc0[j], ta[j]);
                            or64(acc1[j], tb[j]);
                        }
                    }
                }
            } else {
                if (wmask && !timed_out) {
                    const uint64_t *q = &S.q[stage][(4 * warp) * 64];
#pragma unroll
                    for (int kk = 0; kk < 64; kk += 2) {
                        const uint32_t pa = kk < 32 ? pp.x : pp.y;  // row 2l
                        const uint32_t pb = kk < 32 ? pp.z : pp.w;  // row 2l+1
                        const int b = kk & 31;
                        const uint32_t ma0 = bitmask(pa, b), ma1 = bitmask(pa, b + 1);
                        const uint32_t mb0 = bitmask(pb, b), mb1 = bitmask(pb, b + 1);
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const uint4 qv = *reinterpret_cast<const uint4 *>(q + j * 64 + kk);
                            acc0[j].x |= (qv.x & ma0) | (qv.z & ma1);
                            acc0[j].y |= (qv.y & ma0) | (qv.w & ma1);
                            acc1[j].x |= (qv.x & mb0) | (qv.z & mb1);
                            acc1[j].y |= (qv.y & mb0) | (qv.w & mb1);
                        }
                    }
                }
            }
            // all threads are done with this stage (and the tables) before they
            // are refilled; a timeout anywhere in the CTA stops every later wait
            timed_out = __syncthreads_or(timed_out) != 0;
            stage ^= 1;
        }
        // ---- epilogue ----
        bool any_new = false;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t tj = tj0 + 4 * warp + j;
            uint32_t newcnt = 0;
            if (tj < T) {
#pragma unroll
                for (int rr = 0; rr < 2; ++rr) {
                    const uint2 a2 = rr ? acc1[j] : acc0[j];
                    const uint64_t a = ((uint64_t)a2.y << 32) | a2.x;
                    if (!a) continue;
                    ++outw;
                    const size_t off = tile_offset(T, ti, tj) + 2 * lane + rr;
                    unsigned long long *cw = reinterpret_cast<unsigned long long *>(C.bits + off);
                    const uint64_t seen = __ldcg(cw);
                    if (!(a & ~seen)) continue;
                    const uint64_t prev = atomicOr(cw, (unsigned long long)a);
                    const uint64_t nw = a & ~prev;
                    if (nw) {
                        ++neww;
                        newcnt += __popcll(nw);
                        if (D.bits) atomicOr(reinterpret_cast<unsigned long long *>(D.bits + off), (unsigned long long)nw);
                    }
                }
            }
            const uint32_t tile_new = __reduce_add_sync(kFull, newcnt);
            if (tile_new) {
                any_new = true;
                if (lane == 0) {
                    atomicAdd(C.nnz + (size_t)ti * T + tj, tile_new);
                    atomicOr(C.occ + (size_t)ti * C.ow + (tj >> 5), 1u << (tj & 31));
                    if (D.bits) {
                        atomicAdd(D.nnz + (size_t)ti * T + tj, tile_new);
                        atomicOr(D.occ + (size_t)ti * D.ow + (tj >> 5), 1u << (tj & 31));
                    }
                }
            }
        }
        if (any_new && lane == 0) {
            st->changed = 1u;
            if (qchanged) qchanged[pd.query] = 1u;
        }
        __syncthreads();  // S.item / k-list reuse
    }
    // per-CTA counters (warp-reduced) for statistics and the roofline report
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
    if (tid == 0 && staged) atomicAdd(&st->bytes_staged, staged);
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
                                 cudaStream_t s) {
    if (m4r)
        k_product_tiled<true><<<grid, kThreads, sizeof(TiledSmem<true>), s>>>(d_prods, d_slots, d_st, d_items, list_cap,
                                                                              d_qchanged);
    else
        k_product_tiled<false><<<grid, kThreads, sizeof(TiledSmem<false>), s>>>(d_prods, d_slots, d_st, d_items,
                                                                                list_cap, d_qchanged);
    return cudaGetLastError();
}

}  // namespace cfpq
