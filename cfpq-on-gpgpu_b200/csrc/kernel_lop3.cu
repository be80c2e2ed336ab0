// Variant LOP3: tiled word-level Boolean product C |= P * Q over the work items
// of one closure iteration (or one add_mul).
//
// Work item = (product, output tile-row ti, block of kBJ output tiles).  A CTA
// of 4 warps owns the 64 x (64*kBJ) output block in registers: warp w owns
// tiles 4w..4w+3 of the block, lane l owns rows 2l and 2l+1, so every thread
// keeps 2 rows x 4 tiles x 64 bits = 16 uint32 accumulators.
//
// Inner dimension: the CTA walks the k-tiles tk whose P tile (ti, tk) is
// occupied and whose Q tiles (tk, block) are not all empty (the list is built
// once per item by warp 0).  For each tk one elected thread stages the P tile
// (512 B) and the kBJ Q tiles (kBJ*512 B, one contiguous range in the tiled
// layout) into shared memory with bulk copies (cp.async.bulk, the TMA engine)
// completing on an mbarrier; two stages double-buffer the staging.  A warp
// whose 4 Q tiles are all empty skips the k-tile.
//
// Inner loop per row and inner index k: mask = -(P[row] bit k) (2 ALU ops),
// then acc |= mask & Q[k] for 8 uint32 words (one LOP3 each).  Q rows k, k+1 of
// a tile come in one 16-byte shared load that every lane of the warp reads at
// the same address (broadcast).
//
// Epilogue: for each non-zero accumulator word, new = acc & ~old via a 64-bit
// atomicOr (several products of one iteration may write the same head); new
// bits also go to the head's next-delta matrix D, and the occupancy bits of
// the touched tiles of C and D are set.  Concurrent reads of matrices that
// other CTAs are OR-ing into are safe: every bit only ever goes 0 -> 1, so a
// read sees a subset of the final and a superset of the iteration-start value.
#include "launch.h"

namespace cfpq {

namespace {

constexpr int kBJ = 16;          // output tiles per work item (1024 columns)
constexpr int kThreads = 128;    // 4 warps
constexpr int kMaxTiles = 2048;  // k-list capacity (n <= 131072)
constexpr unsigned kFull = 0xffffffffu;

struct __align__(128) Lop3Smem {
    uint64_t q[2][kBJ * 64];     // 2 x 8 KiB
    uint64_t p[2][64];           // 2 x 512 B
    uint64_t bar[2];
    uint16_t ktile[kMaxTiles];   // k-list: tile index
    uint16_t kmask[kMaxTiles];   // k-list: occupancy of the kBJ Q tiles
    uint32_t nk;
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

__global__ void __launch_bounds__(kThreads, 4)
    k_product_lop3(const ProdDesc *__restrict__ prods, const MatSlot *__restrict__ slots, IterState *st,
                   const uint64_t *__restrict__ items, uint32_t *qchanged) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Lop3Smem &S = *reinterpret_cast<Lop3Smem *>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;  // bit s = next parity to wait for on stage s
    const uint32_t iter = st->iter;
    const uint32_t nitems = st->item_count;
    unsigned long long triples = 0;
    bool timed_out = false;

    for (;;) {
        if (tid == 0) S.item = atomicAdd(&st->item_next, 1u);
        __syncthreads();
        const uint32_t idx = S.item;
        if (idx >= nitems) break;
        const uint64_t it = items[idx];
        const ProdDesc pd = prods[item_prod(it)];
        const uint32_t ti = item_ti(it), tjb = item_tjb(it);
        const DevMat P = resolve_operand(slots[pd.pslot], pd.p_delta, iter);
        const DevMat Q = resolve_operand(slots[pd.qslot], pd.q_delta, iter);
        const DevMat C = slots[pd.head].cur;
        const DevMat D = slots[pd.head].dlt[(iter & 1) ^ 1];
        const uint32_t T = pd.T, ow = P.ow;
        const uint32_t tj0 = tjb * kBJ;
        const uint32_t nblk = min((uint32_t)kBJ, T - tj0);
        const uint32_t qword = tj0 >> 5, qshift = tj0 & 31;

        // ---- k-list: tk with occP(ti,tk) and a non-empty Q block (warp 0) ----
        if (warp == 0) {
            uint32_t nk = 0;
            const uint32_t *prow = P.occ + (size_t)ti * ow;
            for (uint32_t base = 0; base < ow; base += 32) {
                uint32_t bits = (base + lane < ow) ? prow[base + lane] : 0u;
                while (__any_sync(kFull, bits != 0)) {
                    const bool has = bits != 0;
                    uint32_t tk = 0, mask = 0;
                    if (has) {
                        tk = (base + lane) * 32 + (__ffs(bits) - 1);
                        bits &= bits - 1;
                        mask = (Q.occ[(size_t)tk * ow + qword] >> qshift) & ((1u << kBJ) - 1);
                    }
                    const unsigned ball = __ballot_sync(kFull, mask != 0);
                    if (mask) {
                        const uint32_t pos = nk + __popc(ball & ((1u << lane) - 1));
                        S.ktile[pos] = (uint16_t)tk;
                        S.kmask[pos] = (uint16_t)mask;
                    }
                    nk += __popc(ball);
                }
            }
            if (lane == 0) S.nk = nk;
        }
        __syncthreads();
        const uint32_t nk = S.nk;

        uint2 acc0[4], acc1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) acc0[j] = acc1[j] = make_uint2(0, 0);

        auto issue = [&](uint32_t e, uint32_t stage) {
            const uint32_t tk = S.ktile[e];
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&S.bar[stage], 512u + nblk * 512u);
            bulk_g2s(S.p[stage], P.bits + tile_offset(T, ti, tk), 512u, &S.bar[stage]);
            bulk_g2s(S.q[stage], Q.bits + tile_offset(T, tk, tj0), nblk * 512u, &S.bar[stage]);
        };

        if (tid == 0 && nk > 0) issue(0, 0);
        uint32_t stage = 0;
        for (uint32_t e = 0; e < nk; ++e) {
            if (tid == 0 && e + 1 < nk) issue(e + 1, stage ^ 1);
            if (!mbar_wait_bounded(&S.bar[stage], (phase >> stage) & 1u)) timed_out = true;
            phase ^= 1u << stage;
            const uint32_t wmask = ((uint32_t)S.kmask[e] >> (4 * warp)) & 0xFu;
            if (wmask && !timed_out) {
                triples += (lane == 0) ? __popc(wmask) : 0;
                const uint4 pp = *reinterpret_cast<const uint4 *>(&S.p[stage][2 * lane]);
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
            __syncthreads();
            stage ^= 1;
        }

        // ---- epilogue ----
        bool any_new = false;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t tj = tj0 + 4 * warp + j;
            bool newbits = false;
            if (tj < T) {
#pragma unroll
                for (int rr = 0; rr < 2; ++rr) {
                    const uint2 a2 = rr ? acc1[j] : acc0[j];
                    const uint64_t a = ((uint64_t)a2.y << 32) | a2.x;
                    if (!a) continue;
                    const size_t off = tile_offset(T, ti, tj) + 2 * lane + rr;
                    unsigned long long *cw = reinterpret_cast<unsigned long long *>(C.bits + off);
                    const uint64_t seen = __ldcg(reinterpret_cast<const unsigned long long *>(cw));
                    if (!(a & ~seen)) continue;
                    const uint64_t prev = atomicOr(cw, (unsigned long long)a);
                    const uint64_t nw = a & ~prev;
                    if (nw) {
                        newbits = true;
                        if (D.bits) atomicOr(reinterpret_cast<unsigned long long *>(D.bits + off), (unsigned long long)nw);
                    }
                }
            }
            if (__any_sync(kFull, newbits)) {
                any_new = true;
                if (lane == 0) {
                    atomicOr(C.occ + (size_t)ti * C.ow + (tj >> 5), 1u << (tj & 31));
                    if (D.bits) atomicOr(D.occ + (size_t)ti * D.ow + (tj >> 5), 1u << (tj & 31));
                }
            }
        }
        if (any_new && lane == 0) {
            st->changed = 1u;
            if (qchanged) qchanged[pd.query] = 1u;
        }
        __syncthreads();  // S.item / k-list reuse
    }
    if (triples) atomicAdd(&st->tile_triples, triples);
    if (timed_out && tid == 0) atomicExch(&st->error, 5u);
}

}  // namespace

int product_lop3_tiles_per_block() { return kBJ; }
int product_lop3_max_tiles() { return kMaxTiles; }
// Called once per context (before any stream capture): sets the kernel's
// shared-memory attribute and returns the resident CTAs per SM.
int product_lop3_blocks_per_sm() {
    cudaFuncSetAttribute(k_product_lop3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Lop3Smem));
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_product_lop3, kThreads, sizeof(Lop3Smem));
    return nb > 0 ? nb : 1;
}

cudaError_t launch_product_lop3(const ProdDesc *d_prods, const MatSlot *d_slots, IterState *d_st,
                                const uint64_t *d_items, uint32_t *d_qchanged, int grid, cudaStream_t s) {
    k_product_lop3<<<grid, kThreads, sizeof(Lop3Smem), s>>>(d_prods, d_slots, d_st, d_items, d_qchanged);
    return cudaGetLastError();
}

}  // namespace cfpq
