// Variant TC: exact Boolean product C |= P * Q on the 5th-generation tensor
// cores (tcgen05.mma kind::i8, 0/1 operands, int32 accumulators in TMEM,
// result bit = accumulator > 0).
//
// Operands travel as packed bits and are expanded on chip.  Per k-tile tk of
// a work item the copy warp stages the 4 P tiles (ti0..ti0+3, tk) and the Q
// block (tk, tj0..tj0+3) -- 4 KiB of bits, bulk copies completing on the
// stage's mbarrier -- into one of kPkStages packed stages.  Sixteen expander
// warps in two groups of eight (group g takes the k-tiles of parity g, so a
// warp has two k-tiles' time for each of its expansions) turn a packed stage
// into the MMA operands in one of kOpStages operand stages: warp w < 4 of a
// group writes P tile w as 0/1 bytes by rows (64 rows x 64 k)
// in the canonical no-swizzle K-major layout (8-row x 16-byte core matrices,
// K-adjacent core matrices 128 B apart, 8-row groups 512 B apart), warp
// w >= 4 writes Q tile w-4 by its rows (k) in the MN-major layout (16 output
// columns x 8 k-rows per 128-byte core matrix, column groups 128 B apart,
// 8-row k groups 2048 B apart), so neither operand is transposed; each
// nibble of bits becomes 4 bytes of 0/1 by one multiply and one mask.
// The warps then fence the writes for the async proxy and arrive on the
// operand stage's "full" barrier.  The MMA warp issues 4
// tcgen05.mma per k-tile (2 accumulators of M=128 x N=256, 2 K-halves of 32)
// and commits them to the operand stage's "empty" barrier, which the
// expanders wait on before reusing it; after the item's last k-tile a commit
// to the accumulator barrier releases the epilogue.  Global memory only ever
// supplies packed bits (512 B per 64x64 tile): the operands of a dense
// n = 8192 product are 16 MiB and stay in L2.
//
// Work item (item list 2) = (product, group of 4 output tile-rows, block of 4
// output tiles): a 256 x 256-bit output block over the whole inner dimension,
// accumulated in TMEM as two 128 x 256 int32 matrices (all 512 TMEM columns;
// one CTA per SM).  Epilogue (the 16 expander warps): tcgen05.ld 32x32b.x32
// (warp w reads accumulator (w/4)%2, TMEM lanes 32*(w%4).., output tiles
// 2*(w/8) and 2*(w/8)+1 of the block), threshold > 0, pack 64 columns into a
// word, then the atomic-OR epilogue of the word-level kernels (C, next delta
// D, occupancy, populations).
//
// Arithmetic: 256*256*64 MACs per k-tile; bound = the tensor pipe's dense int8
// rate.  Every wait is bounded; a wait that gives up raises the CTA's abort
// flag (which ends every other role's waits), the CTA then waits (bounded) for
// each bulk copy and MMA still in flight, frees TMEM and reports
// CFPQ_ERR_TIMEOUT.
#include "launch.h"

namespace cfpq {

namespace {

constexpr int kGroupWarps = 8;           // expanders of one k-tile: 4 P tiles, 4 Q tiles
constexpr int kExpWarps = 2 * kGroupWarps;  // two groups (k-tile parity), then the epilogue
constexpr int kCopyWarp = kExpWarps;     // lane 0 issues the bulk copies
constexpr int kMmaWarp = kExpWarps + 1;  // lane 0 issues the MMAs
constexpr int kThreads = 32 * (kExpWarps + 2);
constexpr int kMaxTiles = 2048;
constexpr uint32_t kTmemCols = 512;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kOperandBytes = 256 * 64;  // one operand, one stage: 256 rows x 64 bytes
constexpr uint32_t kPkStages = 8;             // packed k-tiles in flight (4 KiB each)
constexpr uint32_t kOpStages = 3;             // expanded operand stages (32 KiB each)

// Instruction descriptor, kind::i8: D = S32 (bits 4-5 = 2), A = B = U8 (0),
// A K-major (bit 15 = 0), B MN-major (bit 16 = 1), N = 256 (bits 17-22 =
// N/8), M = 128 (bits 24-28 = M/16).
constexpr uint32_t kIdesc = (2u << 4) | (1u << 16) | ((256u / 8) << 17) | ((128u / 16) << 24);
// B operand (MN-major, no swizzle): 16-column groups 128 B apart (SBO),
// 8-row k groups 2048 B apart (LBO).
constexpr uint32_t kBSbo = 128, kBLbo = 2048;

struct __align__(1024) TcSmem {
    uint8_t a[kOpStages][kOperandBytes];  // P rows of 4 tile-rows, 4 x 4 KiB per stage
    uint8_t b[kOpStages][kOperandBytes];  // Q^T of 4 tiles, 4 x 4 KiB per stage
    uint64_t pk[kPkStages][8][64];        // packed: P tiles 0..3, then Q tiles 0..3
    uint64_t pk_full[kPkStages], pk_empty[kPkStages];
    uint64_t op_full[kOpStages], op_empty[kOpStages];
    uint64_t acc_full;
    uint32_t tmem_base;
    uint32_t item;
    uint32_t abort;    // a role's wait gave up: every other wait ends too
    uint32_t pk_seen[2];  // group g: 1 + the last packed stage its warp 0 saw land (sequence number)
    uint16_t cand[kMaxTiles];
    uint16_t cmask[kMaxTiles];
    uint16_t ktile[kMaxTiles];
    uint32_t rball[kMaxTiles / 32], roff[kMaxTiles / 32];
    uint32_t nc, nk;
};

__device__ __forceinline__ DevMat resolve_operand(const MatSlot &s, uint8_t use_delta, uint32_t iter) {
    if (!use_delta || iter == 0) return s.cur;
    return s.dlt[iter & 1];
}

// 64-bit shared-memory matrix descriptor, no swizzle, sm_100 version bit 46.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ULL << 46);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 32 consecutive 32-bit TMEM columns -> 32 registers.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16 bits of `bits` starting at bit 16*c -> 16 bytes of 0/1 (bit i -> byte
// i): each nibble times 0x00204081 puts its bits at 0, 8, 16, 24 without
// overlapping sums; the mask keeps them.
__device__ __forceinline__ uint4 expand16(uint64_t bits, int c) {
    const uint32_t x = (uint32_t)(bits >> (16 * c));
    uint4 v;
    v.x = ((x & 15u) * 0x00204081u) & 0x01010101u;
    v.y = (((x >> 4) & 15u) * 0x00204081u) & 0x01010101u;
    v.z = (((x >> 8) & 15u) * 0x00204081u) & 0x01010101u;
    v.w = (((x >> 12) & 15u) * 0x00204081u) & 0x01010101u;
    return v;
}

// A operand (K-major), operand row r (0..63) of a 4 KiB block: its 64 k-bytes
// as 4 16-byte chunks at ((r/8)*4 + kg)*128 + (r%8)*16.
__device__ __forceinline__ void store_row_k(uint8_t *block, uint32_t r, uint64_t bits) {
    uint8_t *base = block + (r >> 3) * 512 + (r & 7) * 16;
#pragma unroll
    for (int kg = 0; kg < 4; ++kg) *reinterpret_cast<uint4 *>(base + kg * 128) = expand16(bits, kg);
}

// B operand (MN-major), k-row k (0..63) of Q tile j (output columns
// 64j .. 64j+63): 16-column chunk c of the row at
// (4j + c)*kBSbo + (k/8)*kBLbo + (k%8)*16.
__device__ __forceinline__ void store_row_mn(uint8_t *b, uint32_t j, uint32_t k, uint64_t bits) {
    uint8_t *base = b + (k >> 3) * kBLbo + (k & 7) * 16 + 4 * j * kBSbo;
#pragma unroll
    for (int c = 0; c < 4; ++c) *reinterpret_cast<uint4 *>(base + c * kBSbo) = expand16(bits, c);
}

// Bounded wait that also ends when another role raised the abort flag.
__device__ __forceinline__ bool wait_or_abort(uint64_t *bar, uint32_t parity, const volatile uint32_t *abort) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 63u && *abort) return false;
    }
    return false;
}

__global__ void __launch_bounds__(kThreads, 1)
    k_product_tc(const ProdDesc *__restrict__ prods, const MatSlot *__restrict__ slots, IterState *st,
                 const uint64_t *__restrict__ items_all, size_t list_cap, uint32_t *qchanged, BufCounters *cnts) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TcSmem &S = *reinterpret_cast<TcSmem *>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t *items = items_all + 2 * list_cap;
    volatile uint32_t *abort = &S.abort;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&S.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (uint32_t s = 0; s < kPkStages; ++s) {
            mbar_init(&S.pk_full[s], 1);
            mbar_init(&S.pk_empty[s], kGroupWarps);
        }
        for (uint32_t s = 0; s < kOpStages; ++s) {
            mbar_init(&S.op_full[s], kGroupWarps);
            mbar_init(&S.op_empty[s], 1);
        }
        mbar_init(&S.acc_full, 1);
        S.abort = 0;
        S.pk_seen[0] = S.pk_seen[1] = 0;
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem_base;
    const uint32_t iter = st->iter;
    const uint32_t nitems = st->item_count[2];
    unsigned long long triples = 0, outw = 0, neww = 0;
    // k-tile sequence numbers across the CTA's items: stage = seq % stages,
    // use = seq / stages; a "full" barrier is waited with parity use & 1, an
    // "empty" one with (use & 1) ^ 1 (a fresh barrier counts its previous
    // phase as complete, so the first use of every stage passes)
    uint32_t seq = 0, items_done = 0;
    uint32_t pk_issued = 0;      // copy warp: packed stages issued (sequence count)
    uint32_t mma_committed = 0;  // MMA warp: k-tiles committed (sequence count)

    for (;;) {
        if (tid == 0) S.item = atomicAdd(&st->item_next[2], 1u);
        __syncthreads();
        const uint32_t idx = S.item;
        if (idx >= nitems || *abort) break;
        const uint64_t it = items[idx];
        const ProdDesc pd = prods[item_prod(it)];
        const uint32_t tig = item_ti(it), tjb = item_tjb(it), klo = item_klo(it), khi = item_khi(it);
        const DevMat P = resolve_operand(slots[pd.pslot], pd.p_delta, iter);
        const DevMat Q = resolve_operand(slots[pd.qslot], pd.q_delta, iter);
        const DevMat C = slots[pd.head].cur;
        const DevMat D = slots[pd.head].dlt[(iter & 1) ^ 1];
        const uint32_t T = pd.T, ow = P.ow;
        const uint32_t ti0 = tig * 4, tj0 = tjb * 4;
        const uint32_t qword = tj0 >> 5, qshift = tj0 & 31;
        const uint32_t np = min(4u, T - ti0), nq = min(4u, T - tj0);  // existing P tile-rows / Q tiles

        // ---- k-list: tk with an occupied P tile in the 4 tile-rows and a
        // non-empty Q block, increasing tk, within the item's range ----
        if (warp == 0) {
            uint32_t nc = 0;
            for (uint32_t base = 0; base < ow; base += 32) {
                uint32_t bits = 0;
                if (base + lane < ow) {
                    for (uint32_t g = 0; g < np; ++g) bits |= P.occ[(size_t)(ti0 + g) * ow + base + lane];
                    bits &= range_word_mask(base + lane, klo, khi);
                }
                const uint32_t cnt = __popc(bits);
                uint32_t pre = cnt;
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
        const uint32_t nc = S.nc, rounds = (nc + 31) / 32;
        for (uint32_t r = warp; r < rounds; r += kThreads / 32) {
            const uint32_t c = r * 32 + lane;
            uint32_t mask = 0;
            if (c < nc) mask = (Q.occ[(size_t)S.cand[c] * ow + qword] >> qshift) & 0xFu;
            const unsigned ball = __ballot_sync(kFull, mask != 0);
            if (c < nc) S.cmask[c] = (uint16_t)mask;
            if (lane == 0) S.rball[r] = ball;
        }
        __syncthreads();
        if (warp == 0) {
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
            if (!S.cmask[c]) continue;
            const uint32_t rank = S.roff[c >> 5] + __popc(S.rball[c >> 5] & ((1u << (c & 31)) - 1));
            S.ktile[rank] = S.cand[c];  // keeps increasing tk order
            triples += 16;
        }
        if (tid == 0) S.nk = rounds ? S.roff[rounds - 1] + __popc(S.rball[rounds - 1]) : 0u;
        __syncthreads();
        const uint32_t nk = S.nk;

        // ---- pipeline over the item's k-tiles ----
        if (warp == kCopyWarp) {
            if (lane == 0) {
                for (uint32_t e = 0; e < nk; ++e) {
                    const uint32_t q = seq + e, s = q % kPkStages, use = q / kPkStages;
                    if (!wait_or_abort(&S.pk_empty[s], (use & 1u) ^ 1u, abort)) {
                        *abort = 1;
                        break;
                    }
                    const uint32_t tk = S.ktile[e];
                    mbar_arrive_expect_tx(&S.pk_full[s], (np + nq) * 512u);
                    for (uint32_t g = 0; g < np; ++g)
                        bulk_g2s(S.pk[s][g], P.bits + tile_offset(T, ti0 + g, tk), 512u, &S.pk_full[s]);
                    bulk_g2s(S.pk[s][4], Q.bits + tile_offset(T, tk, tj0), nq * 512u, &S.pk_full[s]);
                    ++pk_issued;
                }
            }
        } else if (warp == kMmaWarp) {
            if (lane == 0) {
                for (uint32_t e = 0; e < nk; ++e) {
                    const uint32_t q = seq + e, o = q % kOpStages, use = q / kOpStages;
                    if (!wait_or_abort(&S.op_full[o], use & 1u, abort)) {
                        *abort = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t abase = smem_addr(S.a[o]), bbase = smem_addr(S.b[o]);
#pragma unroll
                    for (uint32_t h = 0; h < 2; ++h) {      // accumulator h: operand rows 128h .. 128h+127
#pragma unroll
                        for (uint32_t kh = 0; kh < 2; ++kh) {  // K halves of 32 bytes
                            const uint64_t ad = smem_desc(abase + h * 8192 + kh * 256, 128, 512);
                            const uint64_t bd = smem_desc(bbase + kh * 4 * kBLbo, kBLbo, kBSbo);
                            mma_i8(tmem + h * 256, ad, bd, (e > 0 || kh > 0) ? 1u : 0u);
                        }
                    }
                    mma_commit(&S.op_empty[o]);
                    ++mma_committed;
                }
                if (nk && !*abort) mma_commit(&S.acc_full);  // completes after every MMA of the item
            }
        } else {
            // expander warp w of group gp (k-tiles e with e % 2 == gp): P tile
            // w (w < 4) or Q tile w - 4 (by rows, no transpose)
            const uint32_t gp = warp / kGroupWarps, wr = warp % kGroupWarps;
            const bool is_p = wr < 4;
            const uint32_t g = is_p ? wr : wr - 4;
            const bool present = g < (is_p ? np : nq);
            for (uint32_t e = gp; e < nk; e += 2) {
                const uint32_t q = seq + e, s = q % kPkStages, o = q % kOpStages;
                // waits are warp-uniform: one lane giving up ends the whole warp's loop
                if (!__all_sync(kFull, wait_or_abort(&S.pk_full[s], (q / kPkStages) & 1u, abort))) {
                    if (lane == 0) *abort = 1;
                    break;
                }
                if (wr == 0 && lane == 0) S.pk_seen[q & 1u] = q + 1;
                uint64_t lo = 0, hi = 0;
                if (present) {
                    lo = S.pk[s][is_p ? g : 4 + g][lane];
                    hi = S.pk[s][is_p ? g : 4 + g][lane + 32];
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&S.pk_empty[s]);  // the packed stage may be refilled
                if (!__all_sync(kFull, wait_or_abort(&S.op_empty[o], ((q / kOpStages) & 1u) ^ 1u, abort))) {
                    if (lane == 0) *abort = 1;
                    break;
                }
                if (present) {
                    if (is_p) {
                        store_row_k(S.a[o] + g * 4096, lane, lo);
                        store_row_k(S.a[o] + g * 4096, lane + 32, hi);
                    } else {
                        store_row_mn(S.b[o], g, lane, lo);
                        store_row_mn(S.b[o], g, lane + 32, hi);
                    }
                }
                fence_proxy_async_smem();  // generic-proxy writes before the tensor core reads them
                __syncwarp();
                if (lane == 0) mbar_arrive(&S.op_full[o]);
            }
        }
        seq += nk;
        __syncthreads();
        if (*abort) break;

        // ---- epilogue (expander warps) ----
        bool any_new = false;
        if (nk > 0 && warp < kExpWarps) {
            const bool acc_ok = __all_sync(kFull, wait_or_abort(&S.acc_full, items_done & 1u, abort));
            if (!acc_ok && lane == 0) *abort = 1;
            tc_fence_after();
            if (acc_ok) {
                uint32_t tile_new[2] = {0, 0};
                const uint32_t h = (warp >> 2) & 1u, qq = warp & 3, half = warp >> 3;
                const uint32_t m = 128 * h + 32 * qq + lane;  // output row within the 256-row block
                const uint32_t ti = ti0 + (m >> 6), r = m & 63;
#pragma unroll 1
                for (uint32_t jh = 0; jh < 2; ++jh) {
                    const uint32_t jt = 2 * half + jh;
                    uint32_t a32[2];
#pragma unroll
                    for (int x = 0; x < 2; ++x) {
                        uint32_t v[32];
                        tmem_ld32(tmem + ((32 * qq) << 16) + h * 256 + jt * 64 + x * 32, v);
                        uint32_t w = 0;
#pragma unroll
                        for (int c = 0; c < 32; ++c) w |= (uint32_t)(v[c] != 0) << c;
                        a32[x] = w;
                    }
                    const uint64_t a = (uint64_t)a32[0] | ((uint64_t)a32[1] << 32);
                    const uint32_t tj = tj0 + jt;
                    uint32_t newcnt = 0;
                    if (a && ti < T && tj < T) {
                        ++outw;
                        const size_t off = tile_offset(T, ti, tj) + r;
                        unsigned long long *cw = reinterpret_cast<unsigned long long *>(C.bits + off);
                        const uint64_t seen = __ldcg(cw);
                        if (a & ~seen) {
                            const uint64_t prev = atomicOr(cw, (unsigned long long)a);
                            const uint64_t nw = a & ~prev;
                            if (nw) {
                                ++neww;
                                newcnt = __popcll(nw);
                                if (D.bits)
                                    atomicOr(reinterpret_cast<unsigned long long *>(D.bits + off),
                                             (unsigned long long)nw);
                            }
                        }
                    }
                    tile_new[jh] = __reduce_add_sync(kFull, newcnt);  // the warp's 32 rows share (ti, tj)
                }
                any_new = (tile_new[0] | tile_new[1]) != 0;
                if (any_new && ti < T) {  // lane j: tile tj0 + 2 * half + j (populations, occupancy, counters)
                    const uint32_t mine = lane == 0 ? tile_new[0] : lane == 1 ? tile_new[1] : 0u;
                    tiles_gain(C, ti, tj0 + 2 * half, mine, cnts ? cnts + 3 * pd.head : nullptr);
                    if (D.bits)
                        tiles_gain(D, ti, tj0 + 2 * half, mine,
                                   cnts ? cnts + 3 * pd.head + 1 + ((iter & 1) ^ 1) : nullptr);
                }
            }
        }
        if (nk > 0) ++items_done;
        if (any_new && lane == 0) {
            st->changed = 1u;
            if (qchanged) qchanged[pd.query] = 1u;
        }
        tc_fence_before();
        __syncthreads();  // TMEM reads done before the next item's first MMA overwrites it
        tc_fence_after();
        if (*abort) break;
    }

    // ---- exit: after a wait gave up, wait (bounded) for every bulk copy and
    // MMA still in flight before TMEM is freed and the CTA ends ----
    __syncthreads();
    const bool aborted = *abort != 0;
    if (aborted) {
        if (warp == kCopyWarp && lane == 0) {
            // copies of the stages not seen by their group may still be
            // landing (a stage is refilled only after its group saw it)
            const uint32_t seen0 = S.pk_seen[0], seen1 = S.pk_seen[1];
            for (uint32_t q = min(seen0, seen1); q < pk_issued; ++q)
                if (q >= ((q & 1u) ? seen1 : seen0)) mbar_wait_bounded(&S.pk_full[q % kPkStages], (q / kPkStages) & 1u);
        }
        if (warp == kMmaWarp && lane == 0 && mma_committed) {
            // the last commit completes after every MMA issued before it
            const uint32_t q = mma_committed - 1;
            mbar_wait_bounded(&S.op_empty[q % kOpStages], (q / kOpStages) & 1u);
        }
    }
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
    if (aborted && tid == 0) atomicExch(&st->error, 5u);
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

}  // namespace

int product_tc_blocks_per_sm() {
    cudaFuncSetAttribute(k_product_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem));
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_product_tc, kThreads, sizeof(TcSmem));
    return nb;
}

cudaError_t launch_product_tc(const ProdDesc *d_prods, const MatSlot *d_slots, IterState *d_st,
                              const uint64_t *d_items, size_t list_cap, uint32_t *d_qchanged, int grid,
                              BufCounters *cnts, cudaStream_t s) {
    k_product_tc<<<grid, kThreads, sizeof(TcSmem), s>>>(d_prods, d_slots, d_st, d_items, list_cap, d_qchanged, cnts);
    return cudaGetLastError();
}

}  // namespace cfpq
