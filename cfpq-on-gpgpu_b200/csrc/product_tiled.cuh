// Word-level tiled product: shared-memory layout and the processing of one
// work item, used by the product kernels (kernel_lop3.cu) and by the
// persistent closure kernel (kernel_persistent.cu).  The algorithm is
// described in kernel_lop3.cu.
#pragma once

#include "common.cuh"

namespace cfpq {
namespace tiled {


constexpr int kBJ = 16;              // output tiles per work item (1024 columns)
constexpr uint32_t kStages = 4;      // staged k-tiles in flight per CTA (product kernels)
constexpr uint32_t kLaneBits = 4;    // sparse loop: bits per row a lane walks before the warp helps
constexpr int kThreads = 128;        // 4 warps (product kernels; the persistent kernel runs 8)
constexpr int kMaxTiles = 2048;      // k-list capacity (n <= 131072)
constexpr uint32_t kSparseMax = 96;  // P-tile population up to which the sparse loop runs
constexpr int kTabRow = 17;          // padded table row (uint64 words): 16 keys, or kBJ tiles
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kGateSpinLimit = 1u << 24;  // ~1 s of polling
constexpr uint32_t kShortRange = 64;            // k ranges up to this length build the k-list in one round trip

template <bool kM4R, uint32_t kS = kStages>
struct __align__(128) TiledSmem {
    static constexpr uint32_t kNumStages = kS;
    uint64_t q[kS][kBJ * 64];  // kS x 8 KiB
    uint64_t p[kS][64];        // kS x 512 B
    // M4R tables, 34 KiB: [tile][slab][key] when each warp builds its own
    // tiles' tables (8 warps), [slab][key][tile] when the CTA builds them all
    uint64_t tab[kM4R ? kBJ * 16 * kTabRow : 1];
    uint64_t bar[kS];
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

// Position of the n-th (0-based) set bit of x (x has more than n set bits).
__device__ __forceinline__ uint32_t nth_bit(uint32_t x, uint32_t n) {
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

__device__ __forceinline__ void or64(uint2 &a, uint64_t v) {
    a.x |= (uint32_t)v;
    a.y |= (uint32_t)(v >> 32);
}

// Per-CTA statistics of the product kernels (reduced at kernel exit).
struct ItemCounters {
    unsigned long long triples = 0, staged = 0, outw = 0, neww = 0;
};

// Process work item `it` (all kW warps of the CTA; warp w owns output tiles
// kTPW*w .. kTPW*w + kTPW-1 of the block, lane l rows 2l and 2l+1).  `phase`
// is the CTA's mbarrier parity state (bit s = next parity of stage s),
// `timed_out` is set (CTA-uniformly) when a bounded wait gave up; new bits
// set *changed and qchanged[query].  gate and *gate non-null: the results
// are merged only once **gate reaches gate_target (bounded wait; on timeout
// the item merges nothing), after which *gate is cleared so that the CTA's
// later items skip the check.  direct_merge: every non-zero result word goes
// straight to its atomic OR (one round trip less per item; for latency-bound
// closures), else only words with bits C does not hold yet.  stamps non-null
// (thread 0): %globaltimer after the k-list, after the first staged k-tile
// arrived, after the last k-tile and after the gate.  Ends with the CTA
// synchronised.
template <bool kM4R, int kW, class Smem>
__device__ __forceinline__ void process_item(Smem &S, uint64_t it, const ProdDesc *__restrict__ prods,
                                             const MatSlot *__restrict__ slots, uint32_t iter, uint32_t *changed,
                                             uint32_t *qchanged, uint32_t &phase, bool &timed_out,
                                             ItemCounters &ctr, BufCounters *cnts,
                                             const uint32_t **gate = nullptr, uint32_t gate_target = 0,
                                             bool direct_merge = false, unsigned long long *stamps = nullptr) {
    static_assert(kBJ % kW == 0 && kBJ / kW <= 4, "whole tiles per warp, at most 4");
    static_assert(kShortRange <= 32u * kW, "one k-tile per thread in the short k-list path");
    constexpr int kTPW = kBJ / kW;             // output tiles per warp
    constexpr uint32_t kNT = 32u * kW;         // threads
    constexpr uint32_t kWMask = (1u << kTPW) - 1;
    constexpr uint32_t kSt = Smem::kNumStages;       // staged k-tiles in flight
    static_assert(kSt <= 32, "one mbarrier parity bit per stage");
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long &triples = ctr.triples, &staged = ctr.staged, &outw = ctr.outw, &neww = ctr.neww;
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

    // ---- k-list: the item's k-tiles (occupied P tile and non-empty Q
    // block), increasing, with their Q block masks and P density ----
    if (khi - klo <= kShortRange) {
        // short range: thread c loads the P occupancy bit, the Q block
        // occupancy and the P tile population of k-tile klo + c together
        // (one round trip instead of two dependent ones; the loads of
        // unoccupied P tiles are wasted, hence only for short ranges), then a
        // block-wide ballot compaction
        const uint32_t tk = klo + tid;
        uint32_t mask = 0;
        bool dense = false;
        if (tk < khi) {
            const uint32_t pw = P.occ[(size_t)ti * ow + (tk >> 5)];
            const uint32_t qw = Q.occ[(size_t)tk * ow + qword];
            const uint32_t pn = P.nnz[(size_t)ti * T + tk];
            if ((pw >> (tk & 31)) & 1u) {
                mask = (qw >> qshift) & ((1u << kBJ) - 1);
                dense = pn > kSparseMax;
            }
        }
        const unsigned ball = __ballot_sync(kFull, mask != 0);
        if (lane == 0) S.rball[warp] = ball;
        __syncthreads();
        uint32_t rank = __popc(ball & ((1u << lane) - 1)), total = 0;
#pragma unroll
        for (int w = 0; w < kW; ++w) {
            const uint32_t c = __popc(S.rball[w]);
            if ((uint32_t)w < warp) rank += c;
            total += c;
        }
        if (mask) {
            triples += __popc(mask);
            S.ktile[rank] = (uint16_t)(tk | (dense ? 0x8000u : 0u));
            S.kmask[rank] = (uint16_t)mask;
        }
        if (tid == 0) S.nk = total;
        __syncthreads();
    } else {
    // long range: warp 0 compacts the occupied P tiles of row ti in
    // [klo, khi) into a candidate list, then all threads classify the
    // candidates in parallel
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
    for (uint32_t r = warp; r < rounds; r += kW) {
        const uint32_t c = r * 32 + lane;
        uint32_t mask = 0;
        bool dense = false;
        if (c < nc) {
            const uint32_t tk = S.cand[c];
            mask = (Q.occ[(size_t)tk * ow + qword] >> qshift) & ((1u << kBJ) - 1);
            dense = P.nnz[(size_t)ti * T + tk] > kSparseMax;  // issued together with the occupancy load
        }
        const unsigned ball = __ballot_sync(kFull, mask != 0);
        if (c < nc) {
            S.cmask[c] = (uint16_t)mask;
            if (dense) S.cand[c] |= 0x8000u;
        }
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
    for (uint32_t c = tid; c < nc; c += kNT) {
        const uint32_t mask = S.cmask[c];
        if (!mask) continue;
        const uint32_t rank = S.roff[c >> 5] + __popc(S.rball[c >> 5] & ((1u << (c & 31)) - 1));
        triples += __popc(mask);
        S.ktile[rank] = S.cand[c];  // tile index, bit 15: dense P tile
        S.kmask[rank] = (uint16_t)mask;
    }
    if (tid == 0) S.nk = rounds ? S.roff[rounds - 1] + __popc(S.rball[rounds - 1]) : 0u;
    __syncthreads();
    }
    const uint32_t nk = S.nk;
    if (stamps && tid == 0) stamps[0] = stamps[1] = globaltimer_ns();
    // thread 0 reads the gate early (with the first staged k-tile) so that
    // the read is usually back, and open, by the time the results are ready
    uint32_t gate_seen = 0;

    uint2 acc0[kTPW], acc1[kTPW];
#pragma unroll
    for (int j = 0; j < kTPW; ++j) acc0[j] = acc1[j] = make_uint2(0, 0);

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
    // k-tile e goes to stage e % kSt; the first kSt are issued up
    // front, a stage is refilled (k-tile e + kSt) once every thread is
    // done with it
    if (tid == 0)
        for (uint32_t e = 0; e < nk && e < kSt; ++e) staged += issue(e, e);
    for (uint32_t e = 0; e < nk; ++e) {
        const uint32_t stage = e % kSt;
        if (!timed_out && !mbar_wait_bounded(&S.bar[stage], (phase >> stage) & 1u)) timed_out = true;
        phase ^= 1u << stage;
        if (tid == 0 && e == 0) {
            if (gate && *gate) gate_seen = ld_acquire_u32(*gate);
            if (stamps) stamps[1] = globaltimer_ns();
        }
        const uint32_t wmask = ((uint32_t)S.kmask[e] >> (kTPW * warp)) & kWMask;
        const uint4 pp = *reinterpret_cast<const uint4 *>(&S.p[stage][2 * lane]);
        const bool dense = (S.ktile[e] & 0x8000u) != 0;
        if (!dense) {
            // sparse P tile, only the occupied Q tiles staged.  Each lane
            // first walks up to kLaneBits set bits of its rows 2l and 2l+1;
            // the bits left (rows of hub vertices) are then handled one row
            // at a time by the whole warp: lane i takes the i-th remaining
            // bit, and the partial ORs meet in a warp OR-reduction.
            if (wmask && !timed_out) {
                const uint64_t *q = &S.q[stage][(kTPW * warp) * 64];
                uint64_t xa = ((uint64_t)pp.y << 32) | pp.x;
                uint64_t xb = ((uint64_t)pp.w << 32) | pp.z;
#pragma unroll 1
                for (uint32_t it = 0; it < kLaneBits && (xa | xb); ++it) {
                    if (xa) {
                        const int k = __ffsll((long long)xa) - 1;
                        xa &= xa - 1;
#pragma unroll
                        for (int j = 0; j < kTPW; ++j)
                            if ((wmask >> j) & 1u) or64(acc0[j], q[j * 64 + k]);
                    }
                    if (xb) {
                        const int k = __ffsll((long long)xb) - 1;
                        xb &= xb - 1;
#pragma unroll
                        for (int j = 0; j < kTPW; ++j)
                            if ((wmask >> j) & 1u) or64(acc1[j], q[j * 64 + k]);
                    }
                }
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    uint64_t &xr = half ? xb : xa;
                    unsigned left = __ballot_sync(kFull, xr != 0);
                    while (left) {
                        const int src = __ffs(left) - 1;
                        left &= left - 1;
                        const uint64_t x = __shfl_sync(kFull, xr, src);
                        const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32), nlo = __popc(lo);
                        const uint32_t cnt = nlo + __popc(hi);
                        uint64_t o[kTPW];
#pragma unroll
                        for (int j = 0; j < kTPW; ++j) o[j] = 0;
                        for (uint32_t b = lane; b < cnt; b += 32) {
                            const uint32_t k = b < nlo ? nth_bit(lo, b) : 32 + nth_bit(hi, b - nlo);
#pragma unroll
                            for (int j = 0; j < kTPW; ++j)
                                if ((wmask >> j) & 1u) o[j] |= q[j * 64 + k];
                        }
#pragma unroll
                        for (int j = 0; j < kTPW; ++j) {
                            if (!((wmask >> j) & 1u)) continue;
#pragma unroll
                            for (int d = 16; d > 0; d >>= 1) o[j] |= __shfl_xor_sync(kFull, o[j], d);
                        }
                        if ((int)lane == src) {
#pragma unroll
                            for (int j = 0; j < kTPW; ++j) or64(half ? acc1[j] : acc0[j], o[j]);
                        }
                    }
                }
            }
        } else if constexpr (kM4R && kTPW > 2) {
            // 4 tiles per warp: the CTA builds every (slab, tile) table
            // (lanes of a warp on 16 different tiles: conflict-free stores),
            // then a barrier, then each warp looks up its tiles
            for (uint32_t pr = tid; pr < 16 * kBJ; pr += kNT) {
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
                    const uint64_t *ta = &S.tab[(s * 16 + (uint32_t)((pa >> (4 * s)) & 15u)) * kTabRow + kTPW * warp];
                    const uint64_t *tb = &S.tab[(s * 16 + (uint32_t)((pb >> (4 * s)) & 15u)) * kTabRow + kTPW * warp];
#pragma unroll
                    for (int j = 0; j < kTPW; ++j) {
                        or64(acc0[j], ta[j]);
                        or64(acc1[j], tb[j]);
                    }
                }
            }
        } else if constexpr (kM4R) {
            // at most 2 tiles per warp: each warp builds the tables of its
            // own tiles only (the only ones it reads), so no CTA-wide barrier
            // separates the build from the lookups.  Table (tile, slab) holds
            // the ORs of the 16 subsets of the slab's 4 Q rows; rows are 17
            // words apart, so the 16 keys of one lookup hit 16 different bank
            // pairs.
            if (wmask && !timed_out) {
                __syncwarp();  // the warp's lookups of the previous k-tile are done
                for (uint32_t pr = lane; pr < 16u * kTPW; pr += 32) {
                    const uint32_t s = pr / kTPW, jj = pr % kTPW;
                    const uint32_t j = kTPW * warp + jj;
                    const uint64_t *qr = &S.q[stage][j * 64 + 4 * s];
                    const uint64_t q0 = qr[0], q1 = qr[1], q2 = qr[2], q3 = qr[3];
                    uint64_t *t = &S.tab[(j * 16 + s) * kTabRow];
                    const uint64_t a01 = q0 | q1, a23 = q2 | q3;
                    t[0] = 0;
                    t[1] = q0;
                    t[2] = q1;
                    t[3] = a01;
                    t[4] = q2;
                    t[5] = q0 | q2;
                    t[6] = q1 | q2;
                    t[7] = a01 | q2;
                    t[8] = q3;
                    t[9] = q0 | q3;
                    t[10] = q1 | q3;
                    t[11] = a01 | q3;
                    t[12] = a23;
                    t[13] = q0 | a23;
                    t[14] = q1 | a23;
                    t[15] = a01 | a23;
                }
                __syncwarp();
                const uint64_t pa = ((uint64_t)pp.y << 32) | pp.x;  // row 2l
                const uint64_t pb = ((uint64_t)pp.w << 32) | pp.z;  // row 2l+1
#pragma unroll
                for (int s = 0; s < 16; ++s) {
                    const uint32_t ka = (uint32_t)((pa >> (4 * s)) & 15u), kb = (uint32_t)((pb >> (4 * s)) & 15u);
#pragma unroll
                    for (int j = 0; j < kTPW; ++j) {
                        const uint64_t *t = &S.tab[((kTPW * warp + j) * 16 + s) * kTabRow];
                        or64(acc0[j], t[ka]);
                        or64(acc1[j], t[kb]);
                    }
                }
            }
        } else {
            if (wmask && !timed_out) {
                const uint64_t *q = &S.q[stage][(kTPW * warp) * 64];
#pragma unroll
                for (int kk = 0; kk < 64; kk += 2) {
                    const uint32_t pa = kk < 32 ? pp.x : pp.y;  // row 2l
                    const uint32_t pb = kk < 32 ? pp.z : pp.w;  // row 2l+1
                    const int b = kk & 31;
                    const uint32_t ma0 = bitmask(pa, b), ma1 = bitmask(pa, b + 1);
                    const uint32_t mb0 = bitmask(pb, b), mb1 = bitmask(pb, b + 1);
#pragma unroll
                    for (int j = 0; j < kTPW; ++j) {
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
        if (tid == 0 && !timed_out && e + kSt < nk) staged += issue(e + kSt, stage);
    }
    if (stamps && tid == 0) stamps[2] = stamps[3] = globaltimer_ns();
    if (gate && *gate) {
        bool gave_up = false;
        if (tid == 0 && !timed_out && gate_seen < gate_target) {
            uint32_t spins = 0;
            while (ld_acquire_u32(*gate) < gate_target) {
                if (++spins > kGateSpinLimit) {
                    gave_up = true;
                    break;
                }
                __nanosleep(64);
            }
        }
        timed_out = __syncthreads_or(timed_out || gave_up) != 0;
        if (timed_out) return;
        *gate = nullptr;
        if (stamps && tid == 0) stamps[3] = globaltimer_ns();
    }
    // ---- epilogue: the 2*kTPW words of the thread in three batches (loads of C,
    // then the atomics that can add bits, then D / populations), so that
    // their global round trips overlap ----
    constexpr int kWords = 2 * kTPW;
    uint64_t av[kWords], seen[kWords], prev[kWords];
    size_t off[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
        const int j = k >> 1, rr = k & 1;
        const uint2 a2 = rr ? acc1[j] : acc0[j];
        const uint32_t tj = tj0 + kTPW * warp + j;
        av[k] = tj < T ? (((uint64_t)a2.y << 32) | a2.x) : 0ULL;
        off[k] = tile_offset(T, ti, tj < T ? tj : 0) + 2 * lane + rr;
        outw += av[k] != 0;
    }
#pragma unroll
    for (int k = 0; k < kWords; ++k)
        seen[k] = !av[k] ? ~0ULL
                  : direct_merge ? 0ULL
                                 : __ldcg(reinterpret_cast<const unsigned long long *>(C.bits + off[k]));
#pragma unroll
    for (int k = 0; k < kWords; ++k)
        prev[k] = (av[k] & ~seen[k]) ? atomicOr(reinterpret_cast<unsigned long long *>(C.bits + off[k]),
                                                (unsigned long long)av[k])
                                     : ~0ULL;
    uint32_t tile_new[kTPW];
#pragma unroll
    for (int j = 0; j < kTPW; ++j) {
        uint32_t newcnt = 0;
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int k = 2 * j + rr;
            const uint64_t nw = av[k] & ~prev[k];
            if (nw) {
                ++neww;
                newcnt += __popcll(nw);
                if (D.bits) atomicOr(reinterpret_cast<unsigned long long *>(D.bits + off[k]), (unsigned long long)nw);
            }
        }
        tile_new[j] = __reduce_add_sync(kFull, newcnt);  // the warp's rows of tile tj0 + kTPW*warp + j
    }
    uint32_t mine = 0, any = 0;  // lane j updates tile j of the warp (populations, occupancy, buffer counters)
#pragma unroll
    for (int j = 0; j < kTPW; ++j) {
        any |= tile_new[j];
        if (lane == (uint32_t)j) mine = tile_new[j];
    }
    const bool any_new = any != 0;
    if (any_new) {
        tiles_gain(C, ti, tj0 + kTPW * warp, mine, cnts ? cnts + 3 * pd.head : nullptr);
        if (D.bits) tiles_gain(D, ti, tj0 + kTPW * warp, mine, cnts ? cnts + 3 * pd.head + 1 + ((iter & 1) ^ 1) : nullptr);
    }
    if (any_new && lane == 0) {
        *changed = 1u;
        if (qchanged) qchanged[pd.query] = 1u;
    }
    __syncthreads();  // k-list and stage reuse by the next item
}

}  // namespace tiled
}  // namespace cfpq
