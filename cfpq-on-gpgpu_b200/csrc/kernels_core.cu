// Core kernels: layout conversion, tile statistics (occupancy + population),
// bit scatter, result hash, the plain dense product, and the plan / advance
// steps of the device-resident closure iteration.
#include <algorithm>

#include "input_device.cuh"
#include "launch.h"
#include "plan_device.cuh"

namespace cfpq {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr unsigned long long kHashMod = 1000000007ULL;  // cfpq-cpp/Grammar.cpp:14

inline unsigned grid_for(size_t n, unsigned block) {
    size_t g = (n + block - 1) / block;
    return (unsigned)(g ? g : 1);
}

inline unsigned capped_grid(size_t n, unsigned block, unsigned cap) {
    const unsigned g = grid_for(n, block);
    return g > cap ? cap : g;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
    return __reduce_add_sync(kFull, v);
}

// Programmatic dependent launch: let the stream's next kernel (launched with
// the programmatic-serialization attribute) start before this one ends /
// wait until the stream's previous kernel has completed and its writes are
// visible (returns at once for a kernel launched without the attribute).
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---- initialisation ---------------------------------------------------------

__global__ void k_set_bits(DevMat m, const uint32_t *__restrict__ rows, const uint32_t *__restrict__ cols,
                           size_t count, uint32_t *bad) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        const uint32_t r = rows[e], c = cols[e];
        if (r >= m.n || c >= m.n) {
            atomicAdd(bad, 1u);
            continue;
        }
        set_one_bit(m, r, c);
    }
}

// Edge scatter: edge e sets (from, to) in every matrix its label derives
// (cfpq-cpp/Grammar.h:41-45).  The label -> matrices tables and the matrix
// descriptors (kLoadTableBytes at most) are copied into shared memory while
// the block's first edges load, so an edge waits only for its vertex order
// entries and its bit's atomic; larger tables are read from global memory.
// After the input phase's first kernel (programmatic dependent launch) the
// block starts while that kernel still clears the matrices: the edge and
// table loads, which do not depend on it, go first, and pdl_wait() keeps
// every write to the matrices and the counter after its end.
constexpr uint32_t kLoadTableBytes = 12288;

template <bool kSmem>
__global__ void k_load_edges(const DevMat *__restrict__ mats, uint32_t nmats, const uint32_t *__restrict__ from,
                             const uint32_t *__restrict__ label, const uint32_t *__restrict__ to, size_t ne,
                             const uint32_t *__restrict__ off, const uint32_t *__restrict__ lm, uint32_t nlabels,
                             uint32_t nlm, uint32_t *bad) {
    extern __shared__ __align__(16) unsigned char load_smem[];
    if constexpr (kSmem) {
        DevMat *sm = reinterpret_cast<DevMat *>(load_smem);
        uint32_t *so = reinterpret_cast<uint32_t *>(sm + nmats), *sl = so + nlabels + 1;
        for (uint32_t i = threadIdx.x; i < nmats; i += blockDim.x) sm[i] = mats[i];
        for (uint32_t i = threadIdx.x; i <= nlabels; i += blockDim.x) so[i] = off[i];
        for (uint32_t i = threadIdx.x; i < nlm; i += blockDim.x) sl[i] = lm[i];
        mats = sm;
        off = so;
        lm = sl;
    }
    size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    uint32_t l = 0, r = 0, c = 0;
    if (e < ne) {  // the first edge's loads overlap the table copies
        l = label[e];
        r = from[e];
        c = to[e];
    }
    if constexpr (kSmem) __syncthreads();
    pdl_wait();
    for (; e < ne; e += (size_t)gridDim.x * blockDim.x) {
        scatter_edge(mats, off, lm, nlabels, l, r, c, bad);
        const size_t e2 = e + (size_t)gridDim.x * blockDim.x;
        if (e2 < ne) {
            l = label[e2];
            r = from[e2];
            c = to[e2];
        }
    }
}

__global__ void k_set_diag(DevMat m) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m.n; i += gridDim.x * blockDim.x) set_one_bit(m, i, i);
}

// Recompute occupancy and population from the bits.  One warp per occupancy
// word (32 tiles of one tile-row).
__global__ void k_tile_stats(DevMat m) {
    const size_t gw = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (gw >= (size_t)m.T * m.ow) return;
    const uint32_t ti = (uint32_t)(gw / m.ow), w = (uint32_t)(gw % m.ow);
    uint32_t word = 0;
    for (uint32_t t = 0; t < 32; ++t) {
        const uint32_t tj = w * 32 + t;
        if (tj >= m.T) break;
        const uint64_t *tile = m.bits + tile_offset(m.T, ti, tj);
        const uint32_t cnt = warp_sum(__popcll(tile[lane]) + __popcll(tile[lane + 32]));
        if (cnt) word |= 1u << t;
        if (lane == 0) m.nnz[(size_t)ti * m.T + tj] = cnt;
    }
    if (lane == 0) m.occ[(size_t)ti * m.ow + w] = word;
}

// Seeded random matrix (autotuner inputs): bit (r, c) set with probability
// thresh / 2^32 from a hash of (seed, r, c); padding rows/columns stay zero.
__device__ __forceinline__ uint32_t hash3(uint64_t seed, uint32_t r, uint32_t c) {
    uint64_t x = seed ^ ((uint64_t)r << 32 | c);
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return (uint32_t)((x ^ (x >> 31)) >> 32);
}

__global__ void k_random_fill(DevMat m, uint32_t thresh, uint64_t seed) {
    const size_t total = (size_t)m.T * m.T * 64;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        const size_t tile = x >> 6;
        const uint32_t row = (uint32_t)(tile / m.T) * 64 + (uint32_t)(x & 63), tj = (uint32_t)(tile % m.T);
        uint64_t w = 0;
        if (row < m.n)
            for (uint32_t b = 0; b < 64; ++b) {
                const uint32_t c = tj * 64 + b;
                if (c < m.n && hash3(seed, row, c) < thresh) w |= 1ULL << b;
            }
        m.bits[x] = w;
    }
}

// Row-major staging (n rows x T words) -> tiles.
__global__ void k_rows_to_tiles(DevMat m, const uint64_t *__restrict__ rows) {
    const size_t total = (size_t)m.T * m.T * 64;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(x & 63);
        const size_t tile = x >> 6;
        const uint32_t ti = (uint32_t)(tile / m.T), tj = (uint32_t)(tile % m.T);
        const uint32_t row = ti * 64 + r;
        m.bits[x] = row < m.n ? rows[(size_t)row * m.T + tj] : 0ULL;
    }
}

__global__ void k_tiles_to_rows(DevMat m, uint64_t *__restrict__ rows) {
    const size_t total = (size_t)m.n * m.T;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(x / m.T), w = (uint32_t)(x % m.T);
        if (!m.perm) {
            rows[x] = m.bits[tile_offset(m.T, row >> 6, w) + (row & 63)];
            continue;
        }
        // ordered matrix: gather the 64 bits of original columns 64w..64w+63
        const uint32_t ir = m.perm[row];
        const uint64_t *rbase = m.bits + tile_offset(m.T, ir >> 6, 0) + (ir & 63);
        uint64_t out = 0;
        const uint32_t cend = min(m.n, 64 * w + 64);
        for (uint32_t c = 64 * w; c < cend; ++c) {
            const uint32_t ic = m.perm[c];
            out |= ((rbase[(size_t)(ic >> 6) * 64] >> (ic & 63)) & 1ULL) << (c & 63);
        }
        rows[x] = out;
    }
}

// Ordered upload: scatter the set bits of row-major staging (original ids).
__global__ void k_rows_scatter(DevMat m, const uint64_t *__restrict__ rows) {
    const size_t total = (size_t)m.n * m.T;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        uint64_t v = rows[x];
        const uint32_t row = (uint32_t)(x / m.T), w = (uint32_t)(x % m.T);
        while (v) {
            const uint32_t c = 64 * w + (__ffsll((long long)v) - 1);
            v &= v - 1;
            if (c < m.n) set_one_bit(m, row, c);
        }
    }
}

// ---- result hash ------------------------------------------------------------
// The reference's Horner loop (cfpq-cpp/Grammar.cpp:86-97) equals
//   hash = sum over set bits (r, c) of 11^(n-1-c) * 13^(n-1-r)   (mod p),
// a sum that is linear in the bits, so every tile is reduced independently
// and only occupied tiles are read.
//
// Column terms of one occupied tile (ti, tj) (one warp): lane l takes rows
// l and l + 32.  A row's column term, Sum over its set bits c of
// 11^(n-1-c), is the sum over the 16 nibbles of its tile word of a nibble
// table entry: sub[p * 16 + v] = Sum over the set bits b of v of
// 11^(n-1-c) for column c = 64 tj + 4 p + b (k_pow_nibbles, 256 entries per
// tile column).  The warp loads the column's table with 8 coalesced loads
// (lane l of register k holds entry 32 k + l), so the lookup of nibble p is
// one shuffle from register p / 2, lane 16 (p & 1) + v: a tile costs one
// round of coalesced loads and 32 shuffles.  The row power 13^(n-1-r) is
// the same for every tile of the row, so the column terms are only added
// here (acc0 / acc1, rows l and l + 32) and multiplied once per row by the
// caller.  Entries are below p < 2^30, so a tile adds less than 2^34 to
// acc0 and acc1.
__device__ __forceinline__ void hash_tile(const DevMat &m, const uint32_t *__restrict__ nib11, uint32_t ti,
                                          uint32_t tj, unsigned long long &acc0, unsigned long long &acc1,
                                          unsigned long long &cnt) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t *tile = m.bits + tile_offset(m.T, ti, tj);
    const uint32_t *tab = nib11 + (size_t)tj * 256;
    uint32_t t[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = tab[k * 32 + lane];
    const uint64_t w0 = tile[lane], w1 = tile[lane + 32];
    cnt += __popcll(w0) + __popcll(w1);
#pragma unroll
    for (int p = 0; p < 16; ++p) {
        const uint32_t hi = (uint32_t)(p & 1) << 4;
        acc0 += __shfl_sync(kFull, t[p >> 1], (int)(hi | (uint32_t)((w0 >> (4 * p)) & 15u)));
        acc1 += __shfl_sync(kFull, t[p >> 1], (int)(hi | (uint32_t)((w1 >> (4 * p)) & 15u)));
    }
}

// Nibble tables of the column powers (one entry per thread):
// sub[tj * 256 + p * 16 + v] = Sum over the set bits b of v of
// pow11[64 tj + 4 p + b] mod p.
__global__ void k_pow_nibbles(const uint32_t *__restrict__ pow11, uint32_t T, uint32_t *__restrict__ sub) {
    const size_t total = (size_t)T * 256;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(x & 15u);
        const size_t col0 = (x >> 4) * 4;  // first column of nibble p of tile column tj
        unsigned long long acc = 0;
#pragma unroll
        for (uint32_t b = 0; b < 4; ++b)
            if ((v >> b) & 1u) acc += pow11[col0 + b];
        sub[x] = (uint32_t)(acc % kHashMod);
    }
}

// Sum of (h, cnt) over the block (8 warps); the totals are valid in thread 0.
__device__ __forceinline__ void block_sum2(unsigned long long &h, unsigned long long &cnt) {
    __shared__ unsigned long long sh[8], sc[8];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        h += __shfl_down_sync(kFull, h, o);
        cnt += __shfl_down_sync(kFull, cnt, o);
    }
    if (lane == 0) {
        sh[warp] = h;
        sc[warp] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (uint32_t i = 1; i < nw; ++i) {
            h += sh[i];
            cnt += sc[i];
        }
    __syncthreads();  // sh / sc free for the next call
}

// Result lines of several matrices in one launch.  Block b hashes tile-row
// b - start[i] of matrix i (its occupied tiles dealt round-robin to the 8
// warps) into partial[b]; the last block to finish (ticket, which it resets
// to 0 for the next launch) adds every matrix's partials and writes out[2i]
// = hash mod p and out[2i+1] = bit count, so the output needs no zeroing
// and may live in mapped host memory.  No sum can overflow: a tile adds
// less than 2^33 to a lane's row sums (below 2^59 over fewer than 2^26
// tiles), every thread's term and every row's partial are reduced mod p
// (< 2^30) before they are added up, and a matrix has fewer than 2^26
// tile-rows.
__global__ void __launch_bounds__(256, 6) k_hash_lines(HashBatch hb, unsigned long long *__restrict__ partial,
                                                       uint32_t *ticket, unsigned long long *out) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t i = 0;
    while (i + 1 < hb.count && blockIdx.x >= hb.start[i + 1]) ++i;
    const DevMat &m = hb.m[i];
    const uint32_t ti = blockIdx.x - hb.start[i];
    const uint32_t *orow = m.occ + (size_t)ti * m.ow;
    const uint32_t *nib11 = hb.nib11[i];
    const uint32_t q0 = hb.pow13[i][(size_t)ti * 64 + lane], q1 = hb.pow13[i][(size_t)ti * 64 + lane + 32];
    unsigned long long acc0 = 0, acc1 = 0, cnt = 0;
    uint32_t k = 0;  // occupied tiles of the row seen so far (the deal order)
    for (uint32_t base = 0; base < m.ow; base += 32) {
        const uint32_t mine = base + lane < m.ow ? orow[base + lane] : 0u;
        unsigned todo = __ballot_sync(kFull, mine != 0);
        while (todo) {
            const uint32_t src = __ffs(todo) - 1;
            todo &= todo - 1;
            uint32_t bits = __shfl_sync(kFull, mine, src);
            while (bits) {
                const uint32_t tj = (base + src) * 32 + (__ffs(bits) - 1);
                bits &= bits - 1;
                if (k++ % nw == warp) hash_tile(m, nib11, ti, tj, acc0, acc1, cnt);
            }
        }
    }
    unsigned long long h = (acc0 % kHashMod) * q0 % kHashMod + (acc1 % kHashMod) * q1 % kHashMod;
    block_sum2(h, cnt);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = h % kHashMod;
        partial[2 * blockIdx.x + 1] = cnt;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // warp j adds the partials of matrices j, j + 8, ...: independent loads, no block barrier
    for (uint32_t j = warp; j < hb.count; j += nw) {
        unsigned long long H = 0, C = 0;
#pragma unroll 4
        for (uint32_t b = hb.start[j] + lane; b < hb.start[j + 1]; b += 32) {
            H += __ldcg(partial + 2 * b);
            C += __ldcg(partial + 2 * b + 1);
        }
        for (int o = 16; o > 0; o >>= 1) {
            H += __shfl_xor_sync(kFull, H, o);
            C += __shfl_xor_sync(kFull, C, o);
        }
        if (lane == 0) {
            out[2 * j] = H % kHashMod;
            out[2 * j + 1] = C;
        }
    }
    if (threadIdx.x == 0) *ticket = 0;
}

// ---- plain dense product (variant PLAIN) ------------------------------------
// The "plain single-variant" form: every output word walks the whole inner
// dimension bit by bit, no shared memory, no tiles skipped -- the work shape of
// the reference's naive kernel (cuda/naive-gpu/Multiplication.cu:33-74) on this
// library's layout.  Block = the 64 rows of output tile (ti, tj).
__global__ void __launch_bounds__(64) k_plain_product(DevMat a, DevMat b, DevMat c, int mode, uint32_t *flag) {
    const uint32_t tj = blockIdx.x, ti = blockIdx.y, r = threadIdx.x;
    const uint32_t T = a.T;
    uint64_t acc = 0;
    for (uint32_t tk = 0; tk < T; ++tk) {
        const uint64_t av = a.bits[tile_offset(T, ti, tk) + r];
        const uint64_t *bt = b.bits + tile_offset(T, tk, tj);
        for (int kk = 0; kk < 64; ++kk)
            if ((av >> kk) & 1ULL) acc |= bt[kk];
    }
    uint64_t *cw = c.bits + tile_offset(T, ti, tj) + r;
    __shared__ uint32_t s_cnt;
    if (r == 0) s_cnt = 0;
    __syncthreads();
    if (mode == 0) {
        const uint64_t old = *cw;
        const uint64_t nw = acc & ~old;
        if (nw) {
            *cw = old | acc;
            atomicAdd(&s_cnt, (uint32_t)__popcll(nw));
        }
        __syncthreads();
        if (r == 0 && s_cnt) {
            atomicAdd(c.nnz + (size_t)ti * T + tj, s_cnt);
            set_occ_bit(c, ti, tj);
            *flag = 1;
        }
    } else {
        *cw = acc;
        if (acc) atomicAdd(&s_cnt, (uint32_t)__popcll(acc));
        __syncthreads();
        if (r == 0) {
            c.nnz[(size_t)ti * T + tj] = s_cnt;
            uint32_t *ow = c.occ + (size_t)ti * c.ow + (tj >> 5);
            if (s_cnt)
                atomicOr(ow, 1u << (tj & 31));
            else
                atomicAnd(ow, ~(1u << (tj & 31)));
        }
    }
}

// dst |= src over occupied tiles of src.  Block of 64 threads per tile.
__global__ void __launch_bounds__(64) k_merge_or(DevMat dst, DevMat src, uint32_t *flag) {
    const uint32_t tj = blockIdx.x, ti = blockIdx.y, r = threadIdx.x;
    if (!((src.occ[(size_t)ti * src.ow + (tj >> 5)] >> (tj & 31)) & 1u)) return;
    const uint64_t v = src.bits[tile_offset(src.T, ti, tj) + r];
    uint64_t *dw = dst.bits + tile_offset(dst.T, ti, tj) + r;
    const uint64_t old = *dw;
    const uint64_t nw = v & ~old;
    if (nw) *dw = old | v;
    __shared__ uint32_t s_cnt;
    if (r == 0) s_cnt = 0;
    __syncthreads();
    if (nw) atomicAdd(&s_cnt, (uint32_t)__popcll(nw));
    __syncthreads();
    if (r == 0 && s_cnt) {
        atomicAdd(dst.nnz + (size_t)ti * dst.T + tj, s_cnt);
        set_occ_bit(dst, ti, tj);
        *flag = 1;
    }
}

// ---- closure iteration: plan ---------------------------------------------------
// One warp per (product, tile-row); the planner itself is plan::plan_row.
constexpr int kPlanThreads = 128;

__global__ void __launch_bounds__(kPlanThreads)
    k_plan(const ProdDesc *__restrict__ prods, uint32_t nprods, uint32_t row_begin, uint32_t total_rows,
           const MatSlot *__restrict__ slots, IterState *st, uint64_t *__restrict__ items_all, size_t list_cap,
           int tpb, uint32_t *prod_seen, int tc_mode, PlanSelect ps) {
    __shared__ plan::WarpArea<plan::kPlanMaxBlocks> areas[kPlanThreads / 32];
    const uint32_t gw = row_begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (gw >= total_rows || !st->active) return;
    plan::plan_row(gw, prods, nprods, slots, st->iter, st, st->item_count, items_all, list_cap, tpb, prod_seen,
                   tc_mode, ps, areas[threadIdx.x >> 5].cnt, areas[threadIdx.x >> 5].bnd);
}

// Tensor-core plan of every tensor-core-capable product of a closure in one
// launch: the products' groups of 4 tile-rows laid end to end, one warp per
// group (tc[i].pref groups come before product tc[i].prod).  A product whose
// variant is not TC this iteration plans nothing.
__global__ void __launch_bounds__(kPlanThreads)
    k_plan_tc(const ProdDesc *__restrict__ prods, uint32_t nprods, const TcRows *__restrict__ tc, uint32_t ntc,
              uint32_t total, const MatSlot *__restrict__ slots, IterState *st, uint64_t *__restrict__ items_all,
              size_t list_cap, int tpb, uint32_t *prod_seen, PlanSelect ps) {
    __shared__ plan::WarpArea<plan::kPlanMaxBlocks> areas[kPlanThreads / 32];
    const uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= total || !st->active) return;
    uint32_t lo = 0, hi = ntc;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (tc[mid].pref <= r) lo = mid; else hi = mid;
    }
    const TcRows t = tc[lo];
    plan::plan_row(t.row_start + (r - t.pref), prods, nprods, slots, st->iter, st, st->item_count, items_all,
                   list_cap, tpb, prod_seen, 1, ps, areas[threadIdx.x >> 5].cnt, areas[threadIdx.x >> 5].bnd, t.prod,
                   t.prod + 1);
}

// ---- closure iteration: advance + end ----------------------------------------
// Clears the delta buffer that was read in this iteration (it receives the next
// iteration's new bits): zero every occupied tile and its population, then the
// occupancy row.  One warp per (slot, tile-row).  The last block to finish
// (counter in IterState) then ends the iteration: publishes the changed flag,
// advances the iteration index, decides whether to continue (the graph's
// while-node condition) and records per-query convergence.  A launch after the
// loop has stopped only clears (the host may run a few iterations
// speculatively between checks).
__global__ void k_advance_end(const MatSlot *__restrict__ slots, uint32_t nslots, uint32_t total_rows,
                              IterState *st, QueryTrack qt, cudaGraphConditionalHandle handle, int use_handle,
                              BufCounters *cnts) {
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw < total_rows && nslots > 0) clear_delta_row(slots, nslots, gw, st->iter & 1);

    __shared__ uint32_t s_last, s_run, s_iter, s_go;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&st->blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (cnts) {  // the delta just cleared starts the next iteration empty
        const uint32_t b = 1 + (st->iter & 1);
        for (uint32_t sl = threadIdx.x; sl < nslots; sl += blockDim.x) cnts[3 * sl + b] = BufCounters{0, 0, 0};
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        st->blocks_done = 0;
        s_run = st->active;
        s_go = 0;
        if (s_run) {
            const uint32_t changed = st->changed;
            st->last_changed = changed;
            st->changed = 0;
            st->items_total += st->item_count[0] + st->item_count[1] + st->item_count[2];
            st->items_by_variant[2] += st->item_count[0];
            st->items_by_variant[3] += st->item_count[1];
            st->items_by_variant[4] += st->item_count[2];
            st->item_count[0] = st->item_count[1] = st->item_count[2] = 0;
            st->item_next[0] = st->item_next[1] = st->item_next[2] = 0;
            const uint32_t it = ++st->iter;
            s_iter = it;
            s_go = changed && st->error == 0 && (st->max_iter == 0 || it < st->max_iter);
            st->active = s_go;
        }
    }
    __syncthreads();
    if (s_run && qt.changed) {
        const unsigned long long now = globaltimer_ns();
        for (uint32_t q = threadIdx.x; q < st->nqueries; q += blockDim.x) {
            if (qt.changed[q]) {
                qt.changed[q] = 0;
                qt.last_iter[q] = s_iter;
                qt.done_ns[q] = now;
            }
        }
    }
    if (threadIdx.x == 0 && use_handle) cudaGraphSetConditional(handle, s_go ? 1u : 0u);
}

// Closure prologue in one launch: zero the given word ranges, fill the
// variant choices, initialise the iteration state and stamp its start.
// The closure prologue's work, spread over the whole grid (block 0 also
// initialises the iteration state; every thread of block 0 must call it).
__device__ __forceinline__ void closure_begin_body(const ClosureBegin &a) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nt = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < ClosureBegin::kRanges; ++r)
        for (size_t i = tid; i < a.nwords[r]; i += nt) a.zero[r][i] = 0u;
    for (size_t i = tid; i < a.nchoice; i += nt) a.choice[i] = a.choice_value;
    if (blockIdx.x == 0) {
        uint32_t *w = reinterpret_cast<uint32_t *>(a.st);
        for (size_t i = threadIdx.x; i < sizeof(IterState) / 4; i += blockDim.x) w[i] = 0u;
        __syncthreads();
        if (threadIdx.x == 0) {
            a.st->active = 1;
            a.st->max_iter = a.max_iter;
            a.st->nqueries = a.nqueries;
            a.st->t_start_ns = globaltimer_ns();
        }
    }
}

__global__ void k_closure_begin(ClosureBegin a) { closure_begin_body(a); }

// Clear a list of matrices: one warp per (matrix, tile-row), occupied tiles only.
__global__ void k_clear_rows(const MatRows *__restrict__ tab, uint32_t nmats, uint32_t total_rows) {
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw < total_rows) clear_unit(tab, nmats, gw);
}

// First kernel of a query's input phase: the clear of its matrices, the
// scatter's out-of-range counter set to 0 and (with_begin) the closure
// prologue, in one launch ahead of the scatter.
__global__ void k_input_first(const MatRows *__restrict__ tab, uint32_t nmats, uint32_t total_rows, uint32_t *bad,
                              ClosureBegin begin, int with_begin) {
    pdl_launch_dependents();  // the scatter may start its loads now
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw < total_rows) clear_unit(tab, nmats, gw);
    if (bad && blockIdx.x == 0 && threadIdx.x == 0) *bad = 0u;
    if (with_begin) closure_begin_body(begin);
}

// Diagonals of a list of matrices (epsilon nonterminals).
__global__ void k_set_diags(const DevMat *__restrict__ diag, uint32_t ndiag) {
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x, nt = (size_t)gridDim.x * blockDim.x;
    for (uint32_t d = 0; d < ndiag; ++d) {
        const DevMat m = diag[d];
        for (size_t i = tid; i < m.n; i += nt) set_one_bit(m, (uint32_t)i, (uint32_t)i);
    }
}

}  // namespace

// ---- launch wrappers -------------------------------------------------------------

cudaError_t launch_set_bits(const DevMat &m, const uint32_t *d_rows, const uint32_t *d_cols, size_t count,
                            uint32_t *d_bad, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_set_bits<<<capped_grid(count, 256, 65535u * 16), 256, 0, s>>>(m, d_rows, d_cols, count, d_bad);
    return cudaGetLastError();
}

cudaError_t launch_load_edges(const DevMat *d_mats, uint32_t nmats, const uint32_t *d_from, const uint32_t *d_label,
                              const uint32_t *d_to, size_t ne, const uint32_t *d_off, const uint32_t *d_lm,
                              uint32_t nlabels, uint32_t nlm, uint32_t *d_bad, cudaStream_t s, bool dependent) {
    if (ne == 0) return cudaSuccess;
    const size_t tb = (size_t)nmats * sizeof(DevMat) + ((size_t)nlabels + 1 + nlm) * 4;
    const bool smem = tb <= kLoadTableBytes;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(capped_grid(ne, 256, 65535u * 16));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem ? tb : 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = dependent ? 1 : 0;
    return smem ? cudaLaunchKernelEx(&cfg, k_load_edges<true>, d_mats, nmats, d_from, d_label, d_to, ne, d_off, d_lm,
                                     nlabels, nlm, d_bad)
                : cudaLaunchKernelEx(&cfg, k_load_edges<false>, d_mats, nmats, d_from, d_label, d_to, ne, d_off,
                                     d_lm, nlabels, nlm, d_bad);
}

cudaError_t launch_set_diag(const DevMat &m, cudaStream_t s) {
    if (m.n == 0) return cudaSuccess;
    k_set_diag<<<grid_for(m.n, 256), 256, 0, s>>>(m);
    return cudaGetLastError();
}

cudaError_t launch_occ_rebuild(const DevMat &m, cudaStream_t s) {
    if (m.T == 0) return cudaSuccess;
    const size_t warps = (size_t)m.T * m.ow;
    k_tile_stats<<<grid_for(warps * 32, 256), 256, 0, s>>>(m);
    return cudaGetLastError();
}

cudaError_t launch_random_fill(const DevMat &m, double density, uint64_t seed, cudaStream_t s) {
    if (m.T == 0) return cudaSuccess;
    const double t = density <= 0 ? 0.0 : (density >= 1 ? 4294967295.0 : density * 4294967296.0);
    k_random_fill<<<capped_grid((size_t)m.T * m.T * 64, 256, 1u << 16), 256, 0, s>>>(m, (uint32_t)t, seed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_occ_rebuild(m, s);
}

cudaError_t launch_rows_to_tiles(const DevMat &m, const uint64_t *d_rows, cudaStream_t s) {
    if (m.T == 0) return cudaSuccess;
    if (m.perm) {
        cudaError_t e = launch_clear_matrix(m, s);
        if (e != cudaSuccess) return e;
        const size_t words = (size_t)m.n * m.T;
        k_rows_scatter<<<capped_grid(words, 256, 1u << 20), 256, 0, s>>>(m, d_rows);
        return cudaGetLastError();
    }
    const size_t total = (size_t)m.T * m.T * 64;
    k_rows_to_tiles<<<capped_grid(total, 256, 1u << 20), 256, 0, s>>>(m, d_rows);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_occ_rebuild(m, s);
}

cudaError_t launch_tiles_to_rows(const DevMat &m, uint64_t *d_rows, cudaStream_t s) {
    if (m.n == 0) return cudaSuccess;
    const size_t total = (size_t)m.n * m.T;
    k_tiles_to_rows<<<capped_grid(total, 256, 1u << 20), 256, 0, s>>>(m, d_rows);
    return cudaGetLastError();
}

// delta = cur & ~prev, then prev = cur (whole matrices, word by word); the
// tile statistics of delta and prev are rebuilt afterwards.
__global__ void k_delta_snapshot(DevMat delta, DevMat cur, DevMat prev) {
    const size_t words = (size_t)cur.T * cur.T * 64;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t c = cur.bits[i];
        delta.bits[i] = c & ~prev.bits[i];
        prev.bits[i] = c;
    }
}

cudaError_t launch_delta_snapshot(const DevMat &delta, const DevMat &cur, const DevMat &prev, cudaStream_t s) {
    if (cur.T == 0) return cudaSuccess;
    if (delta.T != cur.T || prev.T != cur.T) return cudaErrorInvalidValue;
    k_delta_snapshot<<<capped_grid((size_t)cur.T * cur.T * 64, 256, 1u << 16), 256, 0, s>>>(delta, cur, prev);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = launch_occ_rebuild(delta, s)) != cudaSuccess) return e;
    return launch_occ_rebuild(prev, s);
}

cudaError_t launch_copy_matrix(const DevMat &dst, const DevMat &src, cudaStream_t s) {
    if (dst.T != src.T) return cudaErrorInvalidValue;
    if (dst.T == 0) return cudaSuccess;
    cudaError_t e = cudaMemcpyAsync(dst.bits, src.bits, (size_t)src.T * src.T * 512, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(dst.nnz, src.nnz, (size_t)src.T * src.T * 4, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(dst.occ, src.occ, (size_t)src.T * src.ow * 4, cudaMemcpyDeviceToDevice, s);
}

cudaError_t launch_clear_matrix(const DevMat &m, cudaStream_t s) {
    if (m.T == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(m.bits, 0, (size_t)m.T * m.T * 512, s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(m.nnz, 0, (size_t)m.T * m.T * 4, s);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(m.occ, 0, (size_t)m.T * m.ow * 4, s);
}

cudaError_t launch_pow_nibbles(const uint32_t *d_pow11, uint32_t T, uint32_t *d_sub, cudaStream_t s) {
    if (T == 0) return cudaSuccess;
    k_pow_nibbles<<<capped_grid((size_t)T * 256, 256, 65535u), 256, 0, s>>>(d_pow11, T, d_sub);
    return cudaGetLastError();
}

cudaError_t launch_hash_lines(const HashBatch &hb, unsigned long long *d_partial, uint32_t *d_ticket,
                              unsigned long long *out, cudaStream_t s) {
    if (hb.count == 0 || hb.start[hb.count] == 0) return cudaErrorInvalidValue;
    k_hash_lines<<<hb.start[hb.count], 256, 0, s>>>(hb, d_partial, d_ticket, out);
    return cudaGetLastError();
}

cudaError_t launch_plain_product(const DevMat &a, const DevMat &b, const DevMat &c, int mode, uint32_t *d_flag,
                                 cudaStream_t s) {
    if (a.T == 0) return cudaSuccess;
    k_plain_product<<<dim3(a.T, a.T), 64, 0, s>>>(a, b, c, mode, d_flag);
    return cudaGetLastError();
}

cudaError_t launch_merge_or(const DevMat &dst, const DevMat &src, uint32_t *d_flag, cudaStream_t s) {
    if (dst.T == 0) return cudaSuccess;
    k_merge_or<<<dim3(dst.T, dst.T), 64, 0, s>>>(dst, src, d_flag);
    return cudaGetLastError();
}

cudaError_t launch_plan(const ProdDesc *d_prods, uint32_t nprods, uint32_t row_begin, uint32_t row_end,
                        const MatSlot *d_slots, IterState *d_st, uint64_t *d_items, size_t list_cap,
                        int tiles_per_block, uint32_t *d_prod_seen, int tc_mode, const uint8_t *d_choice,
                        cudaStream_t s, const PlanSelect *sel, const uint32_t *d_q_last) {
    if (row_end <= row_begin || nprods == 0) return cudaSuccess;
    PlanSelect ps = sel ? *sel
                        : PlanSelect{nullptr, nullptr, nullptr, const_cast<uint8_t *>(d_choice), nullptr, 0, nullptr};
    ps.q_last = d_q_last;
    k_plan<<<grid_for((size_t)(row_end - row_begin) * 32, kPlanThreads), kPlanThreads, 0, s>>>(
        d_prods, nprods, row_begin, row_end, d_slots, d_st, d_items, list_cap, tiles_per_block, d_prod_seen, tc_mode,
        ps);
    return cudaGetLastError();
}

cudaError_t launch_plan_tc(const ProdDesc *d_prods, uint32_t nprods, const TcRows *d_tc, uint32_t ntc,
                           uint32_t total_groups, const MatSlot *d_slots, IterState *d_st, uint64_t *d_items,
                           size_t list_cap, int tiles_per_block, uint32_t *d_prod_seen, const uint8_t *d_choice,
                           cudaStream_t s, const uint32_t *d_q_last) {
    if (ntc == 0 || total_groups == 0) return cudaSuccess;
    const PlanSelect ps{nullptr, nullptr, nullptr, const_cast<uint8_t *>(d_choice), nullptr, 0, d_q_last};
    k_plan_tc<<<grid_for((size_t)total_groups * 32, kPlanThreads), kPlanThreads, 0, s>>>(
        d_prods, nprods, d_tc, ntc, total_groups, d_slots, d_st, d_items, list_cap, tiles_per_block, d_prod_seen, ps);
    return cudaGetLastError();
}

cudaError_t launch_advance_end(const MatSlot *d_slots, uint32_t nslots, uint32_t total_rows, IterState *d_st,
                               const QueryTrack &qt, cudaGraphConditionalHandle handle, int use_handle,
                               BufCounters *d_cnts, cudaStream_t s) {
    k_advance_end<<<grid_for((size_t)total_rows * 32, 256), 256, 0, s>>>(d_slots, nslots, total_rows, d_st, qt,
                                                                         handle, use_handle, d_cnts);
    return cudaGetLastError();
}

cudaError_t launch_clear_rows(const MatRows *d_tab, uint32_t nmats, uint32_t total_rows, cudaStream_t s) {
    if (total_rows == 0 || nmats == 0) return cudaSuccess;
    k_clear_rows<<<grid_for((size_t)total_rows * 32, 256), 256, 0, s>>>(d_tab, nmats, total_rows);
    return cudaGetLastError();
}

static unsigned closure_begin_blocks(const ClosureBegin &a, int num_sms) {
    size_t words = a.nchoice;
    for (int r = 0; r < ClosureBegin::kRanges; ++r) words = words > a.nwords[r] ? words : a.nwords[r];
    return (unsigned)std::max<size_t>(1, std::min<size_t>((words + 255) / 256, (size_t)num_sms * 4));
}

cudaError_t launch_closure_input(const ClosureInput &in, int num_sms, cudaStream_t s, const ClosureBegin *begin) {
    if (in.clear_rows || in.bad || begin) {
        const unsigned clear_blocks = in.clear_rows && in.nclear ? grid_for((size_t)in.clear_rows * 32, 256) : 1;
        const unsigned blocks = begin ? std::max(clear_blocks, closure_begin_blocks(*begin, num_sms)) : clear_blocks;
        ClosureBegin none;
        memset(&none, 0, sizeof(none));
        k_input_first<<<blocks, 256, 0, s>>>(in.clear, in.nclear, in.nclear ? in.clear_rows : 0, in.bad,
                                             begin ? *begin : none, begin ? 1 : 0);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const bool first_launched = in.clear_rows || in.bad || begin;
    if (in.nedges) {
        cudaError_t e = launch_load_edges(in.mats, in.nmats, in.from, in.label, in.to, in.nedges, in.off, in.lm,
                                          in.nlabels, in.nlm, in.bad, s, first_launched);
        if (e != cudaSuccess) return e;
    }
    if (in.ndiag) {
        k_set_diags<<<num_sms * 4, 256, 0, s>>>(in.diag, in.ndiag);
        return cudaGetLastError();
    }
    return cudaSuccess;
}

cudaError_t launch_closure_begin(const ClosureBegin &a, int num_sms, cudaStream_t s) {
    k_closure_begin<<<closure_begin_blocks(a, num_sms), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace cfpq
