// Core kernels: layout conversion, occupancy, bit scatter, result hash,
// the plain dense product, and the plan / advance steps of the device-resident
// closure iteration.
#include "launch.h"

namespace cfpq {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr unsigned long long kHashMod = 1000000007ULL;  // cfpq-cpp/Grammar.cpp:14

inline unsigned grid_for(size_t n, unsigned block) {
    size_t g = (n + block - 1) / block;
    return (unsigned)(g ? g : 1);
}

__device__ __forceinline__ void set_occ_bit(const DevMat &m, uint32_t ti, uint32_t tj) {
    atomicOr(m.occ + (size_t)ti * m.ow + (tj >> 5), 1u << (tj & 31));
}

// ---- initialisation ---------------------------------------------------------

__global__ void k_set_bits(DevMat m, const uint32_t *__restrict__ rows, const uint32_t *__restrict__ cols,
                           size_t count, uint32_t *bad) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        const uint32_t r = rows[e], c = cols[e];
        if (r >= m.n || c >= m.n) {
            atomicAdd(bad, 1u);
            continue;
        }
        unsigned long long *w =
            reinterpret_cast<unsigned long long *>(m.bits + tile_offset(m.T, r >> 6, c >> 6) + (r & 63));
        atomicOr(w, 1ULL << (c & 63));
        set_occ_bit(m, r >> 6, c >> 6);
    }
}

// Edge scatter: edge e sets (from, to) in every matrix its label derives
// (cfpq-cpp/Grammar.h:41-45).  All matrices share n.
__global__ void k_load_edges(const DevMat *__restrict__ mats, const uint32_t *__restrict__ from,
                             const uint32_t *__restrict__ label, const uint32_t *__restrict__ to, size_t ne,
                             const uint32_t *__restrict__ off, const uint32_t *__restrict__ lm, uint32_t nlabels,
                             uint32_t *bad) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ne; e += (size_t)gridDim.x * blockDim.x) {
        const uint32_t l = label[e];
        if (l >= nlabels) continue;
        const uint32_t r = from[e], c = to[e];
        for (uint32_t j = off[l]; j < off[l + 1]; ++j) {
            const DevMat m = mats[lm[j]];
            if (r >= m.n || c >= m.n) {
                atomicAdd(bad, 1u);
                continue;
            }
            unsigned long long *w =
                reinterpret_cast<unsigned long long *>(m.bits + tile_offset(m.T, r >> 6, c >> 6) + (r & 63));
            atomicOr(w, 1ULL << (c & 63));
            set_occ_bit(m, r >> 6, c >> 6);
        }
    }
}

__global__ void k_set_diag(DevMat m) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m.n; i += gridDim.x * blockDim.x) {
        unsigned long long *w =
            reinterpret_cast<unsigned long long *>(m.bits + tile_offset(m.T, i >> 6, i >> 6) + (i & 63));
        atomicOr(w, 1ULL << (i & 63));
        set_occ_bit(m, i >> 6, i >> 6);
    }
}

// One warp per occupancy word (32 tiles of one tile-row).
__global__ void k_occ_rebuild(DevMat m) {
    const size_t gw = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (gw >= (size_t)m.T * m.ow) return;
    const uint32_t ti = (uint32_t)(gw / m.ow), w = (uint32_t)(gw % m.ow);
    uint32_t word = 0;
    for (uint32_t t = 0; t < 32; ++t) {
        const uint32_t tj = w * 32 + t;
        if (tj >= m.T) break;
        const uint64_t *tile = m.bits + tile_offset(m.T, ti, tj);
        const uint64_t v = tile[lane] | tile[lane + 32];
        if (__any_sync(kFull, v != 0)) word |= 1u << t;
    }
    if (lane == 0) m.occ[(size_t)ti * m.ow + w] = word;
}

// Row-major staging (n rows x T words) -> tiles.  Thread per (tile-row, word, row-in-tile).
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
        rows[x] = m.bits[tile_offset(m.T, row >> 6, w) + (row & 63)];
    }
}

// ---- result hash ------------------------------------------------------------
// line_hash(row) = sum over set columns c of 11^(n-1-c)   (mod p)
// hash           = sum over rows r of line_hash(r) * 13^(n-1-r) (mod p)
// which is the closed form of the reference's Horner loop
// (cfpq-cpp/Grammar.cpp:86-97).  One block of 64 threads per tile-row; thread r
// owns row ti*64 + r and walks its words tile by tile (coalesced across the
// block).  d_out[0] accumulates the per-row terms (each < 2^30, so the 64-bit
// sum cannot overflow for n < 2^33), d_out[1] the bit count.
__global__ void k_hash_count(DevMat m, const uint32_t *__restrict__ pow11, const uint32_t *__restrict__ pow13,
                             unsigned long long *out) {
    const uint32_t ti = blockIdx.x;
    const uint32_t r = threadIdx.x;
    const uint32_t row = ti * 64 + r;
    unsigned long long line = 0, cnt = 0;
    for (uint32_t tj = 0; tj < m.T; ++tj) {
        if (!((m.occ[(size_t)ti * m.ow + (tj >> 5)] >> (tj & 31)) & 1u)) continue;
        uint64_t v = m.bits[tile_offset(m.T, ti, tj) + r];
        cnt += __popcll(v);
        const uint32_t base = tj * 64;
        while (v) {
            const int b = __ffsll((long long)v) - 1;
            v &= v - 1;
            line += pow11[base + b];
        }
    }
    unsigned long long h = 0;
    if (row < m.n) h = ((line % kHashMod) * pow13[row]) % kHashMod;
    for (int o = 16; o > 0; o >>= 1) {
        h += __shfl_down_sync(kFull, h, o);
        cnt += __shfl_down_sync(kFull, cnt, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, h);
        atomicAdd(out + 1, cnt);
    }
}

// ---- plain dense product (variant PLAIN) ------------------------------------
// The "plain single-variant" form: every output word walks the whole inner
// dimension bit by bit, no shared memory, no tiles skipped -- the same work
// shape as the reference's naive kernel (cuda/naive-gpu/Multiplication.cu:33-74)
// on this library's layout.  Block = the 64 rows of output tile (ti, tj).
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
    if (mode == 0) {
        const uint64_t old = *cw;
        const int changed = (acc & ~old) != 0;
        if (changed) *cw = old | acc;
        if (__syncthreads_or(changed) && r == 0) {
            set_occ_bit(c, ti, tj);
            *flag = 1;
        }
    } else {
        *cw = acc;
        const int nz = __syncthreads_or(acc != 0);
        if (r == 0) {
            uint32_t *ow = c.occ + (size_t)ti * c.ow + (tj >> 5);
            if (nz)
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
    const int changed = (v & ~old) != 0;
    if (changed) *dw = old | v;
    if (__syncthreads_or(changed) && r == 0) {
        set_occ_bit(dst, ti, tj);
        *flag = 1;
    }
}

// ---- closure iteration: plan ---------------------------------------------------
// One warp per (product, output tile-row ti).  The warp forms the coarse
// (tile-level) product row  OR_{tk : occP(ti,tk)} occQ(tk, :)  and emits one
// work item per block of `tpb` output tiles that can receive a bit.  The coarse
// product is exact for skipping: a tile pair contributes only if both tiles are
// occupied.
__device__ __forceinline__ DevMat resolve_operand(const MatSlot &s, uint8_t use_delta, uint32_t iter) {
    if (!use_delta || iter == 0) return s.cur;
    return s.dlt[iter & 1];
}

__global__ void k_plan(const ProdDesc *__restrict__ prods, uint32_t nprods, uint32_t row_begin, uint32_t total_rows,
                       const MatSlot *__restrict__ slots, IterState *st, uint64_t *__restrict__ items, int tpb,
                       uint32_t *prod_seen) {
    const uint32_t gw = row_begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (gw >= total_rows || !st->active) return;
    // product index: last p with row_start <= gw
    uint32_t lo = 0, hi = nprods;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (prods[mid].row_start <= gw) lo = mid; else hi = mid;
    }
    const ProdDesc pd = prods[lo];
    const uint32_t iter = st->iter;
    if (pd.term == 1 && iter == 0) return;  // first iteration: delta(A)*B with delta = A covers A*B
    const uint32_t ti = gw - pd.row_start;
    const DevMat P = resolve_operand(slots[pd.pslot], pd.p_delta, iter);
    const DevMat Q = resolve_operand(slots[pd.qslot], pd.q_delta, iter);
    const uint32_t ow = P.ow;
    const uint32_t *prow = P.occ + (size_t)ti * ow;
    const uint32_t bpw = 32 / tpb;  // blocks per occupancy word
    const uint32_t bmask = tpb == 32 ? 0xffffffffu : ((1u << tpb) - 1);
    bool emitted = false;
    for (uint32_t base = 0; base < ow; base += 32) {
        const uint32_t w = base + lane;
        uint32_t acc = 0;
        for (uint32_t pw = 0; pw < ow; ++pw) {
            uint32_t bits = prow[pw];
            while (bits) {
                const uint32_t tk = pw * 32 + (__ffs(bits) - 1);
                bits &= bits - 1;
                if (w < ow) acc |= Q.occ[(size_t)tk * ow + w];
            }
            if (__all_sync(kFull, w >= ow || acc == 0xffffffffu)) break;
        }
        for (uint32_t h = 0; h < bpw; ++h) {
            const bool has = w < ow && ((acc >> (h * tpb)) & bmask) != 0;
            const unsigned ball = __ballot_sync(kFull, has);
            if (!ball) continue;
            emitted = true;
            uint32_t basepos = 0;
            if (lane == 0) basepos = atomicAdd(&st->item_count, (uint32_t)__popc(ball));
            basepos = __shfl_sync(kFull, basepos, 0);
            if (has) {
                const uint32_t pos = basepos + __popc(ball & ((1u << lane) - 1));
                items[pos] = make_item(lo, ti, w * bpw + h);
            }
        }
    }
    if (emitted && lane == 0 && prod_seen) {
        if (atomicExch(&prod_seen[lo], iter + 1) != iter + 1) {
            atomicAdd(&st->products, 1ULL);
            atomicAdd(&st->dense_bitops, (unsigned long long)pd.n * pd.n * pd.n);
        }
    }
}

// ---- closure iteration: advance -------------------------------------------------
// Clears the delta buffer that was read in this iteration (it receives next
// iteration's new bits): zero every occupied tile, then the occupancy row.  One
// warp per (slot, tile-row).
__global__ void k_advance(const MatSlot *__restrict__ slots, uint32_t nslots, uint32_t total_rows, IterState *st) {
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (gw >= total_rows) return;
    uint32_t lo = 0, hi = nslots;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (slots[mid].row_start <= gw) lo = mid; else hi = mid;
    }
    const uint32_t ti = gw - slots[lo].row_start;
    const DevMat D = slots[lo].dlt[st->iter & 1];
    uint32_t *orow = D.occ + (size_t)ti * D.ow;
    for (uint32_t w = 0; w < D.ow; ++w) {
        uint32_t bits = orow[w];
        while (bits) {
            const uint32_t tj = w * 32 + (__ffs(bits) - 1);
            bits &= bits - 1;
            uint4 *tile = reinterpret_cast<uint4 *>(D.bits + tile_offset(D.T, ti, tj));
            tile[lane] = make_uint4(0, 0, 0, 0);
        }
    }
    __syncwarp();
    for (uint32_t w = lane; w < D.ow; w += 32) orow[w] = 0;
}

__global__ void k_mark_start(IterState *st) { st->t_start_ns = globaltimer_ns(); }

// End of one iteration: publish the changed flag, advance the iteration index,
// decide whether to continue, and record per-query convergence.  A call after
// the loop has stopped is a no-op (the host may run a few iterations
// speculatively between checks).
__global__ void k_iter_end(IterState *st, QueryTrack qt, cudaGraphConditionalHandle handle, int use_handle) {
    __shared__ uint32_t s_run, s_iter, s_go;
    if (threadIdx.x == 0) {
        s_run = st->active;
        s_go = 0;
        if (s_run) {
            const uint32_t changed = st->changed;
            st->last_changed = changed;
            st->changed = 0;
            st->items_total += st->item_count;
            st->item_count = 0;
            st->item_next = 0;
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

}  // namespace

// ---- launch wrappers -------------------------------------------------------------

cudaError_t launch_set_bits(const DevMat &m, const uint32_t *d_rows, const uint32_t *d_cols, size_t count,
                            uint32_t *d_bad, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const unsigned g = grid_for(count, 256) > 65535u * 16 ? 65535u * 16 : grid_for(count, 256);
    k_set_bits<<<g, 256, 0, s>>>(m, d_rows, d_cols, count, d_bad);
    return cudaGetLastError();
}

cudaError_t launch_load_edges(const DevMat *d_mats, const uint32_t *d_from, const uint32_t *d_label,
                              const uint32_t *d_to, size_t ne, const uint32_t *d_off, const uint32_t *d_lm,
                              uint32_t nlabels, uint32_t *d_bad, cudaStream_t s) {
    if (ne == 0) return cudaSuccess;
    const unsigned g = grid_for(ne, 256) > 65535u * 16 ? 65535u * 16 : grid_for(ne, 256);
    k_load_edges<<<g, 256, 0, s>>>(d_mats, d_from, d_label, d_to, ne, d_off, d_lm, nlabels, d_bad);
    return cudaGetLastError();
}

cudaError_t launch_set_diag(const DevMat &m, cudaStream_t s) {
    if (m.n == 0) return cudaSuccess;
    k_set_diag<<<grid_for(m.n, 256), 256, 0, s>>>(m);
    return cudaGetLastError();
}

cudaError_t launch_occ_rebuild(const DevMat &m, cudaStream_t s) {
    if (m.T == 0) return cudaSuccess;
    const size_t warps = (size_t)m.T * m.ow;
    k_occ_rebuild<<<grid_for(warps * 32, 256), 256, 0, s>>>(m);
    return cudaGetLastError();
}

cudaError_t launch_rows_to_tiles(const DevMat &m, const uint64_t *d_rows, cudaStream_t s) {
    if (m.T == 0) return cudaSuccess;
    const size_t total = (size_t)m.T * m.T * 64;
    const unsigned g = grid_for(total, 256) > (1u << 20) ? (1u << 20) : grid_for(total, 256);
    k_rows_to_tiles<<<g, 256, 0, s>>>(m, d_rows);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_occ_rebuild(m, s);
}

cudaError_t launch_tiles_to_rows(const DevMat &m, uint64_t *d_rows, cudaStream_t s) {
    if (m.n == 0) return cudaSuccess;
    const size_t total = (size_t)m.n * m.T;
    const unsigned g = grid_for(total, 256) > (1u << 20) ? (1u << 20) : grid_for(total, 256);
    k_tiles_to_rows<<<g, 256, 0, s>>>(m, d_rows);
    return cudaGetLastError();
}

cudaError_t launch_copy_matrix(const DevMat &dst, const DevMat &src, cudaStream_t s) {
    if (dst.T != src.T) return cudaErrorInvalidValue;
    if (dst.T == 0) return cudaSuccess;
    cudaError_t e = cudaMemcpyAsync(dst.bits, src.bits, (size_t)src.T * src.T * 512, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(dst.occ, src.occ, (size_t)src.T * src.ow * 4, cudaMemcpyDeviceToDevice, s);
}

cudaError_t launch_clear_matrix(const DevMat &m, cudaStream_t s) {
    if (m.T == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(m.bits, 0, (size_t)m.T * m.T * 512, s);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(m.occ, 0, (size_t)m.T * m.ow * 4, s);
}

cudaError_t launch_hash_count(const DevMat &m, const uint32_t *d_pow11, const uint32_t *d_pow13,
                              unsigned long long *d_out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(d_out, 0, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess || m.T == 0) return e;
    k_hash_count<<<m.T, 64, 0, s>>>(m, d_pow11, d_pow13, d_out);
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
                        const MatSlot *d_slots, IterState *d_st, uint64_t *d_items, int tiles_per_block,
                        uint32_t *d_prod_seen, cudaStream_t s) {
    if (row_end <= row_begin || nprods == 0) return cudaSuccess;
    k_plan<<<grid_for((size_t)(row_end - row_begin) * 32, 256), 256, 0, s>>>(
        d_prods, nprods, row_begin, row_end, d_slots, d_st, d_items, tiles_per_block, d_prod_seen);
    return cudaGetLastError();
}

cudaError_t launch_advance(const MatSlot *d_slots, uint32_t nslots, uint32_t total_rows, IterState *d_st,
                           cudaStream_t s) {
    if (total_rows == 0 || nslots == 0) return cudaSuccess;
    k_advance<<<grid_for((size_t)total_rows * 32, 256), 256, 0, s>>>(d_slots, nslots, total_rows, d_st);
    return cudaGetLastError();
}

cudaError_t launch_mark_start(IterState *d_st, cudaStream_t s) {
    k_mark_start<<<1, 1, 0, s>>>(d_st);
    return cudaGetLastError();
}

cudaError_t launch_iter_end(IterState *d_st, const QueryTrack &qt, cudaGraphConditionalHandle handle, int use_handle,
                            cudaStream_t s) {
    k_iter_end<<<1, 256, 0, s>>>(d_st, qt, handle, use_handle);
    return cudaGetLastError();
}

}  // namespace cfpq
