// Variant NTSET: the closure of one query as a single n x n matrix whose cells
// are sets of nonterminals (bit x of cell (i, j) = nonterminal x derives a
// path from vertex i to vertex j), closed by repeated squaring
//     M <- M | M (x) M      until a pass changes nothing,
// where the product of two cells is  a (x) b = { X : X -> Y Z, Y in a, Z in b }.
// This is the formulation of the reference's CUTLASS backend
// (cuda/cutlass/CutlassMatrix.cu:290-316: C = A (x) A, then C |= A with a
// changed flag, MatAddKernel :220-230; the rule encoding of
// cfpq-cpp/Grammar.cpp:63-75, one bit per nonterminal) -- one product per
// iteration for all rules instead of one per rule.  Its least fixpoint is the
// same as that of the per-nonterminal matrices, so the result is identical.
//
// Cells: 8 bits for up to 8 nonterminals, 32 bits for up to 32.  Layout:
// row-major, `stride` = n rounded up to 64 cells per row (internal vertex
// order of the query's matrices).
//
// Squaring kernel (one CTA per row at a time, rows taken from an atomic
// counter): the row's non-zero cells (k, a = M[i][k]) are compacted into
// shared memory in segments of kSeg; for each one, row k of M is read with
// 16-byte coalesced loads and combined cell by cell through a lookup table
// held in shared memory:
//   8-bit cells   T[a][b] = a (x) b for all 256 x 256 pairs (64 KiB),
//   32-bit cells  G[Y][p][v] = { X : X -> Y Z, Z in byte p of b = v } (128 KiB),
//                 a (x) b = OR over Y in a of G[Y][0][b0] | ... | G[Y][3][b3].
// Zero cells of the row (no derivation yet) cost nothing beyond the scan.
// The result row is written back in place: one writer per row, and every
// reader of row i (as a row k of another CTA) sees either the old or the new
// cells, both subsets of the fixpoint (values only gain bits), so an in-place
// pass is sound; the loop ends after a pass that changed no cell, which is
// then a fixpoint of M = M | M (x) M.
#include <type_traits>

#include "launch.h"

namespace cfpq {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kSeg = 4096;  // k-range compacted per round (16 per thread)

struct NtRuleDev {
    uint8_t head, body1, body2, pad;
};

template <class Cell>
struct NtTraits;

template <>
struct NtTraits<uint8_t> {
    static constexpr uint32_t kV = 16;            // cells per 16-byte vector
    static constexpr uint32_t kTableBytes = 65536;  // T[a][b]
};

template <>
struct NtTraits<uint32_t> {
    static constexpr uint32_t kV = 4;
    static constexpr uint32_t kTableBytes = 32 * 4 * 256 * 4;  // G[Y][p][v]
};

// Accumulator row in shared memory; at least 4 KiB, which the table build
// uses as scratch before the first row.
template <class Cell>
__host__ __device__ constexpr size_t ntset_acc_bytes(uint32_t stride) {
    return (size_t)stride * sizeof(Cell) > 4096 ? (size_t)stride * sizeof(Cell) : 4096;
}

template <class Cell>
__host__ __device__ constexpr size_t ntset_smem_bytes(uint32_t stride) {
    return NtTraits<Cell>::kTableBytes + ntset_acc_bytes<Cell>(stride) + kSeg * (2 + sizeof(Cell));
}

// Lookup tables from the rule list (all threads).
__device__ void build_table8(uint8_t *T, const NtRuleDev *rules, uint32_t nrules, uint8_t *scratch) {
    uint8_t *h = scratch;           // h[Y][Z] (8 x 8)
    uint8_t *U = scratch + 64;      // U[Y][b] = OR over Z in b of h[Y][Z] (8 x 256)
    const uint32_t tid = threadIdx.x;
    if (tid < 64) {
        uint8_t v = 0;
        for (uint32_t r = 0; r < nrules; ++r)
            if (rules[r].body1 == tid / 8 && rules[r].body2 == tid % 8) v |= (uint8_t)(1u << rules[r].head);
        h[tid] = v;
    }
    __syncthreads();
    for (uint32_t b = tid; b < 256; b += kThreads)
        for (uint32_t y = 0; y < 8; ++y) {
            uint8_t u = 0;
            for (uint32_t z = 0; z < 8; ++z)
                if ((b >> z) & 1u) u |= h[y * 8 + z];
            U[y * 256 + b] = u;
        }
    __syncthreads();
    for (uint32_t b = tid; b < 256; b += kThreads) {
        T[b] = 0;  // a = 0
        for (uint32_t a = 1; a < 256; ++a) T[a * 256 + b] = T[(a & (a - 1)) * 256 + b] | U[(__ffs(a) - 1) * 256 + b];
    }
    __syncthreads();
}

__device__ void build_table32(uint32_t *G, const NtRuleDev *rules, uint32_t nrules, uint32_t *scratch) {
    uint32_t *h = scratch;  // h[Y][Z] (32 x 32), reuses the accumulator row (not live yet)
    const uint32_t tid = threadIdx.x;
    for (uint32_t e = tid; e < 32 * 32; e += kThreads) {
        uint32_t v = 0;
        for (uint32_t r = 0; r < nrules; ++r)
            if (rules[r].body1 == e / 32 && rules[r].body2 == e % 32) v |= 1u << rules[r].head;
        h[e] = v;
    }
    __syncthreads();
    for (uint32_t e = tid; e < 32 * 4 * 256; e += kThreads) {
        const uint32_t y = e / 1024, p = (e / 256) % 4, v = e % 256;
        uint32_t g = 0;
        for (uint32_t z = 0; z < 8; ++z)
            if ((v >> z) & 1u) g |= h[y * 32 + 8 * p + z];
        G[e] = g;
    }
    __syncthreads();
}

// acc (kV cells in a uint4) |= a (x) b (kV cells in a uint4)
__device__ __forceinline__ void combine(uint4 &acc, uint32_t a, const uint4 &b, const uint8_t *T, uint32_t) {
    const uint8_t *Ta = T + a * 256;
    const uint32_t bw[4] = {b.x, b.y, b.z, b.w};
    uint32_t aw[4] = {0, 0, 0, 0};
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        const uint32_t x = bw[w];
        if (!x) continue;
        aw[w] = (uint32_t)Ta[x & 255] | ((uint32_t)Ta[(x >> 8) & 255] << 8) | ((uint32_t)Ta[(x >> 16) & 255] << 16) |
                ((uint32_t)Ta[x >> 24] << 24);
    }
    acc.x |= aw[0];
    acc.y |= aw[1];
    acc.z |= aw[2];
    acc.w |= aw[3];
}

__device__ __forceinline__ void combine(uint4 &acc, uint32_t a, const uint4 &b, const uint32_t *G, uint32_t ymask) {
    const uint32_t bw[4] = {b.x, b.y, b.z, b.w};
    uint32_t r[4] = {0, 0, 0, 0};
    uint32_t ys = a & ymask;
    while (ys) {
        const uint32_t y = __ffs(ys) - 1;
        ys &= ys - 1;
        const uint32_t *Gy = G + y * 1024;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const uint32_t x = bw[w];
            if (!x) continue;
            r[w] |= Gy[x & 255] | Gy[256 + ((x >> 8) & 255)] | Gy[512 + ((x >> 16) & 255)] | Gy[768 + (x >> 24)];
        }
    }
    acc.x |= r[0];
    acc.y |= r[1];
    acc.z |= r[2];
    acc.w |= r[3];
}

__device__ __forceinline__ bool any_cell(const uint4 &v) { return (v.x | v.y | v.z | v.w) != 0; }

// Cell value of element e (0..kV-1) of a vector.
template <class Cell>
__device__ __forceinline__ uint32_t cell_of(const uint4 &v, uint32_t e) {
    const uint32_t w = e * sizeof(Cell) / 4;
    const uint32_t word = w == 0 ? v.x : w == 1 ? v.y : w == 2 ? v.z : v.w;
    if (sizeof(Cell) == 4) return word;
    return (word >> (8 * (e % 4))) & 0xFFu;
}

template <class Cell>
__global__ void __launch_bounds__(kThreads) k_ntset_square(Cell *__restrict__ M, uint32_t n, uint32_t stride,
                                                         const NtRuleDev *__restrict__ rules, uint32_t nrules,
                                                         uint32_t ymask, uint32_t *counters) {
    using Tr = NtTraits<Cell>;
    constexpr uint32_t kV = Tr::kV;
    extern __shared__ __align__(16) unsigned char smem[];
    using Table = typename std::conditional<sizeof(Cell) == 1, uint8_t, uint32_t>::type;
    Table *tab = reinterpret_cast<Table *>(smem);
    Cell *acc_row = reinterpret_cast<Cell *>(smem + Tr::kTableBytes);
    Cell *list_a = reinterpret_cast<Cell *>(smem + Tr::kTableBytes + ntset_acc_bytes<Cell>(stride));
    uint16_t *list_k = reinterpret_cast<uint16_t *>(reinterpret_cast<unsigned char *>(list_a) + kSeg * sizeof(Cell));
    __shared__ uint32_t s_row, s_cnt, s_wcnt[kThreads / 32];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if constexpr (sizeof(Cell) == 1)
        build_table8(tab, rules, nrules, reinterpret_cast<uint8_t *>(acc_row));
    else
        build_table32(tab, rules, nrules, reinterpret_cast<uint32_t *>(acc_row));
    uint32_t changed = 0;
    const uint32_t vecs = stride / kV;  // 16-byte vectors per row
    for (;;) {
        if (tid == 0) s_row = atomicAdd(&counters[0], 1u);
        __syncthreads();
        const uint32_t i = s_row;
        if (i >= n) break;
        const uint4 *rowi = reinterpret_cast<const uint4 *>(M + (size_t)i * stride);
        for (uint32_t v = tid; v < vecs; v += kThreads) reinterpret_cast<uint4 *>(acc_row)[v] = make_uint4(0, 0, 0, 0);
        for (uint32_t k0 = 0; k0 < n; k0 += kSeg) {
            // compact the non-zero cells of row i in [k0, k0 + kSeg): thread
            // t scans kSeg / kThreads consecutive cells
            constexpr uint32_t kPer = kSeg / kThreads;
            constexpr uint32_t kVecs = kPer / kV;  // vectors per thread (1 or 4)
            Cell cells[kPer];
            uint32_t cnt = 0;
#pragma unroll
            for (uint32_t q = 0; q < kVecs; ++q) {
                const uint32_t vi = (k0 + tid * kPer) / kV + q;
                const uint4 x = vi < vecs ? __ldcg(rowi + vi) : make_uint4(0, 0, 0, 0);
#pragma unroll
                for (uint32_t e = 0; e < kV; ++e) {
                    const uint32_t c = cell_of<Cell>(x, e);
                    cells[q * kV + e] = (Cell)c;
                    cnt += c != 0;
                }
            }
            uint32_t pre = cnt;  // inclusive scan over the warp, then over warps
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, pre, o);
                if (lane >= (uint32_t)o) pre += t;
            }
            if (lane == 31) s_wcnt[warp] = pre;
            __syncthreads();
            uint32_t base = pre - cnt, total = 0;
            for (uint32_t w = 0; w < kThreads / 32; ++w) {
                if (w < warp) base += s_wcnt[w];
                total += s_wcnt[w];
            }
#pragma unroll
            for (uint32_t e = 0; e < kPer; ++e) {
                const uint32_t k = k0 + tid * kPer + e;
                if (cells[e] && k < n) {
                    list_a[base] = cells[e];
                    list_k[base] = (uint16_t)k;
                    ++base;
                }
            }
            if (tid == 0) s_cnt = total;
            __syncthreads();
            const uint32_t m = s_cnt;
            // combine: thread owns vectors v = tid, tid + kThreads, ... of the row
            for (uint32_t v = tid; v < vecs && m; v += kThreads) {
                uint4 acc = reinterpret_cast<const uint4 *>(acc_row)[v];
#pragma unroll 4
                for (uint32_t e = 0; e < m; ++e) {
                    const uint4 b = __ldcg(reinterpret_cast<const uint4 *>(M + (size_t)list_k[e] * stride) + v);
                    if (any_cell(b)) combine(acc, (uint32_t)list_a[e], b, tab, ymask);
                }
                reinterpret_cast<uint4 *>(acc_row)[v] = acc;
            }
            __syncthreads();  // lists reused by the next segment
        }
        // merge into row i (single writer); cells only gain bits
        for (uint32_t v = tid; v < vecs; v += kThreads) {
            const uint4 a = reinterpret_cast<const uint4 *>(acc_row)[v];
            if (!any_cell(a)) continue;
            const uint4 old = __ldcg(rowi + v);
            const uint4 nw = make_uint4(old.x | a.x, old.y | a.y, old.z | a.z, old.w | a.w);
            if (nw.x != old.x || nw.y != old.y || nw.z != old.z || nw.w != old.w) {
                __stcg(const_cast<uint4 *>(rowi) + v, nw);
                changed = 1;
            }
        }
        __syncthreads();  // acc_row and s_row reuse
    }
    if (__syncthreads_or(changed) && tid == 0) atomicOr(&counters[1], 1u);
}

// Pack: cell (i, j) bit x = bit (i, j) of matrix x.  One thread per
// (row, 16-byte vector of cells); the cells of a vector lie in one tile.
template <class Cell>
__global__ void k_ntset_pack(Cell *__restrict__ M, uint32_t stride, const DevMat *__restrict__ mats, uint32_t nm) {
    constexpr uint32_t kV = NtTraits<Cell>::kV;
    const uint32_t vecs = stride / kV;
    const size_t total = (size_t)stride * vecs;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(g / vecs), v = (uint32_t)(g % vecs);
        const uint32_t c0 = v * kV, ti = i >> 6, r = i & 63, tj = c0 >> 6, sh = c0 & 63;
        uint32_t w[4] = {0, 0, 0, 0};
        for (uint32_t x = 0; x < nm; ++x) {
            const DevMat &m = mats[x];
            if (!((m.occ[(size_t)ti * m.ow + (tj >> 5)] >> (tj & 31)) & 1u)) continue;
            uint32_t bits = (uint32_t)((m.bits[tile_offset(m.T, ti, tj) + r] >> sh) & ((1ull << kV) - 1));
            while (bits) {
                const uint32_t e = __ffs(bits) - 1;
                bits &= bits - 1;
                if (sizeof(Cell) == 1)
                    w[e / 4] |= (1u << x) << (8 * (e % 4));
                else
                    w[e] |= 1u << x;
            }
        }
        reinterpret_cast<uint4 *>(M)[g] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Unpack: bit (i, j) of matrix x = bit x of cell (i, j), for the whole
// matrix (tile populations and occupancy are rebuilt afterwards).  One
// thread per (row, tile).
template <class Cell>
__global__ void k_ntset_unpack(const Cell *__restrict__ M, uint32_t stride, const DevMat *__restrict__ mats,
                               uint32_t nm) {
    constexpr uint32_t kV = NtTraits<Cell>::kV;
    const uint32_t T = stride / 64;
    const size_t total = (size_t)stride * T;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(g / T), tj = (uint32_t)(g % T);
        const uint4 *src = reinterpret_cast<const uint4 *>(M + (size_t)i * stride + (size_t)tj * 64);
        uint64_t words[32];
#pragma unroll
        for (uint32_t x = 0; x < 32; ++x) words[x] = 0;
        for (uint32_t q = 0; q < 64 / kV; ++q) {
            const uint4 vv = __ldcg(src + q);
            if (!any_cell(vv)) continue;
            for (uint32_t e = 0; e < kV; ++e) {
                uint32_t c = cell_of<Cell>(vv, e);
                while (c) {
                    const uint32_t x = __ffs(c) - 1;
                    c &= c - 1;
#pragma unroll
                    for (uint32_t y = 0; y < 32; ++y)
                        if (y == x) words[y] |= 1ull << (q * kV + e);
                }
            }
        }
        const uint32_t ti = i >> 6, r = i & 63;
        for (uint32_t x = 0; x < nm; ++x) {
            uint64_t wx = 0;
#pragma unroll
            for (uint32_t y = 0; y < 32; ++y)
                if (y == x) wx = words[y];
            mats[x].bits[tile_offset(mats[x].T, ti, tj) + r] = wx;
        }
    }
}

template <class Cell>
cudaError_t set_smem(uint32_t stride) {
    return cudaFuncSetAttribute(k_ntset_square<Cell>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ntset_smem_bytes<Cell>(stride));
}

}  // namespace

size_t ntset_cell_bytes(uint32_t nmats) { return nmats <= 8 ? 1 : 4; }

cudaError_t launch_ntset_pack(void *cells, uint32_t stride, uint32_t nmats, const DevMat *d_mats, int num_sms,
                              cudaStream_t s) {
    const unsigned grid = (unsigned)num_sms * 8;
    if (ntset_cell_bytes(nmats) == 1)
        k_ntset_pack<uint8_t><<<grid, 256, 0, s>>>(static_cast<uint8_t *>(cells), stride, d_mats, nmats);
    else
        k_ntset_pack<uint32_t><<<grid, 256, 0, s>>>(static_cast<uint32_t *>(cells), stride, d_mats, nmats);
    return cudaGetLastError();
}

cudaError_t launch_ntset_unpack(const void *cells, uint32_t stride, uint32_t nmats, const DevMat *d_mats, int num_sms,
                                cudaStream_t s) {
    const unsigned grid = (unsigned)num_sms * 8;
    if (ntset_cell_bytes(nmats) == 1)
        k_ntset_unpack<uint8_t><<<grid, 256, 0, s>>>(static_cast<const uint8_t *>(cells), stride, d_mats, nmats);
    else
        k_ntset_unpack<uint32_t><<<grid, 256, 0, s>>>(static_cast<const uint32_t *>(cells), stride, d_mats, nmats);
    return cudaGetLastError();
}

// One squaring pass; counters[0] (row counter) and counters[1] (changed flag)
// must be zero before the launch.
cudaError_t launch_ntset_square(void *cells, uint32_t n, uint32_t stride, uint32_t nmats, const void *d_rules,
                                uint32_t nrules, uint32_t ymask, uint32_t *counters, int num_sms, cudaStream_t s) {
    const NtRuleDev *rules = static_cast<const NtRuleDev *>(d_rules);
    if (ntset_cell_bytes(nmats) == 1) {
        const size_t smem = ntset_smem_bytes<uint8_t>(stride);
        cudaError_t e = set_smem<uint8_t>(stride);
        if (e != cudaSuccess) return e;
        k_ntset_square<uint8_t><<<num_sms * 2, kThreads, smem, s>>>(static_cast<uint8_t *>(cells), n, stride, rules,
                                                                    nrules, ymask, counters);
    } else {
        const size_t smem = ntset_smem_bytes<uint32_t>(stride);
        cudaError_t e = set_smem<uint32_t>(stride);
        if (e != cudaSuccess) return e;
        k_ntset_square<uint32_t><<<num_sms, kThreads, smem, s>>>(static_cast<uint32_t *>(cells), n, stride, rules,
                                                                 nrules, ymask, counters);
    }
    return cudaGetLastError();
}

size_t ntset_max_n(uint32_t nmats) { return nmats <= 8 ? 16384 : 8192; }

}  // namespace cfpq
