// Input phase of a query (Grammar::intersection_with_graph, cfpq-cpp/Grammar.h:41-51):
// clear the query's matrices, scatter the labelled edges into the matrices of
// their terminals' nonterminals, set the diagonals of the epsilon
// nonterminals.  Device helpers of the input kernels (kernels_core.cu), which
// cfpq_intersection enqueues right before the closure's own launches.
#pragma once

#include "common.cuh"

namespace cfpq {

// One query's input, all device pointers.  clear: one unit per (matrix, tile-row), row_start the
// prefix sum of tile-rows; edges: label l sets its bit in the matrices
// lm[off[l] .. off[l+1]) of `mats`; diag: matrices whose diagonal is set.
struct ClosureInput {
    const MatRows *clear;
    uint32_t nclear, clear_rows;
    const DevMat *mats;
    uint32_t nmats, nlabels;
    const uint32_t *from, *label, *to;
    size_t nedges;
    const uint32_t *off, *lm;
    uint32_t nlm;
    uint32_t ndiag;
    const DevMat *diag;
    uint32_t *bad;  // out-of-range vertex ids are counted here (and skipped)
};

#ifdef __CUDACC__

__device__ __forceinline__ void set_occ_bit(const DevMat &m, uint32_t ti, uint32_t tj) {
    atomicOr(m.occ + (size_t)ti * m.ow + (tj >> 5), 1u << (tj & 31));
}

// Set bit (r, c) given in vertex ids (mapped through the matrix's vertex
// order); keep occupancy and population exact.  Only the bit that takes its
// tile's population from 0 sets the occupancy bit (a population above 0
// always has its occupancy bit set): a hub vertex's tile-row gets thousands
// of new bits, and one atomic on its occupancy word per bit serialised them.
__device__ __forceinline__ void set_one_bit(const DevMat &m, uint32_t r, uint32_t c) {
    if (m.perm) {
        r = m.perm[r];
        c = m.perm[c];
    }
    unsigned long long *w =
        reinterpret_cast<unsigned long long *>(m.bits + tile_offset(m.T, r >> 6, c >> 6) + (r & 63));
    const unsigned long long bit = 1ULL << (c & 63);
    const unsigned long long old = atomicOr(w, bit);
    if (!(old & bit) && atomicAdd(m.nnz + (size_t)(r >> 6) * m.T + (c >> 6), 1u) == 0u)
        set_occ_bit(m, r >> 6, c >> 6);
}

// One edge (label l, r -> c) into every matrix of its label; ids out of a
// matrix's range are counted in *bad and skipped.
__device__ __forceinline__ void scatter_edge(const DevMat *mats, const uint32_t *off, const uint32_t *lm,
                                             uint32_t nlabels, uint32_t l, uint32_t r, uint32_t c, uint32_t *bad) {
    if (l >= nlabels) return;
    for (uint32_t j = off[l]; j < off[l + 1]; ++j) {
        const DevMat m = mats[lm[j]];
        if (r >= m.n || c >= m.n) {
            atomicAdd(bad, 1u);
            continue;
        }
        set_one_bit(m, r, c);
    }
}

// Clear unit u (one warp): tile-row u of the concatenated tile-rows of the
// clear list.
__device__ __forceinline__ void clear_unit(const MatRows *tab, uint32_t nmats, uint32_t u) {
    uint32_t lo = 0, hi = nmats;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (tab[mid].row_start <= u) lo = mid; else hi = mid;
    }
    clear_tile_row(tab[lo].m, u - tab[lo].row_start);
}

#endif  // __CUDACC__

}  // namespace cfpq
