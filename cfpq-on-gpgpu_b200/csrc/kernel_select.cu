// Variant selection per rule product and iteration, on the device.
//
// Every iteration of an AUTO closure starts with k_select: one warp per
// product term computes its feature vector from the buffer counters that the
// product epilogues keep exact (no pass over the matrices), then chooses the
// variant that runs the term's work items in this iteration:
//   heuristic  thresholds on tile density found by the autotuner
//              (cfpq_autotune): tensor cores when the term is large enough
//              and both operands have densely populated tiles, Four Russians
//              when enough P tiles are dense, LOP3 otherwise;
//   MLP        a 16-64-64-3 perceptron predicting log-microseconds of LOP3,
//              M4R and TC from the features; its fastest allowed variant is
//              taken when the prediction is confident (every feature inside
//              the training range widened by range_margin, and the best
//              prediction ahead of the second by conf_margin), else the
//              heuristic decides.
// The choice never changes a result bit: every variant computes the same
// exact product.  Each decision can be logged with its features.
//
// Features (all scaled to roughly [0, 1]):
//   0 log2 n / 17            1 term (0: dA*B, 1: A*dB)
//   2 P occupied-tile frac   3 Q occupied-tile frac
//   4 P mean tile population / 4096          5 same for Q
//   6 P dense-tile fraction (population > 96 of occupied)   7 same for Q
//   8 log2(1 + nnz P) / 34   9 log2(1 + nnz Q) / 34
//  10 nnz of the delta operand / nnz of its slot's current matrix
//  11 log2(1 + occP * occQ / T) / 32  (expected tile triples, uniform tiles)
//  12 min(iteration, 64) / 64            13 log2 T / 11       14, 15: 0
#include "launch.h"
#include "select_device.cuh"

namespace cfpq {

namespace {

constexpr unsigned kFull = 0xffffffffu;


// One warp per product: features, decision, log row.
__global__ void k_select(const ProdDesc *__restrict__ prods, uint32_t nprods, const BufCounters *__restrict__ cnts,
                         const IterState *st, const SelectorParams *__restrict__ sp, uint8_t *choice,
                         const uint8_t *__restrict__ tc_ok, SelLogRow *log, uint32_t log_iters) {
    const uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (p >= nprods || !st->active) return;
    const ProdDesc pd = prods[p];
    const uint32_t iter = st->iter;
    float f[kSelFeatures], pred[kSelOutputs] = {0.f, 0.f, 0.f};
    uint32_t flags = 0;
    const uint32_t v = sel::select_product(pd, cnts, iter, sp, tc_ok && tc_ok[p], f, pred, &flags);
    if (lane == 0) {
        choice[p] = (uint8_t)v;
        if (log && iter < log_iters) {
            SelLogRow &r = log[(size_t)iter * nprods + p];
#pragma unroll
            for (int i = 0; i < kSelFeatures; ++i) r.f[i] = f[i];
#pragma unroll
            for (int o = 0; o < kSelOutputs; ++o) r.pred[o] = pred[o];
            r.choice = v | flags;
        }
    }
}

// Buffer counters at closure start: current matrices from their occupancy
// bitmaps and tile populations, deltas zero.  One block per slot.
__global__ void k_counters_init(const MatSlot *__restrict__ slots, BufCounters *cnts) {
    const MatSlot sl = slots[blockIdx.x];
    const DevMat m = sl.cur;
    unsigned long long nnz = 0;
    uint32_t occ = 0, dense = 0;
    const size_t tiles = (size_t)m.T * m.T, words = (size_t)m.T * m.ow;
    for (size_t i = threadIdx.x; i < tiles; i += blockDim.x) {
        const uint32_t pop = m.nnz[i];
        nnz += pop;
        dense += pop > kDenseTilePop;
    }
    for (size_t i = threadIdx.x; i < words; i += blockDim.x) occ += __popc(m.occ[i]);
    __shared__ unsigned long long s_nnz[32];
    __shared__ uint32_t s_occ[32], s_dense[32];
    for (int d = 16; d > 0; d >>= 1) {
        nnz += __shfl_xor_sync(kFull, nnz, d);
        occ += __shfl_xor_sync(kFull, occ, d);
        dense += __shfl_xor_sync(kFull, dense, d);
    }
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0) {
        s_nnz[warp] = nnz;
        s_occ[warp] = occ;
        s_dense[warp] = dense;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        BufCounters c = {0, 0, 0};
        for (uint32_t w = 0; w < nw; ++w) {
            c.nnz += s_nnz[w];
            c.occ_tiles += s_occ[w];
            c.dense_tiles += s_dense[w];
        }
        cnts[3 * blockIdx.x] = c;
        cnts[3 * blockIdx.x + 1] = BufCounters{0, 0, 0};
        cnts[3 * blockIdx.x + 2] = BufCounters{0, 0, 0};
    }
}

__global__ void k_fill_choice(uint8_t *choice, uint32_t n, uint8_t v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) choice[i] = v;
}

}  // namespace

cudaError_t launch_select(const ProdDesc *d_prods, uint32_t nprods, const BufCounters *d_cnts, const IterState *d_st,
                          const SelectorParams *d_params, uint8_t *d_choice, const uint8_t *d_tc_ok,
                          SelLogRow *d_log, uint32_t log_iters, cudaStream_t s) {
    if (nprods == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)(((size_t)nprods * 32 + 127) / 128);
    k_select<<<blocks, 128, 0, s>>>(d_prods, nprods, d_cnts, d_st, d_params, d_choice, d_tc_ok, d_log, log_iters);
    return cudaGetLastError();
}

cudaError_t launch_counters_init(const MatSlot *d_slots, uint32_t nslots, BufCounters *d_cnts, cudaStream_t s) {
    if (nslots == 0) return cudaSuccess;
    k_counters_init<<<nslots, 256, 0, s>>>(d_slots, d_cnts);
    return cudaGetLastError();
}

cudaError_t launch_fill_choice(uint8_t *d_choice, uint32_t n, uint8_t v, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_fill_choice<<<(n + 255) / 256, 256, 0, s>>>(d_choice, n, v);
    return cudaGetLastError();
}

}  // namespace cfpq
