// Variant selection of one product term (one warp), shared by the select
// kernel (kernel_select.cu) and the persistent closure kernel.  The selection
// rules and the feature vector are described in kernel_select.cu.
#pragma once

#include "common.cuh"

namespace cfpq {
namespace sel {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t operand_buffer(uint32_t slot, uint8_t use_delta, uint32_t iter) {
    return 3 * slot + ((!use_delta || iter == 0) ? 0u : 1u + (iter & 1));
}

__device__ __forceinline__ void product_features(const ProdDesc &pd, const BufCounters *cnts, uint32_t iter, float *f) {
    const BufCounters P = cnts[operand_buffer(pd.pslot, pd.p_delta, iter)];
    const BufCounters Q = cnts[operand_buffer(pd.qslot, pd.q_delta, iter)];
    const float T = (float)pd.T, T2 = T * T;
    const float occP = (float)P.occ_tiles, occQ = (float)Q.occ_tiles;
    f[0] = log2f((float)pd.n) / 17.f;
    f[1] = (float)pd.term;
    f[2] = occP / T2;
    f[3] = occQ / T2;
    f[4] = occP > 0 ? (float)P.nnz / (occP * 4096.f) : 0.f;
    f[5] = occQ > 0 ? (float)Q.nnz / (occQ * 4096.f) : 0.f;
    f[6] = occP > 0 ? (float)P.dense_tiles / occP : 0.f;
    f[7] = occQ > 0 ? (float)Q.dense_tiles / occQ : 0.f;
    f[8] = log2f(1.f + (float)P.nnz) / 34.f;
    f[9] = log2f(1.f + (float)Q.nnz) / 34.f;
    if (iter == 0) {
        f[10] = 1.f;
    } else {
        const uint32_t slot = pd.term == 0 ? pd.pslot : pd.qslot;
        const BufCounters &dl = pd.term == 0 ? P : Q;
        const float cur = (float)cnts[3 * slot].nnz;
        f[10] = cur > 0 ? fminf(1.f, (float)dl.nnz / cur) : 0.f;
    }
    f[11] = log2f(1.f + occP * occQ / fmaxf(T, 1.f)) / 32.f;
    f[12] = fminf((float)iter, 64.f) / 64.f;
    f[13] = log2f(fmaxf(T, 1.f)) / 11.f;
    f[14] = 0.f;
    f[15] = 0.f;
}

__device__ __forceinline__ uint32_t heuristic_choice(const SelectorParams &sp, const float *f, uint32_t T, bool tc_ok) {
    const uint32_t allowed = sp.allowed;
    // tensor cores: a k-tile costs them the same whatever the tiles hold, so
    // they win where the word-level kernels pay full tiles too -- dense P
    // tiles, whose cost does not depend on Q's population or occupancy --
    // and the product is not tiny
    if (tc_ok && (allowed & (1u << 4)) && T >= sp.tc_min_tiles && f[2] >= sp.tc_min_occ && f[6] >= sp.tc_min_dense)
        return 4;
    if ((allowed & (1u << 3)) && f[6] >= sp.m4r_min_dense) return 3;
    if (allowed & (1u << 2)) return 2;
    return (allowed & (1u << 3)) ? 3u : 2u;
}

// MLP forward for one feature vector, one warp (lane l owns hidden units l and
// l + 32).  out[o] = predicted log-microseconds of variant 2 + o.  All lanes
// get the outputs.
__device__ __forceinline__ void selector_mlp_warp(const float *w, const float *x, float *out) {
    const uint32_t lane = threadIdx.x & 31;
    const float *W1 = w, *b1 = W1 + kSelFeatures * kSelHidden;
    const float *W2 = b1 + kSelHidden, *b2 = W2 + kSelHidden * kSelHidden;
    const float *W3 = b2 + kSelHidden, *b3 = W3 + kSelHidden * kSelOutputs;
    float h1[2], h2[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const uint32_t u = lane + 32 * s;
        float a = b1[u];
#pragma unroll
        for (int i = 0; i < kSelFeatures; ++i) a = fmaf(W1[i * kSelHidden + u], x[i], a);
        h1[s] = fmaxf(a, 0.f);
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) h2[s] = b2[lane + 32 * s];
    for (int k = 0; k < kSelHidden; ++k) {
        const float hk = __shfl_sync(kFull, k < 32 ? h1[0] : h1[1], k & 31);
#pragma unroll
        for (int s = 0; s < 2; ++s) h2[s] = fmaf(W2[k * kSelHidden + lane + 32 * s], hk, h2[s]);
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) h2[s] = fmaxf(h2[s], 0.f);
#pragma unroll
    for (int o = 0; o < kSelOutputs; ++o) {
        float p = W3[lane * kSelOutputs + o] * h2[0] + W3[(lane + 32) * kSelOutputs + o] * h2[1];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) p += __shfl_xor_sync(kFull, p, d);
        out[o] = p + b3[o];
    }
}

// Decide the variant of product p (all lanes of one warp; every lane gets the
// result).  tc_ok: the term has a tensor-core launch sequence.
__device__ __forceinline__ uint32_t select_product(const ProdDesc &pd, const BufCounters *cnts, uint32_t iter,
                                                   const SelectorParams *sp, bool tcp, float *f, float *pred,
                                                   uint32_t *flags_out) {
    product_features(pd, cnts, iter, f);
    uint32_t v = heuristic_choice(*sp, f, pd.T, tcp);
    uint32_t flags = 0;
    if (sp->mode == 2 && sp->has_weights) {
        selector_mlp_warp(sp->w, f, pred);
        bool in_range = true;
#pragma unroll
        for (int i = 0; i < kSelFeatures; ++i) {
            const float span = sp->feat_hi[i] - sp->feat_lo[i];
            const float m = sp->range_margin * fmaxf(span, 1e-3f);
            in_range = in_range && f[i] >= sp->feat_lo[i] - m && f[i] <= sp->feat_hi[i] + m;
        }
        uint32_t best = 0xFFu;
        float b1 = 3.0e38f, b2 = 3.0e38f;
#pragma unroll
        for (int o = 0; o < kSelOutputs; ++o) {
            const uint32_t var = 2 + o;
            if (!(sp->allowed & (1u << var)) || (var == 4 && (!tcp || pd.T < sp->tc_min_tiles))) continue;
            if (pred[o] < b1) {
                b2 = b1;
                b1 = pred[o];
                best = var;
            } else if (pred[o] < b2) {
                b2 = pred[o];
            }
        }
        const bool confident = in_range && best != 0xFFu && (b2 - b1 >= sp->conf_margin || b2 > 1.0e38f);
        if (confident) {
            v = best;
            flags = 1u << 8;
        } else {
            flags = 1u << 9;
        }
    }
    *flags_out = flags;
    return v;
}

}  // namespace sel
}  // namespace cfpq
