// Operand expansion for the tensor-core variant: a bit matrix becomes 0/1
// bytes, already in the canonical no-swizzle K-major layout that tcgen05.mma
// reads, one 4 KiB block per 64 x 64 tile so that a 1-D bulk copy of a block
// lands in shared memory ready for the MMA.
//
// Block of tile (ti, tj) at byte ((ti*T + tj) * 4096); inside, operand row r
// (0..63) and 16-byte k-chunk kg (0..3) at ((r/8)*4 + kg)*128 + (r%8)*16.
//   rows: operand row r = matrix row ti*64 + r, k = matrix column (the P side)
//   cols: operand row r = matrix column tj*64 + r, k = matrix row (the Q side,
//         transposed: a warp transposes the 64 x 64 bit tile in registers)
#include "launch.h"

namespace cfpq {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint4 expand16(uint32_t x) {
    uint4 v;  // byte i = bit i ((nibble * 0x00204081) & 0x01010101 spreads 4 bits to 4 bytes)
    v.x = ((x & 15u) * 0x00204081u) & 0x01010101u;
    v.y = (((x >> 4) & 15u) * 0x00204081u) & 0x01010101u;
    v.z = (((x >> 8) & 15u) * 0x00204081u) & 0x01010101u;
    v.w = (((x >> 12) & 15u) * 0x00204081u) & 0x01010101u;
    return v;
}

__device__ __forceinline__ void store_row(uint8_t *block, uint32_t r, uint64_t bits) {
    uint8_t *base = block + (r >> 3) * 512 + (r & 7) * 16;
#pragma unroll
    for (int kg = 0; kg < 4; ++kg)
        *reinterpret_cast<uint4 *>(base + kg * 128) = expand16((uint32_t)(bits >> (16 * kg)) & 0xFFFFu);
}

// Lane l holds rows l (lo) and l+32 (hi) of a 64 x 64 bit tile; afterwards it
// holds columns l and l+32 as bit rows (bit r = original row r).  Exchange
// stages j = 32 .. 1: rows k (bit j clear) and k|j swap the off-diagonal
// j x j blocks, t = ((A[k] >> j) ^ A[k|j]) & m_j.
__device__ __forceinline__ void transpose64(uint64_t &lo, uint64_t &hi, uint32_t lane) {
    {
        const uint64_t t = ((lo >> 32) ^ hi) & 0x00000000FFFFFFFFULL;
        lo ^= t << 32;
        hi ^= t;
    }
#pragma unroll
    for (int j = 16; j >= 1; j >>= 1) {
        const uint64_t m = j == 16 ? 0x0000FFFF0000FFFFULL
                         : j == 8  ? 0x00FF00FF00FF00FFULL
                         : j == 4  ? 0x0F0F0F0F0F0F0F0FULL
                         : j == 2  ? 0x3333333333333333ULL
                                   : 0x5555555555555555ULL;
        const bool low = (lane & j) == 0;
        const uint64_t plo = __shfl_xor_sync(kFull, lo, j), phi = __shfl_xor_sync(kFull, hi, j);
        const uint64_t tlo = low ? (((lo >> j) ^ plo) & m) : (((plo >> j) ^ lo) & m);
        const uint64_t thi = low ? (((hi >> j) ^ phi) & m) : (((phi >> j) ^ hi) & m);
        lo ^= low ? (tlo << j) : tlo;
        hi ^= low ? (thi << j) : thi;
    }
}

// Expand one operand of product p, resolved on the device like the product
// kernels do (the current matrix or the previous iteration's delta).  One warp
// per tile (grid-stride); lane l writes operand rows l and l+32.
__global__ void __launch_bounds__(256) k_expand_operand(const ProdDesc *__restrict__ prods, uint32_t p,
                                                        const MatSlot *__restrict__ slots, const IterState *st,
                                                        int side, uint8_t *__restrict__ out,
                                                        const uint8_t *__restrict__ choice) {
    if (choice && choice[p] != 4) return;  // this iteration runs the product on the word-level kernels
    const ProdDesc pd = prods[p];
    const uint32_t iter = st->iter;
    if (!st->active || (pd.term == 1 && iter == 0)) return;  // the plan emits nothing for this product
    const MatSlot &sl = slots[side == 0 ? pd.pslot : pd.qslot];
    const uint8_t use_delta = side == 0 ? pd.p_delta : pd.q_delta;
    const DevMat m = (!use_delta || iter == 0) ? sl.cur : sl.dlt[iter & 1];
    const uint32_t lane = threadIdx.x & 31;
    const size_t tiles = (size_t)m.T * m.T;
    for (size_t t = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5; t < tiles;
         t += ((size_t)gridDim.x * blockDim.x) >> 5) {
        uint64_t lo = m.bits[t * 64 + lane], hi = m.bits[t * 64 + lane + 32];
        if (side == 1) transpose64(lo, hi, lane);
        uint8_t *block = out + t * 4096;
        store_row(block, lane, lo);
        store_row(block, lane + 32, hi);
    }
}

__global__ void k_reset_list(IterState *st, int list) {
    st->items_total += st->item_count[list];
    st->items_by_variant[4] += st->item_count[list];
    st->item_count[list] = 0;
    st->item_next[list] = 0;
}

}  // namespace

cudaError_t launch_expand_operand(const ProdDesc *d_prods, uint32_t p, uint32_t T, const MatSlot *d_slots,
                                  const IterState *d_st, int side, uint8_t *out, int num_sms,
                                  const uint8_t *d_choice, cudaStream_t s) {
    if (T == 0) return cudaSuccess;
    size_t blocks = ((size_t)T * T + 7) / 8;
    const size_t cap = (size_t)num_sms * 16;
    if (blocks > cap) blocks = cap;
    k_expand_operand<<<(unsigned)blocks, 256, 0, s>>>(d_prods, p, d_slots, d_st, side, out, d_choice);
    return cudaGetLastError();
}

cudaError_t launch_reset_list(IterState *st, int list, cudaStream_t s) {
    k_reset_list<<<1, 1, 0, s>>>(st, list);
    return cudaGetLastError();
}

}  // namespace cfpq
