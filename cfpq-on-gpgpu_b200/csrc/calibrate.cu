// cfpq_calibrate: measured LOP3-pipe rate (the denominator of the word-level
// product rooflines).  Eight independent chains per thread of
// `a |= (q ^ b) & m` (two 3-input logic instructions each), all operands in
// registers, grid = 8 CTAs of 256 threads per SM; the result of every thread
// is stored so nothing is eliminated.
#include <cstring>

#include "cfpq_b200.h"
#include "launch.h"

namespace cfpq {
namespace {

__global__ void __launch_bounds__(256) k_logic_rate(uint32_t *out, int iters, uint32_t seed) {
    uint32_t a0 = seed ^ threadIdx.x, a1 = a0 * 3, a2 = a0 * 5, a3 = a0 * 7, a4 = a0 * 11, a5 = a0 * 13,
             a6 = a0 * 17, a7 = a0 * 19;
    const uint32_t m = seed * 0x9e3779b9u, q = seed + 0x12345u;
#pragma unroll 1
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            a0 |= (q ^ a1) & m;
            a1 |= (q ^ a2) & m;
            a2 |= (q ^ a3) & m;
            a3 |= (q ^ a4) & m;
            a4 |= (q ^ a5) & m;
            a5 |= (q ^ a6) & m;
            a6 |= (q ^ a7) & m;
            a7 |= (q ^ a0) & m;
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
}

}  // namespace

cudaError_t measure_logic_rate(int num_sms, uint32_t *d_out, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1,
                               double *ops_per_s, double *ms_out) {
    const int threads = 256, blocks = num_sms * 8, iters = 2048;
    k_logic_rate<<<blocks, threads, 0, s>>>(d_out, 64, 1);  // warm-up
    cudaEventRecord(e0, s);
    k_logic_rate<<<blocks, threads, 0, s>>>(d_out, iters, 7);
    cudaEventRecord(e1, s);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) return e;
    float ms = 0;
    e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) return e;
    const double ops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    *ops_per_s = ops / (ms * 1e-3);
    *ms_out = ms;
    return cudaGetLastError();
}

}  // namespace cfpq
