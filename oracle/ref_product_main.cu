// TEST INFRASTRUCTURE ONLY -- times single rule products of the reference's
// naive GPU backend: gpu_lib::matrix_product_add_wrapper
// (cuda/naive-gpu/Multiplication.cu:145-166), linked from the reference's own
// Multiplication.cu (oracle/Makefile, target naiveGPU-product).  Used by the
// benchmark to give the reference's per-product time at sizes where its whole
// closure would take hours.  Nothing of the product path uses it.
//
//   naiveGPU-product N LOG2_INV_DENSITY REPS SEED
//
// A and B are random N x N bit matrices in the backend's own layout (words of
// 32 row bits, column strips; cuda/naive-gpu/GpuMatrix.cpp:15-18) in which
// each bit is set with probability 2^-LOG2_INV_DENSITY (the AND of that many
// random words; 1 gives 0.5).  Prints one line: "ms_per_product <t>", the
// mean wall time of REPS calls of the wrapper (each ends with the backend's
// own device synchronisation and flag read), after one untimed call.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "Multiplication.h"

static uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int main(int argc, char **argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s N LOG2_INV_DENSITY REPS SEED\n", argv[0]);
        return 2;
    }
    const int N = std::atoi(argv[1]), m = std::atoi(argv[2]), reps = std::atoi(argv[3]);
    uint64_t seed = std::strtoull(argv[4], nullptr, 10);
    if (N <= 0 || N % 32 != 0 || m < 1 || reps < 1) {
        std::fprintf(stderr, "N must be a positive multiple of 32, LOG2_INV_DENSITY and REPS >= 1\n");
        return 2;
    }
    const size_t words = (size_t)gpu_lib::rows(N) * gpu_lib::cols(N);
    TYPE *h[2];
    TYPE *d[4];
    for (int k = 0; k < 2; ++k) {
        h[k] = gpu_lib::host_matrix_calloc(N);
        for (size_t i = 0; i < words; i += 2) {
            uint64_t w = ~0ull;
            for (int j = 0; j < m; ++j) w &= splitmix(seed);
            h[k][i] = (TYPE)w;
            if (i + 1 < words) h[k][i + 1] = (TYPE)(w >> 32);
        }
    }
    for (int k = 0; k < 4; ++k) d[k] = gpu_lib::device_matrix_alloc(N);
    gpu_lib::cpu_to_gpu_transfer_async(N, h[0], d[0]);
    gpu_lib::cpu_to_gpu_transfer_async(N, h[1], d[1]);
    gpu_lib::synchronize();
    gpu_lib::matrix_product_add_wrapper(d[0], d[1], d[2], N, d[3]);  // warm-up
    const auto t0 = std::chrono::steady_clock::now();
    for (int r = 0; r < reps; ++r) gpu_lib::matrix_product_add_wrapper(d[0], d[1], d[2], N, d[3]);
    const auto t1 = std::chrono::steady_clock::now();
    std::printf("ms_per_product %.3f\n", std::chrono::duration<double, std::milli>(t1 - t0).count() / reps);
    for (int k = 0; k < 4; ++k) gpu_lib::device_matrix_dealloc(d[k]);
    for (int k = 0; k < 2; ++k) gpu_lib::host_matrix_dealloc(h[k]);
    return 0;
}
