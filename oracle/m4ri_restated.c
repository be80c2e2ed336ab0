/*
 * TEST INFRASTRUCTURE ONLY -- part of the CPU oracle (see m4ri_restated.h).
 *
 * Restated Boolean M4RM product and the libm4ri API subset used by the
 * reference CPU backend (m4ri/m4ri_matrix.cpp:8-28).  OpenMP-parallel like the
 * reference's --enable-openmp libm4ri build (Dockerfile:17).
 */
#include "m4ri_restated.h"
#include "m4ri_shim/m4ri/m4ri.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define M4RM_K 8         /* slab width in bits: one table has 2^8 entries */
#define M4RM_SLABS 8     /* 8 slabs of 8 bits cover one 64-bit word of A */
#define M4RM_CBW 32      /* column block in words (2048 columns) so that the  */
                         /* 8 tables (8 x 256 x 32 words = 512 KiB) stay in L2 */

static int resolve_threads(int threads) {
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

void orc_m4rm_product_or(int n, int wpr, const uint64_t *A, const uint64_t *B,
                         uint64_t *out, int threads) {
    if (n <= 0 || wpr <= 0) return;
    const int nt = resolve_threads(threads);
    const int cbw = wpr < M4RM_CBW ? wpr : M4RM_CBW;
    uint64_t *tables = (uint64_t *)malloc((size_t)M4RM_SLABS * 256 * cbw * sizeof(uint64_t));
    if (!tables) {
        fprintf(stderr, "oracle: out of memory in M4RM tables\n");
        abort();
    }
    for (int c0 = 0; c0 < wpr; c0 += cbw) {
        const int cw = (wpr - c0) < cbw ? (wpr - c0) : cbw;
        for (int kw = 0; kw < wpr; ++kw) {
            const int kbase = kw * 64;
            /* Build the 8 slab tables for inner indices kbase .. kbase+63. */
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int s = 0; s < M4RM_SLABS; ++s) {
                uint64_t *T = tables + (size_t)s * 256 * cw;
                memset(T, 0, (size_t)cw * sizeof(uint64_t));
                for (int x = 1; x < 256; ++x) {
                    const int bit = __builtin_ctz((unsigned)x);
                    const int k = kbase + M4RM_K * s + bit;
                    uint64_t *dst = T + (size_t)x * cw;
                    const uint64_t *prev = T + (size_t)(x & (x - 1)) * cw;
                    if (k < n) {
                        const uint64_t *brow = B + (size_t)k * wpr + c0;
                        for (int w = 0; w < cw; ++w) dst[w] = prev[w] | brow[w];
                    } else {
                        for (int w = 0; w < cw; ++w) dst[w] = prev[w];
                    }
                }
            }
            /* Apply: out[i] |= T_s[byte_s(A[i][kw])] for the 8 slabs. */
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int i = 0; i < n; ++i) {
                const uint64_t a = A[(size_t)i * wpr + kw];
                if (!a) continue;
                uint64_t *o = out + (size_t)i * wpr + c0;
                for (int s = 0; s < M4RM_SLABS; ++s) {
                    const unsigned key = (unsigned)(a >> (M4RM_K * s)) & 0xffu;
                    if (!key) continue;
                    const uint64_t *t = tables + ((size_t)s * 256 + key) * cw;
                    for (int w = 0; w < cw; ++w) o[w] |= t[w];
                }
            }
        }
    }
    free(tables);
}

void orc_naive_product_or(int n, int wpr, const uint64_t *A, const uint64_t *B,
                          uint64_t *out, int threads) {
    if (n <= 0 || wpr <= 0) return;
    const int nt = resolve_threads(threads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        uint64_t *o = out + (size_t)i * wpr;
        for (int kw = 0; kw < wpr; ++kw) {
            uint64_t a = A[(size_t)i * wpr + kw];
            while (a) {
                const int k = kw * 64 + __builtin_ctzll(a);
                a &= a - 1;
                const uint64_t *b = B + (size_t)k * wpr;
                for (int w = 0; w < wpr; ++w) o[w] |= b[w];
            }
        }
    }
}

/* ---------------- libm4ri API subset (restated) ---------------- */

mzd_t *mzd_init(rci_t r, rci_t c) {
    mzd_t *M = (mzd_t *)calloc(1, sizeof(mzd_t));
    if (!M) abort();
    M->nrows = r;
    M->ncols = c;
    M->width = (c + 63) / 64;
    const size_t words = (size_t)r * (size_t)M->width;
    M->data = (word *)calloc(words ? words : 1, sizeof(word));
    if (!M->data) abort();
    return M;
}

void mzd_free(mzd_t *A) {
    if (!A) return;
    free(A->data);
    free(A);
}

void mzd_write_bit(mzd_t *M, rci_t row, rci_t col, BIT value) {
    word *w = M->data + (size_t)row * M->width + col / 64;
    const word mask = (word)1 << (col % 64);
    if (value)
        *w |= mask;
    else
        *w &= ~mask;
}

BIT mzd_read_bit(const mzd_t *M, rci_t row, rci_t col) {
    return (BIT)((M->data[(size_t)row * M->width + col / 64] >> (col % 64)) & 1u);
}

mzd_t *mzd_copy(mzd_t *N, const mzd_t *A) {
    if (N == A) return N;
    if (!N) N = mzd_init(A->nrows, A->ncols);
    memcpy(N->data, A->data, (size_t)A->nrows * A->width * sizeof(word));
    return N;
}

int mzd_equal(const mzd_t *A, const mzd_t *B) {
    if (A->nrows != B->nrows || A->ncols != B->ncols) return 0;
    return memcmp(A->data, B->data, (size_t)A->nrows * A->width * sizeof(word)) == 0;
}

mzd_t *mzd_sr_addmul_m4rm(mzd_t *C, const mzd_t *A, const mzd_t *B, int k) {
    (void)k; /* slab width fixed at 8 bits */
    if (A->nrows != C->nrows || B->ncols != C->ncols || A->ncols != B->nrows ||
        C->nrows != C->ncols) {
        fprintf(stderr, "mzd_sr_addmul_m4rm: only square, equally sized operands are supported\n");
        abort();
    }
    const int n = C->nrows;
    const int wpr = C->width;
    if (C == A || C == B) {
        /* Snapshot semantics when the result aliases an operand. */
        mzd_t *T = mzd_init(n, n);
        orc_m4rm_product_or(n, wpr, A->data, B->data, T->data, 0);
        const size_t words = (size_t)n * wpr;
        for (size_t i = 0; i < words; ++i) C->data[i] |= T->data[i];
        mzd_free(T);
    } else {
        orc_m4rm_product_or(n, wpr, A->data, B->data, C->data, 0);
    }
    return C;
}
