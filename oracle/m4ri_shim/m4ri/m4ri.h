/*
 * TEST INFRASTRUCTURE ONLY -- part of the CPU oracle.
 *
 * A restated stand-in for the subset of the libm4ri API that the reference's
 * CPU backend uses (m4ri/m4ri_matrix.h:7-24, m4ri/m4ri_matrix.cpp:8-28):
 *   mzd_init, mzd_free, mzd_write_bit, mzd_read_bit, mzd_copy, mzd_equal and
 *   the fork-specific mzd_sr_addmul_m4rm (Boolean semiring C |= A*B).
 * The real library (bitbucket vkutuev/m4ri fork, unpinned, Dockerfile:15-17)
 * is absent and cannot be installed here, so the oracle build compiles the
 * reference's own m4ri/main.cpp + m4ri/m4ri_matrix.cpp + cfpq-cpp driver
 * against this header.  Semantics follow the call sites; names and signatures
 * follow the public libm4ri API; the implementation is our own (see
 * m4ri_restated.c).
 */
#ifndef CFPQ_ORACLE_M4RI_SHIM_H
#define CFPQ_ORACLE_M4RI_SHIM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int rci_t;     /* row / column index */
typedef int wi_t;      /* word index */
typedef uint64_t word; /* 64-bit limb, column c at bit c % 64 */
typedef int BIT;

typedef struct mzd_t {
    rci_t nrows;
    rci_t ncols;
    wi_t width; /* words per row */
    word *data; /* nrows * width words, row-major */
} mzd_t;

mzd_t *mzd_init(rci_t r, rci_t c);
void mzd_free(mzd_t *A);
void mzd_write_bit(mzd_t *M, rci_t row, rci_t col, BIT value);
BIT mzd_read_bit(const mzd_t *M, rci_t row, rci_t col);
/* Copy of A into N (N == NULL allocates a new matrix). */
mzd_t *mzd_copy(mzd_t *N, const mzd_t *A);
/* Nonzero when A and B hold the same bits. */
int mzd_equal(const mzd_t *A, const mzd_t *B);
/* C := C OR (A * B) over the Boolean semiring (AND, OR); k = 0 picks the
 * slab width.  Returns C. */
mzd_t *mzd_sr_addmul_m4rm(mzd_t *C, const mzd_t *A, const mzd_t *B, int k);

#ifdef __cplusplus
}
#endif

#endif
