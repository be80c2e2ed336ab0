/*
 * TEST INFRASTRUCTURE ONLY -- part of the CPU oracle.
 *
 * Restated Boolean-semiring "Method of Four Russians" (M4RM) product on
 * bit-packed rows.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may link or execute this code, and only as the
 * checker or the timed CPU baseline -- never as the product path.
 *
 * What it restates: the reference's CPU backend calls
 *   m = mzd_sr_addmul_m4rm(m, A->m, B->m, 0)      (m4ri/m4ri_matrix.cpp:24)
 * from a fork of libm4ri (bitbucket vkutuev/m4ri, unpinned HEAD, configured
 * --enable-openmp, Dockerfile:15-17) that is not vendored in the reference and
 * cannot be installed here.  Its contract at the call site is
 * C := C OR (A AND-OR B) over the Boolean semiring, with change detection done
 * by the caller via mzd_copy + mzd_equal (m4ri/m4ri_matrix.cpp:20-28).
 *
 * The algorithm is the published M4RM of Arlazarov, Dinic, Kronrod and
 * Faradzev as described for libm4ri by Albrecht, Bard and Hart (ACM TOMS 37(1),
 * 2010, "Algorithm 898"): split the inner dimension into k-bit slabs, build a
 * 2^k-entry table of all combinations of the slab's k rows of B, and add the
 * table entry indexed by A's k bits of each row into C.  Over the Boolean
 * semiring "add" is OR, so the table entry for index x is the OR of B's slab
 * rows selected by the set bits of x (no Gray code is needed because OR is
 * idempotent; the table is filled in increasing index order from
 * T[x] = T[x & (x-1)] | B[k0 + ctz(x)]).
 *
 * Bit layout (same as libm4ri): row-major, 64-bit words, word c/64 of a row
 * holds column c at bit c%64 (LSB first).
 */
#ifndef CFPQ_ORACLE_M4RI_RESTATED_H
#define CFPQ_ORACLE_M4RI_RESTATED_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* out |= A * B for n x n bit matrices with `wpr` 64-bit words per row.
 * `out` must not alias A or B.  threads <= 0 means "all OpenMP threads". */
void orc_m4rm_product_or(int n, int wpr, const uint64_t *A, const uint64_t *B,
                         uint64_t *out, int threads);

/* out |= A * B by the textbook row-gather definition:
 * out[i] |= OR over k with A[i][k] = 1 of B[k].  Same aliasing rule. */
void orc_naive_product_or(int n, int wpr, const uint64_t *A, const uint64_t *B,
                          uint64_t *out, int threads);

#ifdef __cplusplus
}
#endif

#endif
