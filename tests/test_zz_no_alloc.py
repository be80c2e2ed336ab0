"""cfpq_hash_count_rows_noalloc: the allocation-free result hash.

This entry point serves callers that cannot call cudaMalloc (their own pool
allocator owns the device memory, or they cannot take the synchronisation an
allocation may cause).  They keep the answer matrix in their own device
memory; the library computes the reference result line (hash, count) with
scratch memory from a fixed device array instead of allocating.  The test
checks it through the C ABI against the allocating entry point
(cfpq_matrix_hash_count) on calls in a row, so that the later calls prove
the shared scratch array is re-initialised; with random bits left in the
columns beyond n (they must be ignored), on the default and on another
stream, for n = 0, and checks the size limit.
It lives in its own file so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(rng, n, density):
    wpr = (n + 63) // 64
    bits = rng.random((n, wpr * 64)) < density
    bits[:, n:] = False
    return np.packbits(bits, axis=1, bitorder="little").view(np.uint64).reshape(n, wpr).copy()


def _garbage_tail(rng, rows, n):
    """The same rows with random bits in the columns >= n of the last word,
    which the entry point must ignore (callers may leave them uninitialised)."""
    out = rows.copy()
    if n % 64:
        tail = rng.integers(0, 2**63, size=rows.shape[0], dtype=np.uint64) << np.uint64(n % 64)
        out[:, -1] |= tail
    return out


def test_noalloc_hash_matches_allocating_entry_point(pkg):
    torch = pytest.importorskip("torch")
    lib = pkg.capi.load_library()
    fn = lib.cfpq_hash_count_rows_noalloc
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    lib.cfpq_noalloc_last_error.restype = ctypes.c_char_p
    rng = np.random.default_rng(2024)
    with pkg.capi.Context(0) as ctx:
        side = torch.cuda.Stream()
        cases = [(700, 0.2, False), (300, 0.01, True), (64, 1.0, False), (1, 1.0, True), (130, 0.5, True)]
        for n, density, on_side in cases:  # consecutive calls share the library's scratch array
            rows = _rows(rng, n, density)
            m = ctx.matrix(n)
            m.upload_rows(rows)
            expected = m.hash_count()
            m.destroy()
            d_rows = torch.from_numpy(_garbage_tail(rng, rows, n).view(np.int64)).cuda()
            d_out = torch.full((2,), -1, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            stream = (side if on_side else torch.cuda.current_stream()).cuda_stream
            rc = fn(0, ctypes.c_void_p(d_rows.data_ptr()), n, ctypes.c_void_p(d_out.data_ptr()),
                    ctypes.c_void_p(stream))
            assert rc == 0, lib.cfpq_noalloc_last_error().decode()
            torch.cuda.synchronize()
            got = tuple(int(x) for x in d_out.cpu().numpy().view(np.uint64))
            assert got == expected, (n, density, on_side)
        # n = 0: the empty matrix hashes to (0, 0); no row pointer is needed
        d_out = torch.full((2,), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        assert fn(0, None, 0, ctypes.c_void_p(d_out.data_ptr()), None) == 0, lib.cfpq_noalloc_last_error()
        torch.cuda.synchronize()
        assert d_out.cpu().tolist() == [0, 0]
        # sizes above the fixed scratch capacity are rejected, nothing is launched
        d_out = torch.zeros(2, dtype=torch.int64, device="cuda")
        rc = fn(0, ctypes.c_void_p(d_out.data_ptr()), 65537, ctypes.c_void_p(d_out.data_ptr()), None)
        assert rc == pkg.capi.ERR_UNSUPPORTED
        assert b"65536" in lib.cfpq_noalloc_last_error()
