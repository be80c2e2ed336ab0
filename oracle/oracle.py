"""TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU oracle (liboracle.so)
and to the reference executables built from the reference sources
(oracle/_ref/).  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg / reference arm may use this module, and only as the checker
or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

NAIVE, M4RM = 0, 1

_lib = None


def build() -> None:
    subprocess.run(["make", "-C", ORACLE_DIR, "-s"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp, i32, u32, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint, ctypes.c_longlong
        P = ctypes.POINTER
        L.orc_load.argtypes, L.orc_load.restype = [ctypes.c_char_p, ctypes.c_char_p], vp
        L.orc_free.argtypes, L.orc_free.restype = [vp], None
        L.orc_num_nonterminals.argtypes, L.orc_num_nonterminals.restype = [vp], i32
        L.orc_vertices.argtypes, L.orc_vertices.restype = [vp], u32
        L.orc_num_rules.argtypes, L.orc_num_rules.restype = [vp], i32
        L.orc_rules.argtypes, L.orc_rules.restype = [vp], P(i32)
        L.orc_nonterminal_name.argtypes, L.orc_nonterminal_name.restype = [vp, i32], ctypes.c_char_p
        L.orc_words_per_row.argtypes, L.orc_words_per_row.restype = [vp], i32
        L.orc_matrix.argtypes, L.orc_matrix.restype = [vp, i32], P(ctypes.c_uint64)
        L.orc_products.argtypes, L.orc_products.restype = [vp], ll
        L.orc_closure.argtypes, L.orc_closure.restype = [vp, i32, i32, P(ctypes.c_double)], i32
        L.orc_write_results.argtypes, L.orc_write_results.restype = [vp, ctypes.c_char_p], i32
        L.orc_add_mul.argtypes, L.orc_add_mul.restype = [i32, vp, vp, vp, i32, i32], i32
        L.orc_hash_count.argtypes, L.orc_hash_count.restype = [i32, vp, P(ctypes.c_uint64), P(ctypes.c_uint64)], None
        L.orc_add_mul_rows.argtypes, L.orc_add_mul_rows.restype = [i32, vp, vp, vp, vp, vp, i32, i32], None
        _lib = L
    return _lib


def _p(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def add_mul(c: np.ndarray, a: np.ndarray, b: np.ndarray, n: int, method: int = NAIVE, threads: int = 0) -> bool:
    """c |= a * b in place on row-bit arrays (n x ceil(n/64) uint64)."""
    for x in (a, b, c):
        assert x.dtype == np.uint64 and x.flags["C_CONTIGUOUS"] and x.size == n * ((n + 63) // 64)
    return bool(lib().orc_add_mul(n, _p(c), _p(a), _p(b), method, threads))


def add_mul_rows(c: np.ndarray, a: np.ndarray, b: np.ndarray, n: int, rows: np.ndarray,
                 threads: int = 0) -> np.ndarray:
    """Rows `rows` of c | a * b (row-bit arrays, n x ceil(n/64) uint64): the
    product checked on a row sample where the whole product is too costly."""
    wpr = (n + 63) // 64
    for x in (a, b, c):
        assert x.dtype == np.uint64 and x.flags["C_CONTIGUOUS"] and x.size == n * wpr
    r = np.ascontiguousarray(rows, dtype=np.uint32)
    assert r.size == 0 or int(r.max()) < n
    out = np.zeros((r.size, wpr), dtype=np.uint64)
    lib().orc_add_mul_rows(n, _p(out), _p(c), _p(a), _p(b), _p(r), int(r.size), threads)
    return out


def hash_count(m: np.ndarray, n: int) -> tuple[int, int]:
    h, c = ctypes.c_uint64(), ctypes.c_uint64()
    lib().orc_hash_count(n, _p(np.ascontiguousarray(m, dtype=np.uint64)), ctypes.byref(h), ctypes.byref(c))
    return int(h.value), int(c.value)


class Problem:
    """A grammar + graph loaded by the oracle; closure on the CPU."""

    def __init__(self, grammar_path: str, graph_path: str):
        self.h = lib().orc_load(grammar_path.encode(), graph_path.encode())
        if not self.h:
            raise FileNotFoundError(f"oracle cannot read {grammar_path} / {graph_path}")
        self.algo_ms = None

    def close(self) -> None:
        if self.h:
            lib().orc_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def n(self) -> int:
        return lib().orc_vertices(self.h)

    @property
    def names(self) -> list[str]:
        return [lib().orc_nonterminal_name(self.h, i).decode() for i in range(lib().orc_num_nonterminals(self.h))]

    @property
    def rules(self) -> list[tuple[int, int, int]]:
        r = lib().orc_rules(self.h)
        return [(r[3 * i], r[3 * i + 1], r[3 * i + 2]) for i in range(lib().orc_num_rules(self.h))]

    def closure(self, method: int = M4RM, threads: int = 0) -> float:
        ms = ctypes.c_double()
        if lib().orc_closure(self.h, method, threads, ctypes.byref(ms)) != 0:
            raise MemoryError("oracle closure failed")
        self.algo_ms = ms.value
        return ms.value

    @property
    def products(self) -> int:
        return int(lib().orc_products(self.h))

    def matrix(self, i: int) -> np.ndarray:
        n, w = self.n, lib().orc_words_per_row(self.h)
        ptr = lib().orc_matrix(self.h, i)
        if n == 0:
            return np.zeros((0, 0), dtype=np.uint64)
        return np.ctypeslib.as_array(ptr, shape=(n * w,)).reshape(n, w).copy()

    def results(self) -> dict[str, tuple[int, int]]:
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "answer.txt")
            lib().orc_write_results(self.h, out.encode())
            return parse_answer(open(out).read())


def parse_answer(text: str) -> dict[str, tuple[int, int]]:
    out = {}
    for line in text.splitlines():
        if line.strip():
            name, h, c = line.split()
            out[name] = (int(h), int(c))
    return out


def ref_executable(name: str) -> str | None:
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None


def run_executable(exe: str, grammar_path: str, graph_path: str, timeout: float = 1800,
                   env: dict | None = None) -> tuple[dict[str, tuple[int, int]], tuple[int, int]]:
    """Run a reference-style main: argv <grammar> <graph> <answer>, stdout "total algo"."""
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "answer.txt")
        p = subprocess.run([exe, grammar_path, graph_path, out], capture_output=True, timeout=timeout,
                           env=env)
        if p.returncode != 0 or p.stderr:
            raise RuntimeError(f"{exe} failed ({p.returncode}): {p.stderr.decode(errors='replace')[:500]}")
        total, algo = (int(x) for x in p.stdout.decode().split()[:2])
        return parse_answer(open(out).read()), (total, algo)
