"""ctypes binding of libcfpq_b200.so (the C ABI declared in include/cfpq_b200.h).

Used by the tests, bench.py and the Python query helpers.  The library is
the product; this module only marshals arguments.  Loading fails loudly when
the shared library has not been built -- there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable, Sequence

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libcfpq_b200.so")

OK = 0
ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_UNSUPPORTED, ERR_TIMEOUT, ERR_IO = 1, 2, 3, 4, 5, 6

VARIANT_AUTO, VARIANT_PLAIN, VARIANT_LOP3, VARIANT_M4R, VARIANT_TC, VARIANT_NTSET = 0, 1, 2, 3, 4, 5
VARIANTS = {"auto": 0, "plain": 1, "lop3": 2, "m4r": 3, "tc": 4, "ntset": 5}
LOOPS = {"host": 0, "device": 1, "graph": 2}
DRIVER_ENGINE, DRIVER_WORKLIST = 0, 1

# Every entry point declared in include/cfpq_b200.h.
EXPORTED = (
    "cfpq_abi_version", "cfpq_last_error", "cfpq_ctx_create", "cfpq_ctx_destroy", "cfpq_ctx_synchronize",
    "cfpq_ctx_num_sms", "cfpq_matrix_create", "cfpq_matrix_destroy", "cfpq_matrix_size", "cfpq_matrix_set_bits",
    "cfpq_matrix_set_bits_device", "cfpq_load_edges", "cfpq_matrix_set_diagonal", "cfpq_matrix_clear",
    "cfpq_matrix_copy", "cfpq_matrix_upload_rows", "cfpq_matrix_download_rows", "cfpq_matrix_hash_count",
    "cfpq_matrix_count", "cfpq_hash_count_many", "cfpq_add_mul", "cfpq_closure", "cfpq_closure_batch",
    "cfpq_product_log", "cfpq_last_kernel_profile", "cfpq_ctx_stream", "cfpq_load_edges_device",
    "cfpq_matrix_tile_stats", "cfpq_order_create", "cfpq_order_destroy", "cfpq_order_suggest",
    "cfpq_matrix_create_ordered", "cfpq_hash_count_rows_noalloc", "cfpq_noalloc_last_error", "cfpq_calibrate",
    "cfpq_last_phase_log", "cfpq_matrices_clear", "cfpq_selector_configure", "cfpq_selector_get_config",
    "cfpq_selector_weight_count", "cfpq_selector_set_weights", "cfpq_selector_get_weights", "cfpq_selector_train",
    "cfpq_selector_loss_grad", "cfpq_selector_predict", "cfpq_autotune", "cfpq_item_log", "cfpq_add_mul_rows",
    "cfpq_matrix_block_bytes", "cfpq_matrix_export_block", "cfpq_matrix_import_block", "cfpq_matrix_delta",
    "cfpq_graph_load", "cfpq_edge_list_free", "cfpq_closure_hash", "cfpq_intersection",
)


class Calibration(ctypes.Structure):
    _fields_ = [("logic_ops_per_s", ctypes.c_double), ("logic_ops_per_clk_sm", ctypes.c_double),
                ("bitmac_per_s", ctypes.c_double), ("ms", ctypes.c_double)]


class CfpqError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"cfpq error {code}: {message}")
        self.code = code


class Rule(ctypes.Structure):
    _fields_ = [("head", ctypes.c_uint32), ("body1", ctypes.c_uint32), ("body2", ctypes.c_uint32)]


class Edges(ctypes.Structure):
    """cfpq_edges: a labelled graph for cfpq_intersection."""
    _fields_ = [("from", ctypes.c_void_p), ("label", ctypes.c_void_p), ("to", ctypes.c_void_p),
                ("count", ctypes.c_size_t), ("label_offsets", ctypes.c_void_p), ("label_mats", ctypes.c_void_p),
                ("nlabels", ctypes.c_uint32), ("on_device", ctypes.c_int32)]


class ClosureOpts(ctypes.Structure):
    _fields_ = [("driver", ctypes.c_int32), ("variant", ctypes.c_int32), ("max_iterations", ctypes.c_int32),
                ("use_graph", ctypes.c_int32), ("log_products", ctypes.c_int32), ("wait_limit", ctypes.c_int32),
                ("test_flags", ctypes.c_int32), ("reserved", ctypes.c_int32 * 1)]


TEST_STALL_BARRIER = 1


class ClosureStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint32), ("reserved0", ctypes.c_uint32), ("products", ctypes.c_uint64),
                ("tile_triples", ctypes.c_uint64), ("work_items", ctypes.c_uint64),
                ("dense_bitops", ctypes.c_uint64), ("device_ms", ctypes.c_double),
                ("kernel_launches", ctypes.c_uint64), ("variant_items", ctypes.c_uint64 * 5),
                ("bytes_staged", ctypes.c_uint64), ("out_words", ctypes.c_uint64), ("new_words", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}
        d["variant_items"] = list(self.variant_items)
        return d


class KernelProfile(ctypes.Structure):
    _fields_ = [("plan_ms", ctypes.c_double), ("product_ms", ctypes.c_double), ("advance_ms", ctypes.c_double),
                ("iter_end_ms", ctypes.c_double), ("plan_launches", ctypes.c_uint64),
                ("product_launches", ctypes.c_uint64), ("advance_launches", ctypes.c_uint64),
                ("iter_end_launches", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


LOG_KERNELS, LOG_PRODUCTS = 1, 2


class Query(ctypes.Structure):
    _fields_ = [("rules", ctypes.POINTER(Rule)), ("nrules", ctypes.c_size_t),
                ("mats", ctypes.POINTER(ctypes.c_void_p)), ("nmats", ctypes.c_size_t)]


SEL_FEATURES, SEL_OUTPUTS = 16, 3
SELECT_FIXED, SELECT_HEURISTIC, SELECT_MLP = 0, 1, 2
LOG_SELECTION = 4
LOG_ITEMS = 8

# numpy view of an array of cfpq_item_record
ITEM_RECORD_DTYPE = np.dtype([("item", np.uint64), ("iteration", np.uint32), ("cta", np.uint16),
                              ("list", np.uint16), ("start_ns", np.uint64), ("end_ns", np.uint64),
                              ("klist_ns", np.uint32), ("staged_ns", np.uint32), ("computed_ns", np.uint32),
                              ("gate_ns", np.uint32)])


class ProductRecord(ctypes.Structure):
    _fields_ = [("iteration", ctypes.c_uint32), ("query", ctypes.c_uint32), ("rule", ctypes.c_uint32),
                ("term", ctypes.c_uint32), ("n", ctypes.c_uint32), ("variant", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("features", ctypes.c_float * SEL_FEATURES), ("predicted", ctypes.c_float * SEL_OUTPUTS),
                ("usec", ctypes.c_float * 5)]


# numpy view of an array of cfpq_product_record
PRODUCT_RECORD_DTYPE = np.dtype([("iteration", np.uint32), ("query", np.uint32), ("rule", np.uint32),
                                 ("term", np.uint32), ("n", np.uint32), ("variant", np.uint32),
                                 ("flags", np.uint32), ("reserved", np.uint32),
                                 ("features", np.float32, (SEL_FEATURES,)), ("predicted", np.float32, (SEL_OUTPUTS,)),
                                 ("usec", np.float32, (5,))])


class SelectorConfig(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("allowed", ctypes.c_uint32), ("tc_min_tiles", ctypes.c_uint32),
                ("tc_min_occ", ctypes.c_float), ("tc_min_dense", ctypes.c_float), ("m4r_min_dense", ctypes.c_float),
                ("conf_margin", ctypes.c_float), ("range_margin", ctypes.c_float), ("min_tiles", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TrainOpts(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("learning_rate", ctypes.c_float), ("weight_decay", ctypes.c_float),
                ("seed", ctypes.c_uint32), ("keep_weights", ctypes.c_int32)]


class TrainReport(ctypes.Structure):
    _fields_ = [("loss_first", ctypes.c_float), ("loss_last", ctypes.c_float), ("samples", ctypes.c_uint32),
                ("epochs", ctypes.c_uint32), ("ms", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class EdgeList(ctypes.Structure):
    _fields_ = [("from_", ctypes.POINTER(ctypes.c_uint32)), ("label", ctypes.POINTER(ctypes.c_uint32)),
                ("to", ctypes.POINTER(ctypes.c_uint32)), ("nedges", ctypes.c_size_t),
                ("nvertices", ctypes.c_uint32), ("nlabels", ctypes.c_uint32),
                ("labels", ctypes.POINTER(ctypes.c_char_p))]


class AutotuneOpts(ctypes.Structure):
    _fields_ = [("sizes", ctypes.POINTER(ctypes.c_uint32)), ("nsizes", ctypes.c_size_t),
                ("densities", ctypes.POINTER(ctypes.c_float)), ("ndensities", ctypes.c_size_t),
                ("reps", ctypes.c_uint32), ("seed", ctypes.c_uint32)]


_lib = None


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load libcfpq_b200.so and declare the C signatures (cached)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} is not built; run `make -C cfpq-on-gpgpu_b200` (or __graft_entry__.build())")
    lib = ctypes.CDLL(p)
    vp, u32, u64, sz, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_int
    P = ctypes.POINTER
    sigs = {
        "cfpq_abi_version": ([], i32),
        "cfpq_last_error": ([], ctypes.c_char_p),
        "cfpq_ctx_create": ([i32, P(vp)], i32),
        "cfpq_ctx_destroy": ([vp], i32),
        "cfpq_ctx_synchronize": ([vp], i32),
        "cfpq_ctx_num_sms": ([vp], i32),
        "cfpq_matrix_create": ([vp, u32, P(vp)], i32),
        "cfpq_matrix_destroy": ([vp, vp], i32),
        "cfpq_matrix_size": ([vp], u32),
        "cfpq_matrix_set_bits": ([vp, vp, vp, vp, sz], i32),
        "cfpq_matrix_set_bits_device": ([vp, vp, vp, vp, sz], i32),
        "cfpq_load_edges": ([vp, P(vp), sz, vp, vp, vp, sz, vp, vp, u32], i32),
        "cfpq_matrix_set_diagonal": ([vp, vp], i32),
        "cfpq_matrix_clear": ([vp, vp], i32),
        "cfpq_matrix_copy": ([vp, vp, vp], i32),
        "cfpq_matrix_upload_rows": ([vp, vp, vp], i32),
        "cfpq_matrix_download_rows": ([vp, vp, vp], i32),
        "cfpq_matrix_hash_count": ([vp, vp, P(u64), P(u64)], i32),
        "cfpq_matrix_count": ([vp, vp, P(u64)], i32),
        "cfpq_hash_count_many": ([vp, P(vp), sz, P(u64), P(u64)], i32),
        "cfpq_add_mul": ([vp, vp, vp, vp, i32, P(i32)], i32),
        "cfpq_closure": ([vp, P(Rule), sz, P(vp), sz, P(ClosureOpts), P(ClosureStats)], i32),
        "cfpq_closure_batch": ([vp, P(Query), sz, P(ClosureOpts), P(ClosureStats), P(u32),
                                P(ctypes.c_double)], i32),
        "cfpq_product_log": ([vp, P(ProductRecord), sz], sz),
        "cfpq_last_kernel_profile": ([vp, P(KernelProfile)], i32),
        "cfpq_ctx_stream": ([vp], vp),
        "cfpq_matrix_tile_stats": ([vp, vp, vp, vp], i32),
        "cfpq_order_create": ([vp, u32, vp, P(vp)], i32),
        "cfpq_order_destroy": ([vp, vp], i32),
        "cfpq_order_suggest": ([u32, vp, vp, vp, sz, vp], i32),
        "cfpq_matrix_create_ordered": ([vp, u32, vp, P(vp)], i32),
        "cfpq_calibrate": ([vp, P(Calibration)], i32),
        "cfpq_load_edges_device": ([vp, P(vp), sz, vp, vp, vp, sz, vp, vp, u32], i32),
        "cfpq_last_phase_log": ([vp, P(u64), sz], sz),
        "cfpq_item_log": ([vp, vp, sz], sz),
        "cfpq_matrices_clear": ([vp, P(vp), sz], i32),
        "cfpq_selector_configure": ([vp, P(SelectorConfig)], i32),
        "cfpq_selector_get_config": ([vp, P(SelectorConfig)], i32),
        "cfpq_selector_weight_count": ([], sz),
        "cfpq_selector_set_weights": ([vp, vp, sz], i32),
        "cfpq_selector_get_weights": ([vp, vp, sz], i32),
        "cfpq_selector_train": ([vp, vp, sz, P(TrainOpts), P(TrainReport)], i32),
        "cfpq_selector_loss_grad": ([vp, vp, vp, vp, vp, sz, P(ctypes.c_float), vp], i32),
        "cfpq_selector_predict": ([vp, vp, sz, vp], i32),
        "cfpq_autotune": ([vp, P(AutotuneOpts), P(SelectorConfig), vp], i32),
        "cfpq_add_mul_rows": ([vp, vp, vp, vp, i32, u32, u32, P(i32)], i32),
        "cfpq_matrix_block_bytes": ([vp, u32, u32], sz),
        "cfpq_matrix_export_block": ([vp, vp, u32, u32, vp], i32),
        "cfpq_matrix_import_block": ([vp, vp, u32, u32, vp], i32),
        "cfpq_matrix_delta": ([vp, vp, vp, vp], i32),
        "cfpq_graph_load": ([ctypes.c_char_p, i32, P(P(EdgeList))], i32),
        "cfpq_closure_hash": ([vp, P(Rule), sz, P(vp), sz, P(ClosureOpts), P(ClosureStats), P(u64), P(u64)], i32),
        "cfpq_edge_list_free": ([P(EdgeList)], None),
        "cfpq_intersection": ([vp, P(Rule), sz, P(vp), sz, P(Edges), P(u32), sz, P(ClosureOpts), P(ClosureStats),
                               P(u64), P(u64)], i32),
    }
    for name, (args, res) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    if path is None:
        _lib = lib
    return lib


def _check(lib, rc: int) -> None:
    if rc != OK:
        raise CfpqError(rc, lib.cfpq_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def load_graph_file(path: str, threads: int = 0, lib=None):
    """(src, label, dst, labels, n) of a graph file parsed by the library's
    parallel loader (cfpq_graph_load); arrays are uint32 copies."""
    lib = lib or load_library()
    out = ctypes.POINTER(EdgeList)()
    _check(lib, lib.cfpq_graph_load(os.fsencode(path), int(threads), ctypes.byref(out)))
    try:
        e = out.contents
        m = int(e.nedges)
        arrs = [np.ctypeslib.as_array(ptr, shape=(m,)).copy() if m else np.zeros(0, dtype=np.uint32)
                for ptr in (e.from_, e.label, e.to)]
        labels = [e.labels[i].decode() for i in range(e.nlabels)]
        return arrs[0], arrs[1], arrs[2], labels, int(e.nvertices)
    finally:
        lib.cfpq_edge_list_free(out)


def suggest_order(n: int, src: np.ndarray, label: np.ndarray, dst: np.ndarray, lib=None) -> np.ndarray:
    """Vertex relabeling suggested by the library's heuristic (perm[v] = internal id)."""
    lib = lib or load_library()
    s = np.ascontiguousarray(src, dtype=np.uint32)
    l = np.ascontiguousarray(label, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    perm = np.zeros(max(int(n), 1), dtype=np.uint32)
    _check(lib, lib.cfpq_order_suggest(int(n), _ptr(s), _ptr(l), _ptr(d), s.size, _ptr(perm)))
    return perm[:int(n)]


class Order:
    """A vertex relabeling shared by the matrices of one query."""

    def __init__(self, ctx: "Context", perm: np.ndarray):
        self.ctx = ctx
        self.perm = np.ascontiguousarray(perm, dtype=np.uint32)
        self.n = int(self.perm.size)
        h = ctypes.c_void_p()
        _check(ctx.lib, ctx.lib.cfpq_order_create(ctx.handle, self.n, _ptr(self.perm), ctypes.byref(h)))
        self.handle = h

    def destroy(self) -> None:
        if self.handle:
            _check(self.ctx.lib, self.ctx.lib.cfpq_order_destroy(self.ctx.handle, self.handle))
            self.handle = None


class Matrix:
    """An n x n Boolean matrix resident on the device."""

    def __init__(self, ctx: "Context", n: int, order: Order | None = None):
        self.ctx, self.n, self.order = ctx, int(n), order
        h = ctypes.c_void_p()
        _check(ctx.lib, ctx.lib.cfpq_matrix_create_ordered(ctx.handle, self.n, order.handle if order else None,
                                                           ctypes.byref(h)))
        self.handle = h

    @property
    def words_per_row(self) -> int:
        return (self.n + 63) // 64

    def set_bits(self, rows: Iterable[int], cols: Iterable[int]) -> None:
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.uint32))
        c = np.ascontiguousarray(np.asarray(cols, dtype=np.uint32))
        if r.shape != c.shape:
            raise ValueError("rows and cols differ in length")
        _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_set_bits(self.ctx.handle, self.handle, _ptr(r), _ptr(c), r.size))

    def set_diagonal(self) -> None:
        _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_set_diagonal(self.ctx.handle, self.handle))

    def clear(self) -> None:
        _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_clear(self.ctx.handle, self.handle))

    def copy_from(self, other: "Matrix") -> None:
        _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_copy(self.ctx.handle, self.handle, other.handle))

    def upload_rows(self, rows: np.ndarray) -> None:
        a = np.ascontiguousarray(rows, dtype=np.uint64)
        if a.size != self.n * self.words_per_row:
            raise ValueError(f"expected {self.n * self.words_per_row} words, got {a.size}")
        _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_upload_rows(self.ctx.handle, self.handle, _ptr(a)))

    def download_rows(self) -> np.ndarray:
        a = np.zeros((self.n, self.words_per_row), dtype=np.uint64)
        if self.n:
            _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_download_rows(self.ctx.handle, self.handle, _ptr(a)))
        return a

    def block_bytes(self, row_begin: int, row_end: int) -> int:
        """Bytes of the packed row block [row_begin, row_end) (0 if the range is invalid)."""
        return int(self.ctx.lib.cfpq_matrix_block_bytes(self.handle, int(row_begin), int(row_end)))

    def export_block(self, row_begin: int, row_end: int, dst_ptr: int) -> None:
        """Copy the packed row block to dst_ptr (device or host address; asynchronous)."""
        _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_export_block(self.ctx.handle, self.handle, int(row_begin),
                                                                   int(row_end), ctypes.c_void_p(dst_ptr)))

    def import_block(self, row_begin: int, row_end: int, src_ptr: int) -> None:
        """Overwrite the rows [row_begin, row_end) from a packed block at src_ptr (asynchronous)."""
        _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_import_block(self.ctx.handle, self.handle, int(row_begin),
                                                                   int(row_end), ctypes.c_void_p(src_ptr)))

    def tile_stats(self) -> tuple[np.ndarray, np.ndarray]:
        """(occupancy bitmap [T, ceil(T/32)] uint32, tile populations [T, T] uint32)."""
        T = (self.n + 63) // 64
        occ = np.zeros((T, (T + 31) // 32), dtype=np.uint32)
        nnz = np.zeros((T, T), dtype=np.uint32)
        if T:
            _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_tile_stats(self.ctx.handle, self.handle, _ptr(occ),
                                                                     _ptr(nnz)))
        return occ, nnz

    def hash_count(self) -> tuple[int, int]:
        h, c = ctypes.c_uint64(), ctypes.c_uint64()
        _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_hash_count(self.ctx.handle, self.handle, ctypes.byref(h),
                                                                 ctypes.byref(c)))
        return int(h.value), int(c.value)

    def destroy(self) -> None:
        if self.handle:
            _check(self.ctx.lib, self.ctx.lib.cfpq_matrix_destroy(self.ctx.handle, self.handle))
            self.handle = None


class Context:
    """A device context (one CUDA stream and the engine's scratch state)."""

    def __init__(self, device: int = 0, lib: ctypes.CDLL | None = None):
        self.lib = lib or load_library()
        h = ctypes.c_void_p()
        _check(self.lib, self.lib.cfpq_ctx_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.device = device
        self._closure_args = None  # (key, ctypes arguments) of the last closure() call

    def close(self) -> None:
        if self.handle:
            _check(self.lib, self.lib.cfpq_ctx_destroy(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def num_sms(self) -> int:
        return self.lib.cfpq_ctx_num_sms(self.handle)

    def synchronize(self) -> None:
        _check(self.lib, self.lib.cfpq_ctx_synchronize(self.handle))

    def matrix(self, n: int, order: Order | None = None) -> Matrix:
        return Matrix(self, n, order)

    def order(self, perm: np.ndarray) -> Order:
        return Order(self, perm)

    def add_mul(self, c: Matrix, a: Matrix, b: Matrix, variant: int | str = VARIANT_AUTO) -> bool:
        v = VARIANTS[variant] if isinstance(variant, str) else int(variant)
        ch = ctypes.c_int()
        _check(self.lib, self.lib.cfpq_add_mul(self.handle, c.handle, a.handle, b.handle, v, ctypes.byref(ch)))
        return bool(ch.value)

    def add_mul_rows(self, c: Matrix, a: Matrix, b: Matrix, row_begin: int, row_end: int,
                     variant: int | str = VARIANT_LOP3) -> bool:
        """c[rows] |= a[rows] * b for the rows [row_begin, row_end); True if c changed."""
        v = VARIANTS[variant] if isinstance(variant, str) else int(variant)
        ch = ctypes.c_int(0)
        _check(self.lib, self.lib.cfpq_add_mul_rows(self.handle, c.handle, a.handle, b.handle, v, int(row_begin),
                                                    int(row_end), ctypes.byref(ch)))
        return bool(ch.value)

    def delta(self, delta: Matrix, cur: Matrix, prev: Matrix) -> None:
        """delta = cur & ~prev, then prev = cur (asynchronous)."""
        _check(self.lib, self.lib.cfpq_matrix_delta(self.handle, delta.handle, cur.handle, prev.handle))

    @staticmethod
    def _opts(driver, variant, use_graph, max_iterations, log_products, wait_limit=0, test_flags=0) -> ClosureOpts:
        o = ClosureOpts()
        o.driver = {"engine": DRIVER_ENGINE, "worklist": DRIVER_WORKLIST}.get(driver, driver)
        o.variant = VARIANTS[variant] if isinstance(variant, str) else int(variant)
        # loop sequencing: True / "device" (persistent kernel when possible),
        # "graph" (CUDA-graph loop), False / "host" (host loop)
        o.use_graph = LOOPS[use_graph] if isinstance(use_graph, str) else int(bool(use_graph))
        o.max_iterations = int(max_iterations)
        o.log_products = int(log_products)
        o.wait_limit = int(wait_limit)
        o.test_flags = int(test_flags)
        return o

    def closure(self, rules: Sequence[tuple[int, int, int]], mats: Sequence[Matrix], driver="engine",
                variant="auto", use_graph: bool = True, max_iterations: int = 0, log_products: bool = False,
                wait_limit: int = 0, test_flags: int = 0) -> dict:
        # the ctypes arguments of the last call are kept: a prepared query
        # closed again (the serving loop) pays no argument marshalling
        key = (tuple(map(tuple, rules)), tuple(m.handle for m in mats), driver, variant, use_graph,
               max_iterations, log_products, wait_limit, test_flags)
        args = self._closure_args if self._closure_args and self._closure_args[0] == key else None
        if args is None:
            rs = (Rule * max(len(rules), 1))(*[Rule(*map(int, r)) for r in rules])
            hs = (ctypes.c_void_p * max(len(mats), 1))(*[m.handle for m in mats])
            o = self._opts(driver, variant, use_graph, max_iterations, log_products, wait_limit, test_flags)
            args = self._closure_args = (key, rs, hs, o, ClosureStats())
        _, rs, hs, o, st = args
        _check(self.lib, self.lib.cfpq_closure(self.handle, rs, len(rules), hs, len(mats), ctypes.byref(o),
                                               ctypes.byref(st)))
        return st.as_dict()

    def closure_hash(self, rules: Sequence[tuple[int, int, int]], mats: Sequence[Matrix], variant="auto",
                     use_graph: bool = True) -> tuple[dict, list[tuple[int, int]]]:
        """Closure, then the result line (hash, count) of every matrix, with one
        synchronisation (cfpq_closure_hash).  The ctypes arguments of the last
        call are kept, like closure()."""
        key = (tuple(map(tuple, rules)), tuple(m.handle for m in mats), variant, use_graph)
        args = self._hash_args if getattr(self, "_hash_args", None) and self._hash_args[0] == key else None
        if args is None:
            rs = (Rule * max(len(rules), 1))(*[Rule(*map(int, r)) for r in rules])
            hs = (ctypes.c_void_p * max(len(mats), 1))(*[m.handle for m in mats])
            o = self._opts("engine", variant, use_graph, 0, 0)
            hh = (ctypes.c_uint64 * max(len(mats), 1))()
            cc = (ctypes.c_uint64 * max(len(mats), 1))()
            args = self._hash_args = (key, rs, hs, o, ClosureStats(), hh, cc)
        _, rs, hs, o, st, hh, cc = args
        _check(self.lib, self.lib.cfpq_closure_hash(self.handle, rs, len(rules), hs, len(mats), ctypes.byref(o),
                                                    ctypes.byref(st), hh, cc))
        return st.as_dict(), [(int(hh[i]), int(cc[i])) for i in range(len(mats))]

    def intersection(self, rules: Sequence[tuple[int, int, int]], mats: Sequence[Matrix], src, label, dst,
                     label_offsets: np.ndarray, label_mats: np.ndarray, epsilon: Sequence[int] = (),
                     nedges: int | None = None, variant="auto", use_graph: bool = True, lines: bool = True):
        """One whole query with one synchronisation (cfpq_intersection): clear
        mats, scatter the edges, set the epsilon diagonals, close, and (lines)
        the result line (hash, count) of every matrix.  src/label/dst: uint32
        host arrays, or device pointers as ints (nedges then required).
        Returns (stats, lines or None).  The ctypes arguments of the last call
        are kept (keyed on the arrays' addresses), like closure()."""
        on_device = isinstance(src, int)
        if on_device:
            if nedges is None:
                raise ValueError("nedges is required with device pointers")
            ptrs, keep = (src, label, dst), ()
        else:
            keep = tuple(np.ascontiguousarray(a, dtype=np.uint32) for a in (src, label, dst))
            ptrs, nedges = tuple(a.ctypes.data for a in keep), keep[0].size
        key = (tuple(map(tuple, rules)), tuple(m.handle for m in mats), ptrs, int(nedges),
               tuple(np.asarray(label_offsets).tolist()), tuple(np.asarray(label_mats).tolist()), tuple(epsilon),
               variant, use_graph, lines)
        args = self._isect_args if getattr(self, "_isect_args", None) and self._isect_args[0] == key else None
        if args is None:
            rs = (Rule * max(len(rules), 1))(*[Rule(*map(int, r)) for r in rules])
            hs = (ctypes.c_void_p * max(len(mats), 1))(*[m.handle for m in mats])
            off = np.ascontiguousarray(label_offsets, dtype=np.uint32)
            lm = np.ascontiguousarray(label_mats, dtype=np.uint32)
            if lm.size == 0:
                lm = np.zeros(1, dtype=np.uint32)
            e = Edges(ptrs[0], ptrs[1], ptrs[2], int(nedges), off.ctypes.data, lm.ctypes.data, off.size - 1,
                      1 if on_device else 0)
            eps = (ctypes.c_uint32 * max(len(epsilon), 1))(*[int(x) for x in epsilon])
            o = self._opts("engine", variant, use_graph, 0, 0)
            hh = (ctypes.c_uint64 * max(len(mats), 1))() if lines else None
            cc = (ctypes.c_uint64 * max(len(mats), 1))() if lines else None
            args = self._isect_args = (key, rs, hs, e, eps, o, ClosureStats(), hh, cc, (keep, off, lm))
        _, rs, hs, e, eps, o, st, hh, cc, _ = args
        _check(self.lib, self.lib.cfpq_intersection(self.handle, rs, len(rules), hs, len(mats), ctypes.byref(e),
                                                    eps, len(epsilon), ctypes.byref(o), ctypes.byref(st), hh, cc))
        return st.as_dict(), ([(int(hh[i]), int(cc[i])) for i in range(len(mats))] if lines else None)

    def closure_batch(self, queries: Sequence[tuple[Sequence[tuple[int, int, int]], Sequence[Matrix]]],
                      variant="auto", use_graph: bool = True, max_iterations: int = 0, log_products: int = 0):
        keep = []
        qs = (Query * max(len(queries), 1))()
        for i, (rules, mats) in enumerate(queries):
            rs = (Rule * max(len(rules), 1))(*[Rule(*map(int, r)) for r in rules])
            hs = (ctypes.c_void_p * max(len(mats), 1))(*[m.handle for m in mats])
            keep += [rs, hs]
            qs[i].rules = ctypes.cast(rs, ctypes.POINTER(Rule))
            qs[i].nrules = len(rules)
            qs[i].mats = ctypes.cast(hs, ctypes.POINTER(ctypes.c_void_p))
            qs[i].nmats = len(mats)
        o = self._opts("engine", variant, use_graph, max_iterations, log_products)
        st = ClosureStats()
        iters = np.zeros(max(len(queries), 1), dtype=np.uint32)
        done = np.zeros(max(len(queries), 1), dtype=np.float64)
        _check(self.lib, self.lib.cfpq_closure_batch(
            self.handle, qs, len(queries), ctypes.byref(o), ctypes.byref(st),
            iters.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
            done.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return st.as_dict(), iters[:len(queries)], done[:len(queries)]

    def load_edges(self, mats: Sequence[Matrix], src: np.ndarray, label: np.ndarray, dst: np.ndarray,
                   label_offsets: np.ndarray, label_mats: np.ndarray) -> None:
        s = np.ascontiguousarray(src, dtype=np.uint32)
        l = np.ascontiguousarray(label, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        off = np.ascontiguousarray(label_offsets, dtype=np.uint32)
        lm = np.ascontiguousarray(label_mats, dtype=np.uint32)
        if lm.size == 0:
            lm = np.zeros(1, dtype=np.uint32)
        hs = (ctypes.c_void_p * max(len(mats), 1))(*[m.handle for m in mats])
        _check(self.lib, self.lib.cfpq_load_edges(self.handle, hs, len(mats), _ptr(s), _ptr(l), _ptr(d), s.size,
                                                  _ptr(off), _ptr(lm), off.size - 1))

    @property
    def stream(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(self.lib.cfpq_ctx_stream(self.handle) or 0)

    def load_edges_device(self, mats: Sequence[Matrix], d_src: int, d_label: int, d_dst: int, nedges: int,
                          label_offsets: np.ndarray, label_mats: np.ndarray) -> None:
        """Edge scatter from device-resident arrays (device pointers as ints)."""
        off = np.ascontiguousarray(label_offsets, dtype=np.uint32)
        lm = np.ascontiguousarray(label_mats, dtype=np.uint32)
        if lm.size == 0:
            lm = np.zeros(1, dtype=np.uint32)
        hs = (ctypes.c_void_p * max(len(mats), 1))(*[m.handle for m in mats])
        _check(self.lib, self.lib.cfpq_load_edges_device(self.handle, hs, len(mats), ctypes.c_void_p(d_src),
                                                         ctypes.c_void_p(d_label), ctypes.c_void_p(d_dst),
                                                         int(nedges), _ptr(off), _ptr(lm), off.size - 1))

    def calibrate(self) -> dict:
        c = Calibration()
        _check(self.lib, self.lib.cfpq_calibrate(self.handle, ctypes.byref(c)))
        return {k: getattr(c, k) for k, _ in c._fields_}

    def phase_log(self) -> np.ndarray:
        """Per-iteration durations in microseconds of the last persistent
        closure, shape (iterations, 2): CTA 0's share of the plan, then the
        rest of the iteration up to its grid barrier (items run while other
        CTAs still plan); empty if none."""
        n = self.lib.cfpq_last_phase_log(self.handle, None, 0)
        if n == 0:
            return np.zeros((0, 2))
        buf = np.zeros(3 * n, dtype=np.uint64)
        self.lib.cfpq_last_phase_log(self.handle, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), buf.size)
        t = buf.reshape(n, 3).astype(np.float64)
        return np.stack([t[:, 1] - t[:, 0], t[:, 2] - t[:, 1]], axis=1) / 1e3

    # ---- variant selector -------------------------------------------------
    def selector_config(self) -> dict:
        c = SelectorConfig()
        _check(self.lib, self.lib.cfpq_selector_get_config(self.handle, ctypes.byref(c)))
        return c.as_dict()

    def selector_configure(self, **kw) -> dict:
        """Change selector settings (keys of cfpq_selector_config; mode may be
        "fixed" / "heuristic" / "mlp", allowed a list of variant names)."""
        cur = self.selector_config()
        if isinstance(kw.get("mode"), str):
            kw["mode"] = {"fixed": SELECT_FIXED, "heuristic": SELECT_HEURISTIC, "mlp": SELECT_MLP}[kw["mode"]]
        if isinstance(kw.get("allowed"), (list, tuple)):
            kw["allowed"] = sum(1 << VARIANTS[v] for v in kw["allowed"])
        cur.update(kw)
        c = SelectorConfig(**cur)
        _check(self.lib, self.lib.cfpq_selector_configure(self.handle, ctypes.byref(c)))
        return self.selector_config()

    def selector_weights(self) -> np.ndarray:
        w = np.zeros(self.lib.cfpq_selector_weight_count(), dtype=np.float32)
        _check(self.lib, self.lib.cfpq_selector_get_weights(self.handle, _ptr(w), w.size))
        return w

    def selector_set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(self.lib, self.lib.cfpq_selector_set_weights(self.handle, _ptr(w), w.size))

    def selector_train(self, records: np.ndarray, epochs: int = 2000, learning_rate: float = 3e-3,
                       weight_decay: float = 1e-4, seed: int = 1, keep_weights: bool = False) -> dict:
        rec = np.ascontiguousarray(records, dtype=PRODUCT_RECORD_DTYPE)
        o = TrainOpts(epochs, learning_rate, weight_decay, seed, int(keep_weights))
        r = TrainReport()
        _check(self.lib, self.lib.cfpq_selector_train(self.handle, _ptr(rec), rec.size, ctypes.byref(o),
                                                      ctypes.byref(r)))
        return r.as_dict()

    def selector_loss_grad(self, weights: np.ndarray, x: np.ndarray, y: np.ndarray, m: np.ndarray):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        x, y, m = (np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, m))
        loss = ctypes.c_float()
        grad = np.zeros_like(w)
        _check(self.lib, self.lib.cfpq_selector_loss_grad(self.handle, _ptr(w), _ptr(x), _ptr(y), _ptr(m),
                                                          x.shape[0], ctypes.byref(loss), _ptr(grad)))
        return float(loss.value), grad

    def selector_predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros((x.shape[0], SEL_OUTPUTS), dtype=np.float32)
        _check(self.lib, self.lib.cfpq_selector_predict(self.handle, _ptr(x), x.shape[0], _ptr(out)))
        return out

    def autotune(self, sizes=(2048, 8192), densities=(0.002, 0.02, 0.1, 0.3, 0.6), reps: int = 3, seed: int = 1):
        """Time LOP3 / M4R / TC on random matrices and set the selector's
        thresholds.  Returns (config dict, timings [sizes][densities][3] ms)."""
        sz = np.ascontiguousarray(sizes, dtype=np.uint32)
        de = np.ascontiguousarray(densities, dtype=np.float32)
        o = AutotuneOpts(sz.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), sz.size,
                         de.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), de.size, reps, seed)
        c = SelectorConfig()
        t = np.zeros((sz.size, de.size, 3), dtype=np.float32)
        _check(self.lib, self.lib.cfpq_autotune(self.handle, ctypes.byref(o), ctypes.byref(c), _ptr(t)))
        return c.as_dict(), t

    def product_log(self) -> np.ndarray:
        """Records of the last closure run with LOG_PRODUCTS / LOG_SELECTION."""
        n = self.lib.cfpq_product_log(self.handle, None, 0)
        out = np.zeros(n, dtype=PRODUCT_RECORD_DTYPE)
        if n:
            self.lib.cfpq_product_log(self.handle, out.ctypes.data_as(ctypes.POINTER(ProductRecord)), n)
        return out

    def item_log(self) -> np.ndarray:
        """Work items of the last persistent closure run with LOG_ITEMS: the
        records plus decoded fields product, ti, block, klo, khi."""
        n = self.lib.cfpq_item_log(self.handle, None, 0)
        raw = np.zeros(n, dtype=ITEM_RECORD_DTYPE)
        if n:
            self.lib.cfpq_item_log(self.handle, raw.ctypes.data, n)
        it = raw["item"]
        dec = {"product": it >> 48, "ti": (it >> 37) & 0x7FF, "block": (it >> 28) & 0x1FF,
               "klo": (it >> 16) & 0xFFF, "khi": (it >> 4) & 0xFFF}
        out = np.zeros(n, dtype=ITEM_RECORD_DTYPE.descr + [(k, np.uint32) for k in dec])
        for k in ITEM_RECORD_DTYPE.names:
            out[k] = raw[k]
        for k, v in dec.items():
            out[k] = v.astype(np.uint32)
        return out

    def kernel_profile(self) -> dict:
        p = KernelProfile()
        _check(self.lib, self.lib.cfpq_last_kernel_profile(self.handle, ctypes.byref(p)))
        return p.as_dict()

    def clear_many(self, mats: Sequence[Matrix]) -> None:
        """Clear several matrices with one kernel (occupied tiles only)."""
        if not mats:
            return
        hs = (ctypes.c_void_p * len(mats))(*[m.handle for m in mats])
        _check(self.lib, self.lib.cfpq_matrices_clear(self.handle, hs, len(mats)))

    def hash_count_many(self, mats: Sequence[Matrix]) -> list[tuple[int, int]]:
        if not mats:
            return []
        hs = (ctypes.c_void_p * len(mats))(*[m.handle for m in mats])
        h = (ctypes.c_uint64 * len(mats))()
        c = (ctypes.c_uint64 * len(mats))()
        _check(self.lib, self.lib.cfpq_hash_count_many(self.handle, hs, len(mats), h, c))
        return [(int(h[i]), int(c[i])) for i in range(len(mats))]
