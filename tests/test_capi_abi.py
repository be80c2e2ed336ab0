"""The C ABI library without a GPU: it loads, exports every entry point that
include/*.h declares, and its host-only helpers behave; no compute calls."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "cfpq_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cfpq_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function(pkg):
    lib = pkg.capi.load_library()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(pkg.capi.EXPORTED)


def test_abi_version(pkg):
    lib = pkg.capi.load_library()
    header = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                               "cfpq_b200.h")).read()
    declared = int(re.search(r"#define CFPQ_B200_ABI_VERSION (\d+)", header).group(1))
    assert lib.cfpq_abi_version() == declared


def test_null_arguments_are_errors_not_crashes(pkg):
    lib = pkg.capi.load_library()
    assert lib.cfpq_ctx_create(0, None) == pkg.capi.ERR_INVALID
    assert lib.cfpq_last_error()
    assert lib.cfpq_ctx_destroy(None) == pkg.capi.OK
    assert lib.cfpq_product_log(None, None, 0) == 0


def test_context_without_gpu_reports_an_error(pkg):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.capi.CfpqError):
        pkg.capi.Context(0)


def test_order_suggest_identity_for_local_ids(pkg):
    g = pkg.workloads.chain_graph(4096, 2.0, 0.9, 64, ["a", "b"], 3)
    perm = pkg.capi.suggest_order(g.n, g.src, g.label, g.dst)
    assert np.array_equal(perm, np.arange(g.n))


def test_order_suggest_is_a_permutation_and_clusters(pkg):
    g = pkg.workloads.ontology_graph(2048, 4)
    perm = pkg.capi.suggest_order(g.n, g.src, g.label, g.dst)
    assert np.array_equal(np.sort(perm), np.arange(g.n))
    tiles = lambda p: len(set(zip((p[g.src] // 64).tolist(), (p[g.dst] // 64).tolist())))
    assert tiles(perm.astype(np.int64)) < tiles(np.arange(g.n))


def test_order_suggest_rejects_out_of_range(pkg):
    lib = pkg.capi.load_library()
    src = np.array([0, 5], dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    rc = lib.cfpq_order_suggest(4, src.ctypes.data, src.ctypes.data, src.ctypes.data, 2, out.ctypes.data)
    assert rc == pkg.capi.ERR_INVALID


# ctypes mirror -> C struct of include/cfpq_b200.h
CTYPES_STRUCTS = {
    "Calibration": "cfpq_calibration", "Rule": "cfpq_rule", "ClosureOpts": "cfpq_closure_opts",
    "ClosureStats": "cfpq_closure_stats", "KernelProfile": "cfpq_kernel_profile", "Query": "cfpq_query",
    "ProductRecord": "cfpq_product_record", "SelectorConfig": "cfpq_selector_config", "TrainOpts": "cfpq_train_opts",
    "TrainReport": "cfpq_train_report", "AutotuneOpts": "cfpq_autotune_opts", "Edges": "cfpq_edges",
}


def test_python_record_layouts_match_the_header(pkg, tmp_path):
    """The numpy / ctypes views of the C records have the header's sizes and
    field offsets (compiled with the host C compiler, no GPU)."""
    import subprocess

    capi = pkg.capi
    lines = []
    for py, c in CTYPES_STRUCTS.items():
        cls = getattr(capi, py)
        lines.append(f'  printf("{py} %zu\\n", sizeof({c}));')
        for name, _ in cls._fields_:
            lines.append(f'  printf("{py}.{name} %zu\\n", offsetof({c}, {name}));')
    for name in ITEM_FIELDS:
        lines.append(f'  printf("item.{name} %zu\\n", offsetof(cfpq_item_record, {name}));')
    lines.append('  printf("item %zu\\n", sizeof(cfpq_item_record));')
    src = tmp_path / "sizes.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "cfpq_b200.h"\nint main(void) {\n'
                   + "\n".join(lines) + "\n  return 0;\n}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = dict(ln.split() for ln in subprocess.run([str(exe)], check=True, capture_output=True,
                                                   text=True).stdout.splitlines())
    for py in CTYPES_STRUCTS:
        cls = getattr(capi, py)
        assert ctypes.sizeof(cls) == int(got[py]), py
        for name, _ in cls._fields_:
            assert getattr(cls, name).offset == int(got[f"{py}.{name}"]), f"{py}.{name}"
    assert capi.ITEM_RECORD_DTYPE.itemsize == int(got["item"])
    for name in ITEM_FIELDS:
        assert capi.ITEM_RECORD_DTYPE.fields[name][1] == int(got[f"item.{name}"]), name
    assert capi.PRODUCT_RECORD_DTYPE.itemsize == ctypes.sizeof(capi.ProductRecord)
    for name, _ in capi.ProductRecord._fields_:
        assert capi.PRODUCT_RECORD_DTYPE.fields[name][1] == capi.ProductRecord.__dict__[name].offset, name


ITEM_FIELDS = ("item", "iteration", "cta", "list", "start_ns", "end_ns", "klist_ns", "staged_ns", "computed_ns",
               "gate_ns")
