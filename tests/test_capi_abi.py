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


def test_python_record_layouts_match_the_header(pkg, tmp_path):
    """The numpy / ctypes views of the C records have the header's sizes and
    field offsets (compiled with the host C compiler, no GPU)."""
    import subprocess

    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "cfpq_b200.h"\n'
        "int main(void) {\n"
        '  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(cfpq_item_record), offsetof(cfpq_item_record, start_ns),\n'
        "         offsetof(cfpq_item_record, klist_ns), sizeof(cfpq_product_record),\n"
        "         offsetof(cfpq_product_record, features), offsetof(cfpq_product_record, usec));\n"
        "  return 0;\n}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    item, item_start, item_klist, prod, prod_feat, prod_usec = map(int, subprocess.run(
        [str(exe)], check=True, capture_output=True, text=True).stdout.split())
    capi = pkg.capi
    assert capi.ITEM_RECORD_DTYPE.itemsize == item
    assert capi.ITEM_RECORD_DTYPE.fields["start_ns"][1] == item_start
    assert capi.ITEM_RECORD_DTYPE.fields["klist_ns"][1] == item_klist
    assert capi.PRODUCT_RECORD_DTYPE.itemsize == prod == ctypes.sizeof(capi.ProductRecord)
    assert capi.PRODUCT_RECORD_DTYPE.fields["features"][1] == prod_feat
    assert capi.PRODUCT_RECORD_DTYPE.fields["usec"][1] == prod_usec
