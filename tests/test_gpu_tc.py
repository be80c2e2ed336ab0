"""Parity of the tensor-core variant (tcgen05 kind::i8) with the CPU oracle:
bit-exact products, changed flags, tile statistics and closures."""
import os

import numpy as np
import pytest

from test_gpu_parity import _check_query, check_tile_stats, rand_rows, upload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 64, 65, 130, 257, 300, 640, 1000, 1100])
def test_tc_add_mul_random(ctx, oracle, n):
    rng = np.random.default_rng(n * 13 + 1)
    for density in (0.003, 0.05, 0.5, 1.0):
        a, b, c = (rand_rows(rng, n, d) for d in (density, density, density / 3))
        ma, mb, mc = upload(ctx, n, a), upload(ctx, n, b), upload(ctx, n, c)
        exp = c.copy()
        ch_exp = oracle.add_mul(exp, a, b, n, oracle.NAIVE, 1)
        ch = ctx.add_mul(mc, ma, mb, "tc")
        assert np.array_equal(mc.download_rows(), exp), f"n={n} density={density}"
        assert ch == ch_exp
        check_tile_stats(mc, exp)
        assert ctx.add_mul(mc, ma, mb, "tc") is False
        for m in (ma, mb, mc):
            m.destroy()


def test_tc_structured_products(ctx, oracle):
    """Identity, permutation and single-bit operands pin the operand layouts
    (row/column orientation of the expanded P and transposed Q)."""
    n = 300
    eye = np.zeros((n, (n + 63) // 64), dtype=np.uint64)
    for i in range(n):
        eye[i, i // 64] |= np.uint64(1) << np.uint64(i % 64)
    rng = np.random.default_rng(4)
    x = rand_rows(rng, n, 0.1)
    for a, b in ((eye, x), (x, eye)):
        ma, mb, mc = upload(ctx, n, a), upload(ctx, n, b), ctx.matrix(n)
        ctx.add_mul(mc, ma, mb, "tc")
        assert np.array_equal(mc.download_rows(), x)
        for m in (ma, mb, mc):
            m.destroy()
    for (i, k, j) in ((0, 0, 0), (5, 130, 299), (299, 64, 63), (128, 255, 256)):
        a = np.zeros_like(eye)
        b = np.zeros_like(eye)
        a[i, k // 64] |= np.uint64(1) << np.uint64(k % 64)
        b[k, j // 64] |= np.uint64(1) << np.uint64(j % 64)
        ma, mb, mc = upload(ctx, n, a), upload(ctx, n, b), ctx.matrix(n)
        assert ctx.add_mul(mc, ma, mb, "tc") is True
        got = mc.download_rows()
        exp = np.zeros_like(eye)
        exp[i, j // 64] |= np.uint64(1) << np.uint64(j % 64)
        assert np.array_equal(got, exp), (i, k, j)
        for m in (ma, mb, mc):
            m.destroy()


@pytest.mark.parametrize("alias", ["a", "b", "ab"])
def test_tc_aliasing(ctx, oracle, alias):
    n = 333
    rng = np.random.default_rng(17)
    c = rand_rows(rng, n, 0.02)
    b = rand_rows(rng, n, 0.02)
    mc = upload(ctx, n, c)
    mb = upload(ctx, n, b)
    exp = c.copy()
    if alias == "a":
        ch_exp = oracle.add_mul(exp, c.copy(), b, n)
        ch = ctx.add_mul(mc, mc, mb, "tc")
    elif alias == "b":
        ch_exp = oracle.add_mul(exp, b, c.copy(), n)
        ch = ctx.add_mul(mc, mb, mc, "tc")
    else:
        ch_exp = oracle.add_mul(exp, c.copy(), c.copy(), n)
        ch = ctx.add_mul(mc, mc, mc, "tc")
    assert ch == ch_exp
    assert np.array_equal(mc.download_rows(), exp)


@pytest.mark.parametrize("driver", ["engine", "worklist"])
def test_tc_closure_brackets(ctx, pkg, oracle, tmp_path, driver):
    _check_query(ctx, pkg, oracle, pkg.workloads.brackets_query(), tmp_path, driver=driver, variant="tc")


@pytest.mark.parametrize("seed", [1, 2])
def test_tc_closure_random_cnf(ctx, pkg, oracle, tmp_path, seed):
    labels = ["x", "y", "z"]
    g = pkg.workloads.uniform_graph(900, 2000, labels, seed)
    gram = pkg.workloads.random_cnf(8, 20, labels, seed)
    wl = pkg.workloads.Workload("random_cnf", gram, g, {})
    _check_query(ctx, pkg, oracle, wl, tmp_path, variant="tc")


def test_tc_closure_same_generation(ctx, pkg, oracle, tmp_path):
    _check_query(ctx, pkg, oracle, pkg.workloads.ontology_query(2048, 4), tmp_path, variant="tc")
