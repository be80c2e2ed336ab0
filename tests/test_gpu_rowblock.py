"""The row-block closure on the GPU: the row-range product, block export /
import and the delta kernel through the C ABI against the oracle, then
rowblock.closure with the device engine -- in one process, and as two
processes that share this GPU and exchange their blocks through gloo and
pinned host buffers (each process has its own context; no kernel waits on
the other process)."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def rand_rows(rng, n, density):
    wpr = (n + 63) // 64
    bits = rng.random((n, wpr * 64)) < density
    bits[:, n:] = False
    return np.packbits(bits, axis=1, bitorder="little").view(np.uint64).reshape(n, wpr).copy()


@pytest.mark.parametrize("n", [64, 200, 1000])
@pytest.mark.parametrize("variant", ["lop3", "m4r"])
def test_add_mul_rows_matches_oracle(ctx, oracle, n, variant):
    rng = np.random.default_rng(n + len(variant))
    a, b, c = rand_rows(rng, n, 0.05), rand_rows(rng, n, 0.05), rand_rows(rng, n, 0.02)
    ma, mb, mc = (ctx.matrix(n) for _ in range(3))
    try:
        ma.upload_rows(a)
        mb.upload_rows(b)
        T = (n + 63) // 64
        for t0, t1 in ((0, T), (0, 1), (T // 2, T), (T - 1, T)):
            r0, r1 = t0 * 64, min(t1 * 64, n)
            mc.upload_rows(c)
            ch = ctx.add_mul_rows(mc, ma, mb, r0, r1, variant)
            exp = c.copy()
            rows = np.arange(r0, r1, dtype=np.uint32)
            exp[r0:r1] = oracle.add_mul_rows(c, a, b, n, rows)
            got = mc.download_rows()
            assert np.array_equal(got, exp), (r0, r1)
            assert ch == (not np.array_equal(exp, c))
        mc.upload_rows(c)  # aliasing: c[rows] |= c[rows] * b uses c from before the call
        exp = c.copy()
        exp[:64] = oracle.add_mul_rows(c, c.copy(), b, n, np.arange(0, 64, dtype=np.uint32))
        ctx.add_mul_rows(mc, mc, mb, 0, 64, variant)
        assert np.array_equal(mc.download_rows(), exp)
        with pytest.raises(Exception):
            ctx.add_mul_rows(mc, ma, mb, 1, 64, variant)  # not a multiple of 64
    finally:
        for m in (ma, mb, mc):
            m.destroy()


def test_block_export_import_and_delta(ctx):
    import torch

    n = 333
    rng = np.random.default_rng(3)
    x, y = rand_rows(rng, n, 0.1), rand_rows(rng, n, 0.1)
    mx, my, md, mp_ = (ctx.matrix(n) for _ in range(4))
    try:
        mx.upload_rows(x)
        my.upload_rows(y)
        size = mx.block_bytes(64, 256)
        assert size == 3 * (6 * 512 + 4 + 6 * 4)
        assert mx.block_bytes(1, 64) == 0
        for dev in ("cuda", "cpu"):
            buf = torch.zeros(size, dtype=torch.uint8, device=dev, pin_memory=dev == "cpu")
            mx.export_block(64, 256, buf.data_ptr())
            ctx.synchronize()
            my.upload_rows(y)
            my.import_block(64, 256, buf.data_ptr())
            exp = y.copy()
            exp[64:256] = x[64:256]
            assert np.array_equal(my.download_rows(), exp)
            occ, nnz = my.tile_stats()
            T = (n + 63) // 64
            padded = np.zeros((T * 64, T), dtype=np.uint64)
            padded[:n] = exp
            assert np.array_equal(nnz, np.bitwise_count(padded).reshape(T, 64, T).sum(axis=1).astype(np.uint32))
        # delta = cur & ~prev, prev = cur
        mp_.upload_rows(y)
        ctx.delta(md, mx, mp_)
        assert np.array_equal(md.download_rows(), x & ~y)
        assert np.array_equal(mp_.download_rows(), x)
        assert md.hash_count()[1] == int(np.bitwise_count(x & ~y).sum())
    finally:
        for m in (mx, my, md, mp_):
            m.destroy()


def _expected(oracle, wl, d):
    gp, rp = os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")
    wl.write(gp, rp)
    with oracle.Problem(gp, rp) as p:
        p.closure(oracle.M4RM, 0)
        return p.results()


def _workload(pkg, name):
    W = pkg.workloads
    return W.chain_query(1100, 5) if name == "chain" else W.ontology_query(1500, 8)


def test_single_process_device_engine(ctx, pkg, oracle, tmp_path):
    for name in ("chain", "same_generation"):
        wl = _workload(pkg, name)
        exp = _expected(oracle, wl, str(tmp_path))
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph, order=None)
        eng = pkg.rowblock.DeviceRowEngine(ctx, q.mats)
        try:
            q.load()
            st = pkg.rowblock.closure(eng, wl.grammar.rules)
            assert dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats))) == exp, name
            assert st.iterations >= 2
        finally:
            eng.close()
            q.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import json
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    pkg = importlib.import_module("cfpq-on-gpgpu_b200")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    ctx = pkg.capi.Context(0)
    try:
        wl = _workload(pkg, "chain")
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph, order=None)
        eng = pkg.rowblock.DeviceRowEngine(ctx, q.mats)
        q.load()
        st = pkg.rowblock.closure(eng, wl.grammar.rules, dist)
        lines = dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats)))
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"lines": {k: list(v) for k, v in lines.items()}, "iterations": st.iterations,
                       "exchanged": st.exchanged_bytes}, f)
        eng.close()
        q.close()
    finally:
        ctx.close()
        dist.destroy_process_group()


def test_two_processes_share_the_gpu(pkg, oracle, tmp_path):
    import json

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    exp = _expected(oracle, _workload(pkg, "chain"), str(tmp_path))
    outs = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for o in outs:
        assert {k: tuple(v) for k, v in o["lines"].items()} == exp
        assert o["exchanged"] > 0
    assert outs[0]["iterations"] == outs[1]["iterations"]
