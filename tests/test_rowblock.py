"""Row-block closure of one query over several processes (rowblock.py), on
CPU: world-size 2 and 3 gloo runs in which every rank computes its rows with
a CPU engine (the oracle's row-sample product), exchange through the same
driver code as on GPUs, and the result equals the single-process oracle
closure bit for bit."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def initial_rows(pkg, wl):
    """Row-bit matrices of a query after the edge scatter and the epsilon
    diagonals (cfpq-cpp/Grammar.h:41-51), in the package's nonterminal order."""
    g, gr = wl.graph, wl.grammar
    off, lm = pkg.query.label_map(gr, g)
    n, wpr = g.n, (g.n + 63) // 64
    mats = [np.zeros((n, wpr), dtype=np.uint64) for _ in gr.nonterminals]
    for s, l, d in zip(g.src.tolist(), g.label.tolist(), g.dst.tolist()):
        if l + 1 >= len(off):
            continue
        for m in lm[off[l]:off[l + 1]].tolist():
            mats[m][s, d // 64] |= np.uint64(1) << np.uint64(d % 64)
    for e in gr.epsilon:
        for i in range(n):
            mats[e][i, i // 64] |= np.uint64(1) << np.uint64(i % 64)
    return mats


class HostRowEngine:
    """CPU engine for the row-block driver: row-bit matrices in host memory,
    products of a row range by the oracle (test infrastructure only)."""

    device = "cpu"

    def __init__(self, oracle, mats):
        self.oracle, self.mats = oracle, mats
        self.n = mats[0].shape[0]
        self.nmats = len(mats)
        self.prev = [np.zeros_like(m) for m in mats]
        self.delta = [np.zeros_like(m) for m in mats]

    def block_bytes(self, r0, r1):
        return (r1 - r0) * self.mats[0].shape[1] * 8

    def begin_iteration(self):
        for x in range(self.nmats):
            self.delta[x] = self.mats[x] & ~self.prev[x]
            self.prev[x] = self.mats[x].copy()

    def product(self, head, b1, b2, term, r0, r1):
        if r1 <= r0:
            return False
        a = self.delta[b1] if term == 0 else self.mats[b1]
        b = self.mats[b2] if term == 0 else self.delta[b2]
        rows = np.arange(r0, r1, dtype=np.uint32)
        new = self.oracle.add_mul_rows(self.mats[head], np.ascontiguousarray(a), np.ascontiguousarray(b), self.n, rows)
        changed = not np.array_equal(new, self.mats[head][r0:r1])
        self.mats[head][r0:r1] = new
        return changed

    def export(self, m, r0, r1, buf):
        raw = np.ascontiguousarray(self.mats[m][r0:r1]).view(np.uint8).reshape(-1)
        buf[:raw.size] = __import__("torch").from_numpy(raw)

    def import_(self, m, r0, r1, buf):
        k = (r1 - r0) * self.mats[0].shape[1] * 8
        self.mats[m][r0:r1] = buf[:k].numpy().view(np.uint64).reshape(r1 - r0, -1)

    def sync(self):
        pass


def workload(pkg, name):
    W = pkg.workloads
    if name == "brackets":
        return W.brackets_query(n=700, nedges=2200, seed=4)
    if name == "chain":
        return W.chain_query(650, 2)
    labels = ["x", "y", "z"]
    return W.Workload("random_cnf", W.random_cnf(8, 20, labels, 13), W.uniform_graph(500, 1300, labels, 13), {})


def expected(oracle, wl, d):
    gp, rp = os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")
    wl.write(gp, rp)
    with oracle.Problem(gp, rp) as p:
        p.closure(oracle.M4RM, 1)
        return p.results(), dict(zip(p.names, (p.matrix(i) for i in range(len(p.names)))))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, outdir):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle

    pkg = importlib.import_module("cfpq-on-gpgpu_b200")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        wl = workload(pkg, name)
        eng = HostRowEngine(oracle, initial_rows(pkg, wl))
        st = pkg.rowblock.closure(eng, wl.grammar.rules, dist)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), *eng.mats, iterations=st.iterations,
                 exchanged=st.exchanged_bytes)
    finally:
        dist.destroy_process_group()


def test_row_blocks_partition():
    rb = importlib.import_module("cfpq-on-gpgpu_b200.rowblock")
    for n, world in ((1, 1), (64, 2), (700, 3), (8192, 8), (130, 4), (0, 2)):
        blocks = rb.row_blocks(n, world)
        assert len(blocks) == world
        assert blocks[0][0] == 0 and blocks[-1][1] == n
        for (a, b), (c, _) in zip(blocks, blocks[1:]):
            assert b == c and a <= b
        assert all((a % 64 == 0 or a == b == n) and (b % 64 == 0 or b == n) for a, b in blocks)


def test_single_process_matches_oracle(pkg, oracle, tmp_path):
    wl = workload(pkg, "random_cnf")
    exp_lines, exp_mats = expected(oracle, wl, str(tmp_path))
    eng = HostRowEngine(oracle, initial_rows(pkg, wl))
    st = pkg.rowblock.closure(eng, wl.grammar.rules)
    for nt, m in zip(wl.grammar.nonterminals, eng.mats):
        assert np.array_equal(m, exp_mats[nt]), nt
    assert st.iterations >= 2 and st.exchanged_bytes == 0


@pytest.mark.parametrize("world,name", [(2, "brackets"), (2, "random_cnf"), (3, "chain")])
def test_multi_rank_matches_single_process(pkg, oracle, tmp_path, world, name):
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, name, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    wl = workload(pkg, name)
    _, exp_mats = expected(oracle, wl, str(tmp_path))
    its = set()
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npz")
        its.add(int(got["iterations"]))
        for i, nt in enumerate(wl.grammar.nonterminals):
            assert np.array_equal(got[f"arr_{i}"], exp_mats[nt]), (r, nt)  # every rank holds the whole fixpoint
        assert int(got["exchanged"]) > 0
    assert len(its) == 1  # the ranks stop together
