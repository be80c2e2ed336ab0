"""cfpq_intersection (clear + edge scatter + epsilon diagonals + closure +
result lines, one synchronisation) against the oracle's answer lines and
against the separate calls it replaces: host and device edge arrays, a
grammar with epsilon rules, repeated calls on the same matrices, and the
errors it reports (out-of-range vertex ids, bad epsilon indices)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_lines(oracle, wl, tmp_path):
    gp, rp = str(tmp_path / "g.txt"), str(tmp_path / "r.txt")
    wl.write(gp, rp)
    with oracle.Problem(gp, rp) as p:
        p.closure(oracle.M4RM, 0)
        return p.results()


@pytest.mark.parametrize("where", ["host", "pinned", "device"])
def test_intersection_matches_oracle(ctx, pkg, oracle, tmp_path, where):
    """host: pageable arrays (copied by the call); pinned: page-locked
    arrays, which the scatter kernel reads in place; device: device arrays."""
    import torch

    for wl in (pkg.workloads.ontology_query(1500, 4), pkg.workloads.brackets_query()):
        exp = _oracle_lines(oracle, wl, tmp_path)
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
        g = wl.graph
        try:
            if where == "host":
                arrays = (g.src, g.label, g.dst)
                kw = {}
            elif where == "pinned":
                pinned = [torch.from_numpy(a.view(np.int32)).pin_memory() for a in (g.src, g.label, g.dst)]
                arrays = tuple(t.numpy().view(np.uint32) for t in pinned)
                kw = {}
            else:
                dev = [torch.from_numpy(a.view(np.int32)).cuda() for a in (g.src, g.label, g.dst)]
                torch.cuda.synchronize()
                arrays = tuple(t.data_ptr() for t in dev)
                kw = {"nedges": g.nedges}
            for _ in range(3):  # repeated: the matrices are cleared first, the kept arguments reused
                st, lines = ctx.intersection(wl.grammar.rules, q.mats, *arrays, q.off, q.lm,
                                             epsilon=wl.grammar.epsilon, **kw)
                assert dict(zip(wl.grammar.nonterminals, lines)) == exp
                assert st["iterations"] >= 1
            # without result lines: the matrices hold the closure
            st, none = ctx.intersection(wl.grammar.rules, q.mats, *arrays, q.off, q.lm,
                                        epsilon=wl.grammar.epsilon, lines=False, **kw)
            assert none is None
            assert dict(zip(wl.grammar.nonterminals, ctx.hash_count_many(q.mats))) == exp
        finally:
            q.close()


def test_intersection_epsilon_grammar(ctx, pkg, oracle, tmp_path):
    # Dyck language with the empty word: S -> eps | a S b | S S, in CNF
    wl = pkg.workloads.Workload("dyck_eps", "S\nS A S1\nS1 S B\nS S S\nA a\nB b\n",
                                pkg.workloads.uniform_graph(512, 2048, ["a", "b"], 3), {})
    assert wl.grammar.epsilon, "the grammar has an epsilon rule"
    exp = _oracle_lines(oracle, wl, tmp_path)
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        q.load()
        st_sep, lines_sep = ctx.closure_hash(wl.grammar.rules, q.mats)
        _, lines = ctx.intersection(wl.grammar.rules, q.mats, wl.graph.src, wl.graph.label, wl.graph.dst,
                                    q.off, q.lm, epsilon=wl.grammar.epsilon)
        assert lines == lines_sep
        assert dict(zip(wl.grammar.nonterminals, lines)) == exp
    finally:
        q.close()


def test_intersection_errors(ctx, pkg):
    wl = pkg.workloads.brackets_query()
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    g = wl.graph
    try:
        with pytest.raises(pkg.capi.CfpqError) as e:
            ctx.intersection(wl.grammar.rules, q.mats, g.src, g.label, g.dst, q.off, q.lm, epsilon=[len(q.mats)])
        assert e.value.code == pkg.capi.ERR_INVALID
        bad_dst = g.dst.copy()
        bad_dst[0] = g.n  # one past the last vertex: the scatter's bounds check counts it
        with pytest.raises(pkg.capi.CfpqError) as e:
            ctx.intersection(wl.grammar.rules, q.mats, g.src, g.label, bad_dst, q.off, q.lm,
                             epsilon=wl.grammar.epsilon)
        assert e.value.code == pkg.capi.ERR_INVALID
        assert "out of range" in str(e.value)
        # the context stays usable
        _, lines = ctx.intersection(wl.grammar.rules, q.mats, g.src, g.label, g.dst, q.off, q.lm,
                                    epsilon=wl.grammar.epsilon)
        q.load()
        assert lines == ctx.closure_hash(wl.grammar.rules, q.mats)[1]
    finally:
        q.close()


def test_intersection_empty_graph(ctx, pkg, oracle, tmp_path):
    """No edges: only the epsilon diagonal is set (S -> S S keeps it, the
    other nonterminals stay empty), matching the oracle's line of the n x n
    identity; a later call with the edges gives the full answer on the same
    matrices."""
    graph = pkg.workloads.uniform_graph(200, 600, ["a", "b"], 9)
    wl = pkg.workloads.Workload("dyck_eps", "S\nS A S1\nS1 S B\nS S S\nA a\nB b\n", graph, {})
    n = graph.n
    ident = np.zeros((n, (n + 63) // 64), dtype=np.uint64)
    for v in range(n):
        ident[v, v // 64] |= np.uint64(1) << np.uint64(v % 64)
    exp_empty = {name: (0, 0) for name in wl.grammar.nonterminals}
    exp_empty["S"] = oracle.hash_count(ident, n)
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        z = np.zeros(0, np.uint32)
        _, lines = ctx.intersection(wl.grammar.rules, q.mats, z, z, z, q.off, q.lm, epsilon=wl.grammar.epsilon)
        assert dict(zip(wl.grammar.nonterminals, lines)) == exp_empty
        _, lines = ctx.intersection(wl.grammar.rules, q.mats, graph.src, graph.label, graph.dst, q.off, q.lm,
                                    epsilon=wl.grammar.epsilon)
        assert dict(zip(wl.grammar.nonterminals, lines)) == _oracle_lines(oracle, wl, tmp_path)
    finally:
        q.close()


def test_scatter_hub_vertices_exact_tile_stats(ctx):
    """Edge scatter with hub vertices (one vertex with an edge to every
    other, every vertex with an edge to another hub, duplicates): thousands
    of new bits share a tile-row and tiles, so the population counts and the
    occupancy bits (set once, by the tile's first bit) are checked exactly,
    through cfpq_load_edges and through cfpq_intersection's pinned path."""
    import torch

    n = 3000
    rng = np.random.default_rng(77)
    others = np.arange(n, dtype=np.uint32)
    src = np.concatenate([np.full(n, 5, np.uint32), others, rng.integers(0, n, 4000).astype(np.uint32)])
    dst = np.concatenate([others, np.full(n, 2900, np.uint32), rng.integers(0, n, 4000).astype(np.uint32)])
    src = np.concatenate([src, src[:500]])  # duplicate edges add no bits
    dst = np.concatenate([dst, dst[:500]])
    lab = np.zeros(src.size, np.uint32)
    wpr = (n + 63) // 64
    rows = np.zeros((n, wpr), dtype=np.uint64)
    np.bitwise_or.at(rows, (src, dst // 64), np.left_shift(np.uint64(1), (dst % 64).astype(np.uint64)))
    T = wpr
    padded = np.zeros((T * 64, T), dtype=np.uint64)
    padded[:n] = rows
    exp_nnz = np.bitwise_count(padded).reshape(T, 64, T).sum(axis=1).astype(np.uint32)
    off, lm = np.array([0, 1], np.uint32), np.array([0], np.uint32)

    def check(m):
        assert np.array_equal(m.download_rows(), rows)
        occ, nnz = m.tile_stats()
        assert np.array_equal(nnz, exp_nnz)
        occ_bits = np.unpackbits(occ.view(np.uint8), axis=1, bitorder="little")[:, :T].astype(bool)
        assert np.array_equal(occ_bits, exp_nnz > 0)

    m = ctx.matrix(n)
    try:
        ctx.load_edges([m], src, lab, dst, off, lm)
        check(m)
        ctx.load_edges([m], src, lab, dst, off, lm)  # again on top: nothing new
        check(m)
        pinned = [torch.from_numpy(a.view(np.int32)).pin_memory().numpy().view(np.uint32) for a in (src, lab, dst)]
        st, lines = ctx.intersection([], [m], *pinned, off, lm)
        check(m)
        assert lines == [m.hash_count()]
    finally:
        m.destroy()



def test_intersection_many_nonterminals(ctx, pkg, oracle, tmp_path):
    """A grammar of 20 nonterminals against the oracle: the result lines take
    two hash launches (16 matrices per launch), and the repeated call clears
    the previous closure of all 20 matrices first."""
    labels = ["a", "b", "c"]
    g = pkg.workloads.uniform_graph(700, 2100, labels, 21)
    gram = pkg.workloads.random_cnf(20, 40, labels, 21)
    wl = pkg.workloads.Workload("random_cnf_20", gram, g, {})
    exp = _oracle_lines(oracle, wl, tmp_path)
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        assert len(q.mats) == 20
        for _ in range(2):
            st, lines = ctx.intersection(wl.grammar.rules, q.mats, g.src, g.label, g.dst, q.off, q.lm,
                                         epsilon=wl.grammar.epsilon)
            assert dict(zip(wl.grammar.nonterminals, lines)) == exp
    finally:
        q.close()


def test_intersection_kernel_launch_count(ctx, pkg):
    """kernel_launches counts every kernel the call launches: on the
    persistent path the input phase's first kernel (clear + closure
    prologue), the edge scatter and the closure kernel, plus one hash launch
    when the result lines are asked for."""
    import torch

    wl = pkg.workloads.ontology_query(8192, 1)
    g = wl.graph
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        dev = [torch.from_numpy(a.view(np.int32)).cuda() for a in (g.src, g.label, g.dst)]
        torch.cuda.synchronize()
        ptrs = tuple(t.data_ptr() for t in dev)
        st, _ = ctx.intersection(wl.grammar.rules, q.mats, *ptrs, q.off, q.lm, epsilon=wl.grammar.epsilon,
                                 nedges=g.nedges, lines=False)
        assert st["kernel_launches"] == 3
        st, lines = ctx.intersection(wl.grammar.rules, q.mats, *ptrs, q.off, q.lm, epsilon=wl.grammar.epsilon,
                                     nedges=g.nedges, lines=True)
        assert st["kernel_launches"] == 4
        assert len(lines) == len(q.mats)
    finally:
        q.close()
