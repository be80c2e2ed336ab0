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


@pytest.mark.parametrize("where", ["host", "device"])
def test_intersection_matches_oracle(ctx, pkg, oracle, tmp_path, where):
    import torch

    for wl in (pkg.workloads.ontology_query(1500, 4), pkg.workloads.brackets_query()):
        exp = _oracle_lines(oracle, wl, tmp_path)
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
        g = wl.graph
        try:
            if where == "host":
                arrays = (g.src, g.label, g.dst)
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
