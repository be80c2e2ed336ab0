"""The nonterminal-set variant (CFPQ_VARIANT_NTSET): the whole closure as one
matrix of nonterminal sets squared until it stops changing (the reference's
single-matrix formulation, cuda/cutlass/CutlassMatrix.cu:290-316).  Its
fixpoint must equal the per-nonterminal closure bit for bit: whole matrices
against the oracle, the golden answers, 1-byte cells (<= 8 nonterminals) and
4-byte cells (up to 32), vertex orders, and the size limits."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _oracle(oracle, wl, d):
    gp, rp = str(d / "grammar.txt"), str(d / "graph.txt")
    wl.write(gp, rp)
    with oracle.Problem(gp, rp) as p:
        p.closure(oracle.M4RM, 0)
        return p.results(), dict(zip(p.names, (p.matrix(i) for i in range(len(p.names)))))


def _run(ctx, pkg, wl, order=None):
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph, order=order)
    try:
        q.load()
        st = ctx.closure(wl.grammar.rules, q.mats, variant="ntset")
        lines = dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats)))
        mats = {nt: m.download_rows() for nt, m in zip(q.grammar.nonterminals, q.mats)}
        return st, lines, mats, q
    except Exception:
        q.close()
        raise


@pytest.mark.parametrize("case", ["brackets_1024", "same_generation_700", "random_cnf8_600", "chain10_900",
                                  "random_cnf20_300"])
def test_ntset_matches_oracle(ctx, pkg, oracle, tmp_path, case):
    W = pkg.workloads
    wl = {"brackets_1024": lambda: W.brackets_query(),
          "same_generation_700": lambda: W.ontology_query(700, 3),
          "random_cnf8_600": lambda: W.Workload("random_cnf", W.random_cnf(8, 20, ["x", "y", "z"], 5),
                                               W.uniform_graph(600, 1500, ["x", "y", "z"], 5), {}),
          "chain10_900": lambda: W.chain_query(900, 4),  # 10 nonterminals: 4-byte cells
          "random_cnf20_300": lambda: W.Workload("random_cnf", W.random_cnf(20, 40, ["a", "b", "c", "d"], 9),
                                                W.uniform_graph(300, 700, ["a", "b", "c", "d"], 9), {}),
          }[case]()
    exp_lines, exp_mats = _oracle(oracle, wl, tmp_path)
    st, lines, mats, q = _run(ctx, pkg, wl)
    try:
        assert lines == exp_lines
        for nt, m in mats.items():
            assert np.array_equal(m, exp_mats[nt]), nt
        assert st["iterations"] >= 1
        # tile statistics rebuilt exactly after the unpack
        for nt, m in zip(q.grammar.nonterminals, q.mats):
            occ, nnz = m.tile_stats()
            n, T = m.n, (m.n + 63) // 64
            padded = np.zeros((T * 64, T), dtype=np.uint64)
            padded[:n] = mats[nt]
            assert np.array_equal(nnz, np.bitwise_count(padded).reshape(T, 64, T).sum(axis=1).astype(np.uint32))
        # a second closure on the closed matrices changes nothing and takes one pass
        st2 = ctx.closure(q.grammar.rules, q.mats, variant="ntset")
        assert st2["iterations"] == 1
        assert dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats))) == exp_lines
    finally:
        q.close()


def test_ntset_with_vertex_order(ctx, pkg, oracle, tmp_path):
    wl = pkg.workloads.ontology_query(1024, 6)
    exp_lines, _ = _oracle(oracle, wl, tmp_path)
    st, lines, _, q = _run(ctx, pkg, wl, order="auto")
    q.close()
    assert lines == exp_lines


GOLDEN_CASES = sorted(d for d in os.listdir(GOLDEN) if os.path.isdir(os.path.join(GOLDEN, d)))


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_ntset_golden(ctx, pkg, oracle, case):
    d = os.path.join(GOLDEN, case)
    gp, rp = os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")
    expected = oracle.parse_answer(open(os.path.join(d, "expected.txt")).read())
    grammar, graph = pkg.query.CnfGrammar.from_file(gp), pkg.query.EdgeGraph.from_file(rp)
    q = pkg.query.PreparedQuery(ctx, grammar, graph)
    try:
        q.load()
        ctx.closure(grammar.rules, q.mats, variant="ntset")
        assert dict(zip(grammar.nonterminals, ctx.hash_count_many(q.mats))) == expected
    finally:
        q.close()


def test_ntset_limits(ctx, pkg):
    capi = pkg.capi
    mats = [ctx.matrix(64) for _ in range(33)]
    try:
        with pytest.raises(capi.CfpqError) as e:
            ctx.closure([(0, 1, 2)], mats, variant="ntset")
        assert e.value.code == capi.ERR_UNSUPPORTED
    finally:
        for m in mats:
            m.destroy()
    big = [ctx.matrix(16448) for _ in range(2)]
    try:
        with pytest.raises(capi.CfpqError) as e:
            ctx.closure([(0, 1, 1)], big, variant="ntset")
        assert e.value.code == capi.ERR_UNSUPPORTED
    finally:
        for m in big:
            m.destroy()
    with pytest.raises(capi.CfpqError) as e:  # closure-only variant
        a = ctx.matrix(64)
        try:
            ctx.add_mul(a, a, a, "ntset")
        finally:
            a.destroy()
    assert e.value.code == capi.ERR_UNSUPPORTED
