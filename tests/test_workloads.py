"""Seeded workload generators and the Python loaders (no GPU)."""
import numpy as np
import pytest


def test_generators_are_deterministic(pkg):
    W = pkg.workloads
    for make in (lambda: W.brackets_query(), lambda: W.ontology_query(1024, 3),
                 lambda: W.chain_query(4096, 2), lambda: W.batch_queries(6, 4)[5]):
        a, b = make(), make()
        assert a.grammar_text == b.grammar_text
        for f in ("src", "label", "dst"):
            assert np.array_equal(getattr(a.graph, f), getattr(b.graph, f))


def test_brackets_config_shape(pkg):
    wl = pkg.workloads.brackets_query()
    assert wl.graph.n == 1024 and wl.graph.nedges == 4096
    assert set(wl.graph.labels) == {"a", "b"}
    g = wl.grammar
    assert len(g.nonterminals) == 4 and len(g.rules) == 3


def test_ontology_config_shape(pkg):
    wl = pkg.workloads.ontology_query(8192, 1)
    g = wl.graph
    assert g.n == 8192
    assert set(g.labels) == {"subClassOf", "type", "subClassOf_r", "type_r"}
    forward = g.nedges // 2
    assert 2.0 <= forward / g.n <= 4.0  # mean out-degree ~3
    gram = wl.grammar
    assert len(gram.nonterminals) == 7 and len(gram.rules) == 6
    # every edge has its inverse
    lab = np.asarray(g.labels)[g.label]
    fwd = {(a, l, b) for a, l, b in zip(g.src.tolist(), lab.tolist(), g.dst.tolist()) if not l.endswith("_r")}
    inv = {(b, l[:-2], a) for a, l, b in zip(g.src.tolist(), lab.tolist(), g.dst.tolist()) if l.endswith("_r")}
    assert fwd == inv


def test_ontology_subclass_dag_depth(pkg):
    g = pkg.workloads.ontology_graph(4096, 2)
    lab = np.asarray(g.labels)[g.label]
    sc = [(a, b) for a, l, b in zip(g.src.tolist(), lab.tolist(), g.dst.tolist()) if l == "subClassOf"]
    parents = {}
    for c, p in sc:
        parents.setdefault(c, []).append(p)
    depth = {}

    def d(v):
        if v not in depth:
            depth[v] = 1 + max((d(p) for p in parents.get(v, [])), default=0)
        return depth[v]

    assert max(d(v) for v in parents) <= 12


def test_chain_config_shape(pkg):
    wl = pkg.workloads.chain_query(8192, 5)
    g = wl.graph
    assert g.n == 8192 and abs(g.nedges - 2 * 8192) <= 1
    local = np.abs(g.src.astype(np.int64) - g.dst.astype(np.int64)) <= 64
    assert 0.85 < local.mean() < 0.95
    gram = wl.grammar
    assert len(gram.nonterminals) == 10 and len(gram.rules) == 24
    assert len(g.labels) == 6


def test_batch_config_shape(pkg):
    qs = pkg.workloads.batch_queries(64, 9)
    ns = np.array([q.graph.n for q in qs])
    assert ns.min() >= 256 and ns.max() <= 8192
    assert {q.name for q in qs} == {"brackets", "same_generation", "random_cnf"}
    for q in qs:
        if q.name == "random_cnf":
            assert len(q.grammar.rules) == 20 and len(q.grammar.nonterminals) == 8


def test_text_formats_round_trip(pkg, oracle, tmp_path):
    wl = pkg.workloads.ontology_query(512, 8)
    gp, rp = str(tmp_path / "g.txt"), str(tmp_path / "r.txt")
    wl.write(gp, rp)
    g2 = pkg.query.EdgeGraph.from_file(rp)
    lab1 = np.asarray(wl.graph.labels)[wl.graph.label]
    lab2 = np.asarray(g2.labels)[g2.label]
    assert g2.n == wl.graph.n and np.array_equal(g2.src, wl.graph.src) and np.array_equal(g2.dst, wl.graph.dst)
    assert np.array_equal(lab1, lab2)
    gram = pkg.query.CnfGrammar.from_file(gp)
    with oracle.Problem(gp, rp) as p:
        assert p.names == gram.nonterminals
        assert p.rules == gram.rules
        assert p.n == g2.n


def test_python_grammar_parser_matches_reference_rules():
    import importlib

    q = importlib.import_module("cfpq-on-gpgpu_b200").query
    g = q.CnfGrammar.from_text("S A B\n\nB b\nX y z w\nA a\nE\n")
    assert g.nonterminals == ["S", "A", "B", "X", "E"]
    assert g.rules == [(0, 1, 2)]
    assert g.terminal_to_nts == {"b": [2], "a": [1]}
    assert g.epsilon == [4]
