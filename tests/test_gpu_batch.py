"""The 512-query mixed batch at full size (N log-uniform in [256, 8192], three
grammar families) closed on the GPU in one cfpq_closure_batch, compared with
the answer lines the reference's m4riCPU printed for every query
(tests/golden/batch512_seed1.txt); and a slice closed one query at a time."""
import importlib.util
import os

import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch(pkg):
    spec = importlib.util.spec_from_file_location("make_batch_golden", os.path.join(GOLDEN, "make_batch_golden.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    return mk.read_fixture(os.path.join(GOLDEN, "batch512_seed1.txt")), mk.batch_workloads()


def _lines(ctx, q):
    return dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats)))


@pytest.mark.parametrize("loop", ["device", "graph"])
def test_full_batch_matches_reference_answers(ctx, pkg, batch, loop):
    fx, wls = batch
    qs = [pkg.query.PreparedQuery(ctx, w.grammar, w.graph) for w in wls]
    try:
        for q in qs:
            q.load()
        st, iters, done = ctx.closure_batch([(q.grammar.rules, q.mats) for q in qs], use_graph=loop)
        bad = [i for i, q in enumerate(qs) if _lines(ctx, q) != fx[i]["lines"]]
        assert not bad, f"{len(bad)} of {len(qs)} queries differ, first {bad[:8]}"
        assert st["iterations"] >= int(iters.max()) > 0
    finally:
        for q in qs:
            q.close()


def test_largest_queries_one_at_a_time(ctx, pkg, batch):
    """The 16 largest queries of the batch, each closed alone (the sequential
    baseline of the batch bench), give the same answers."""
    fx, wls = batch
    largest = sorted(range(len(wls)), key=lambda i: -wls[i].graph.n)[:16]
    for i in largest:
        q = pkg.query.PreparedQuery(ctx, wls[i].grammar, wls[i].graph)
        try:
            q.load()
            ctx.closure(q.grammar.rules, q.mats)
            assert _lines(ctx, q) == fx[i]["lines"], i
        finally:
            q.close()
