"""The bounded device waits of the persistent closure kernel, made to run out
without any fault: the CFPQ_TEST_STALL_BARRIER hook has the first grid
barrier wait for one arrival more than there are CTAs (a count that nothing
completes), and a short wait limit makes the poll give up quickly.  The
closure must return CFPQ_ERR_TIMEOUT, leave only true bits in the matrices,
and the same context must then close queries correctly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _answer(oracle, wl, tmp_path):
    gp, rp = str(tmp_path / "grammar.txt"), str(tmp_path / "graph.txt")
    wl.write(gp, rp)
    with oracle.Problem(gp, rp) as p:
        p.closure(oracle.M4RM, 0)
        return p.results(), [p.matrix(i) for i in range(len(p.names))], p.names


@pytest.mark.parametrize("wait_limit", [64, 4096])
def test_stalled_barrier_reports_timeout_and_context_recovers(ctx, pkg, oracle, tmp_path, wait_limit):
    capi = pkg.capi
    wl = pkg.workloads.ontology_query(1024, 2)
    exp_lines, exp_mats, names = _answer(oracle, wl, tmp_path)
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        q.load()
        with pytest.raises(capi.CfpqError) as err:
            ctx.closure(wl.grammar.rules, q.mats, use_graph="device", wait_limit=wait_limit,
                        test_flags=capi.TEST_STALL_BARRIER)
        assert err.value.code == capi.ERR_TIMEOUT
        # what the aborted closure set is a subset of the least fixpoint
        by_name = dict(zip(names, exp_mats))
        for nt, m in zip(q.grammar.nonterminals, q.mats):
            got = m.download_rows()
            assert not np.any(got & ~by_name[nt]), nt
        # the same context, the same prepared query: a normal closure is exact
        for _ in range(2):
            q.load()
            st = ctx.closure(wl.grammar.rules, q.mats, use_graph="device")
            assert dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats))) == exp_lines
            assert st["iterations"] > 1
    finally:
        q.close()


def test_timeout_in_a_batch_then_batch_recovers(ctx, pkg, oracle, tmp_path):
    wls = pkg.workloads.batch_queries(6, seed=9, n_min=128, n_max=600)
    exps = []
    for i, wl in enumerate(wls):
        d = tmp_path / f"q{i}"
        d.mkdir()
        exps.append(_answer(oracle, wl, d)[0])
    qs = [pkg.query.PreparedQuery(ctx, w.grammar, w.graph) for w in wls]
    try:
        for q in qs:
            q.load()
        # a timed-out closure between two uses of the batch's buffers
        single = qs[0]
        with pytest.raises(pkg.capi.CfpqError) as err:
            ctx.closure(single.grammar.rules, single.mats, use_graph="device", wait_limit=256,
                        test_flags=pkg.capi.TEST_STALL_BARRIER)
        assert err.value.code == pkg.capi.ERR_TIMEOUT
        for q in qs:
            q.load()
        ctx.closure_batch([(q.grammar.rules, q.mats) for q in qs], use_graph="device")
        for q, exp in zip(qs, exps):
            assert dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats))) == exp
    finally:
        for q in qs:
            q.close()
