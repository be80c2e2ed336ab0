"""Result lines: the batched hash launch (cfpq_hash_count_many over more
matrices than one launch takes, of different sizes) against one matrix at a
time, and cfpq_closure_hash (closure and lines with one synchronisation)
against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_hash_count_many_matches_single(ctx):
    rng = np.random.default_rng(8)
    sizes = [1, 2, 63, 64, 65, 130, 200, 257, 640, 1000, 0, 64, 333, 1, 700, 90, 129, 128, 511, 64, 1030]
    mats = []
    try:
        for n in sizes:
            m = ctx.matrix(n)
            if n:
                k = max(1, n * 2)
                m.set_bits(rng.integers(0, n, k).astype(np.uint32), rng.integers(0, n, k).astype(np.uint32))
            mats.append(m)
        assert len(mats) > 16  # two launches
        many = ctx.hash_count_many(mats)
        assert many == [m.hash_count() for m in mats]
        assert many[10] == (0, 0)
    finally:
        for m in mats:
            m.destroy()


@pytest.mark.parametrize("loop", ["device", "graph", "host"])
def test_closure_hash_matches_oracle(ctx, pkg, oracle, tmp_path, loop):
    for wl in (pkg.workloads.ontology_query(1500, 4), pkg.workloads.brackets_query()):
        gp, rp = str(tmp_path / "g.txt"), str(tmp_path / "r.txt")
        wl.write(gp, rp)
        with oracle.Problem(gp, rp) as p:
            p.closure(oracle.M4RM, 0)
            exp = p.results()
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
        try:
            for _ in range(2):  # the second call reuses the kept arguments
                q.load()
                st, lines = ctx.closure_hash(wl.grammar.rules, q.mats, use_graph=loop)
                assert dict(zip(wl.grammar.nonterminals, lines)) == exp
                assert st["iterations"] > 1
        finally:
            q.close()


def test_hash_count_many_empty_launch(ctx):
    """A launch whose matrices are all of size 0 (the 17th matrix, alone in
    the second launch) gives (0, 0) without a kernel; the first launch's
    lines are unaffected."""
    rng = np.random.default_rng(9)
    mats = []
    try:
        for i in range(16):
            m = ctx.matrix(100 + 37 * i)
            m.set_bits(rng.integers(0, m.n, 300).astype(np.uint32), rng.integers(0, m.n, 300).astype(np.uint32))
            mats.append(m)
        mats.append(ctx.matrix(0))
        many = ctx.hash_count_many(mats)
        assert many[16] == (0, 0)
        assert many[:16] == [m.hash_count() for m in mats[:16]]
    finally:
        for m in mats:
            m.destroy()

