"""The large chain workload at full size: N = 65536 (512 MiB per matrix), mean
out-degree 2 with 90% of the edges local, 6 labels, random CNF with 10
nonterminals and 24 binary rules.

A CPU closure at this size takes hours, so parity is checked product by
product on real closure states: the closure (variant AUTO: LOP3, Four
Russians or tensor cores per term and iteration) is stopped after a few
iterations, and rule products C |= A * B of that state are run on the device
with every exact variant and compared bit for bit with the CPU oracle
(the add_mul semantics of m4ri/m4ri_matrix.cpp:20-28) on a row sample."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 65536


@pytest.fixture(scope="module")
def chain(pkg, ctx):
    wl = pkg.workloads.chain_query(N, 1)
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    before = ctx.selector_config()
    ctx.selector_configure(min_tiles=1)  # a single query selects per term (n >= 64 tiles)
    try:
        yield wl, q
    finally:
        ctx.selector_configure(**{k: before[k] for k in ("mode", "min_tiles", "tc_min_tiles")})
        q.close()


def _sample_rows(rng):
    # a seeded sample plus the first and last rows and two tile-row boundaries
    extra = np.array([0, 63, 64, N // 2, N - 65, N - 1], dtype=np.int64)
    return np.unique(np.concatenate([rng.choice(N, 58, replace=False), extra])).astype(np.uint32)


def test_chain65536_products_of_a_closure_state_match_oracle(ctx, pkg, oracle, chain):
    wl, q = chain
    rules = wl.grammar.rules
    q.load()
    st = ctx.closure(rules, q.mats, variant="auto", max_iterations=3)
    assert st["iterations"] == 3
    rng = np.random.default_rng(N)
    rows = _sample_rows(rng)
    tmp = ctx.matrix(N)
    try:
        # three rules of the grammar, chosen by a seeded draw among those whose
        # operands hold bits in this state
        cand = [r for r in range(len(rules)) if all(q.mats[i].hash_count()[1] for i in rules[r][1:])]
        assert len(cand) >= 3
        for r in rng.choice(cand, 3, replace=False):
            head, b1, b2 = rules[int(r)]
            A, B, C = (q.mats[i].download_rows() for i in (b1, b2, head))
            exp = oracle.add_mul_rows(C, A, B, N, rows)
            grows = not np.array_equal(exp, C[rows])
            del A, B
            for variant in ("lop3", "m4r", "tc"):
                tmp.copy_from(q.mats[head])
                changed = ctx.add_mul(tmp, q.mats[b1], q.mats[b2], variant)
                got = tmp.download_rows()
                assert np.array_equal(got[rows], exp), (int(r), variant)
                assert not np.any(C & ~got), (int(r), variant)  # C only grows
                if grows:
                    assert changed, (int(r), variant)
                del got
    finally:
        tmp.destroy()
