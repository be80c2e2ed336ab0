"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bit-exact comparisons: whole matrices (row bits), changed flags and the
reference result lines (name, hash, count)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 63, 64, 65, 127, 130, 257, 640, 1000, 1100]


def rand_rows(rng, n, density):
    wpr = (n + 63) // 64
    bits = rng.random((n, wpr * 64)) < density
    bits[:, n:] = False
    return np.packbits(bits, axis=1, bitorder="little").view(np.uint64).reshape(n, wpr).copy()


def upload(ctx, n, rows):
    m = ctx.matrix(n)
    m.upload_rows(rows)
    return m


def tile_popcounts(rows, n):
    T = (n + 63) // 64
    padded = np.zeros((T * 64, T), dtype=np.uint64)
    padded[:n] = rows
    return np.bitwise_count(padded).reshape(T, 64, T).sum(axis=1).astype(np.uint32)


def check_tile_stats(m, rows):
    """The engine's tile populations are exact and occupancy covers every non-empty tile."""
    occ, nnz = m.tile_stats()
    exp = tile_popcounts(rows, m.n)
    assert np.array_equal(nnz, exp)
    T = exp.shape[0]
    occ_bits = np.unpackbits(occ.view(np.uint8), axis=1, bitorder="little")[:, :T].astype(bool)
    assert not np.any((exp > 0) & ~occ_bits)


@pytest.mark.parametrize("variant", ["plain", "lop3", "m4r"])
@pytest.mark.parametrize("n", SIZES)
def test_add_mul_random(ctx, oracle, variant, n):
    rng = np.random.default_rng(n * 7 + len(variant))
    for density in (0.002, 0.05, 0.4):
        a, b, c = (rand_rows(rng, n, d) for d in (density, density, density / 2))
        ma, mb, mc = upload(ctx, n, a), upload(ctx, n, b), upload(ctx, n, c)
        exp = c.copy()
        ch_exp = oracle.add_mul(exp, a, b, n, oracle.NAIVE, 1)
        ch = ctx.add_mul(mc, ma, mb, variant)
        got = mc.download_rows()
        assert np.array_equal(got, exp), f"n={n} density={density}"
        assert ch == ch_exp
        check_tile_stats(mc, exp)
        # a second identical product cannot change anything
        assert ctx.add_mul(mc, ma, mb, variant) is False
        for m in (ma, mb, mc):
            m.destroy()


@pytest.mark.parametrize("variant", ["plain", "lop3", "m4r"])
@pytest.mark.parametrize("alias", ["a", "b", "ab"])
def test_add_mul_aliasing(ctx, oracle, variant, alias):
    n = 200
    rng = np.random.default_rng(11)
    a, b, c = rand_rows(rng, n, 0.03), rand_rows(rng, n, 0.03), rand_rows(rng, n, 0.03)
    mc = upload(ctx, n, c)
    if alias == "a":
        ma, mb = mc, upload(ctx, n, b)
        exp = c.copy()
        ch_exp = oracle.add_mul(exp, c.copy(), b, n)
    elif alias == "b":
        ma, mb = upload(ctx, n, a), mc
        exp = c.copy()
        ch_exp = oracle.add_mul(exp, a, c.copy(), n)
    else:
        ma = mb = mc
        exp = c.copy()
        ch_exp = oracle.add_mul(exp, c.copy(), c.copy(), n)
    ch = ctx.add_mul(mc, ma, mb, variant)
    assert np.array_equal(mc.download_rows(), exp)
    assert ch == ch_exp


@pytest.mark.parametrize("n", [1, 64, 65, 300, 1024])
def test_hash_count(ctx, oracle, n):
    rng = np.random.default_rng(n)
    for density in (0.0, 0.01, 0.5, 1.0):
        rows = rand_rows(rng, n, density)
        m = upload(ctx, n, rows)
        assert m.hash_count() == oracle.hash_count(rows, n)
        m.destroy()


def test_hash_count_large_ragged(ctx, oracle):
    """The result-line hash (one block per tile-row, subset-sum lookups of
    the column powers per row byte) on a ragged n = 20000 (313 tile-rows, 10
    occupancy words per row): scattered bits plus some dense blocks, and the
    single-matrix and batched entry points against the oracle."""
    n = 20000
    rng = np.random.default_rng(20000)
    wpr = (n + 63) // 64
    rows = np.zeros((n, wpr), dtype=np.uint64)
    r = rng.integers(0, n, 300000)
    c = rng.integers(0, n, 300000)
    np.bitwise_or.at(rows, (r, c // 64), np.left_shift(np.uint64(1), (c % 64).astype(np.uint64)))
    rows[4000:4200, 30:40] = np.uint64(0xFFFFFFFFFFFFFFFF)   # dense blocks, a full tile-row stripe
    rows[19990:20000, wpr - 1] = np.uint64((1 << (n % 64)) - 1)  # last columns of the last rows
    m = upload(ctx, n, rows)
    try:
        exp = oracle.hash_count(rows, n)
        assert m.hash_count() == exp
        assert ctx.hash_count_many([m, m]) == [exp, exp]
    finally:
        m.destroy()


def test_upload_download_roundtrip(ctx):
    rng = np.random.default_rng(3)
    for n in (1, 64, 77, 1000):
        rows = rand_rows(rng, n, 0.3)
        m = upload(ctx, n, rows)
        assert np.array_equal(m.download_rows(), rows)
        m.destroy()


def test_set_bits_and_diagonal(ctx, oracle):
    n = 333
    rng = np.random.default_rng(5)
    r = rng.integers(0, n, 500)
    c = rng.integers(0, n, 500)
    m = ctx.matrix(n)
    m.set_bits(r, c)
    m.set_diagonal()
    exp = np.zeros((n, (n + 63) // 64), dtype=np.uint64)
    for i, j in list(zip(r, c)) + [(i, i) for i in range(n)]:
        exp[i, j // 64] |= np.uint64(1) << np.uint64(j % 64)
    assert np.array_equal(m.download_rows(), exp)
    m.destroy()


@pytest.mark.parametrize("n", [1, 63, 130, 700])
def test_ordered_matrices(ctx, pkg, oracle, n):
    """Matrices stored under a vertex relabeling behave exactly like unordered ones."""
    rng = np.random.default_rng(n + 99)
    order = ctx.order(rng.permutation(n).astype(np.uint32))
    a, b, c = rand_rows(rng, n, 0.03), rand_rows(rng, n, 0.03), rand_rows(rng, n, 0.01)
    ma, mb, mc = (ctx.matrix(n, order) for _ in range(3))
    for m, rows in ((ma, a), (mb, b), (mc, c)):
        m.upload_rows(rows)
        assert np.array_equal(m.download_rows(), rows)
        assert m.hash_count() == oracle.hash_count(rows, n)
    exp = c.copy()
    ch_exp = oracle.add_mul(exp, a, b, n)
    for variant in ("lop3", "plain", "m4r"):
        mc.upload_rows(c)
        assert ctx.add_mul(mc, ma, mb, variant) == ch_exp
        assert np.array_equal(mc.download_rows(), exp)
        assert mc.hash_count() == oracle.hash_count(exp, n)
    r, cc = rng.integers(0, n, 50), rng.integers(0, n, 50)
    md = ctx.matrix(n, order)
    md.set_bits(r, cc)
    md.set_diagonal()
    expd = np.zeros((n, (n + 63) // 64), dtype=np.uint64)
    for i, j in list(zip(r, cc)) + [(i, i) for i in range(n)]:
        expd[i, j // 64] |= np.uint64(1) << np.uint64(j % 64)
    assert np.array_equal(md.download_rows(), expd)
    plain = ctx.matrix(n)
    with pytest.raises(pkg.capi.CfpqError):
        ctx.add_mul(plain, ma, mb)
    for m in (ma, mb, mc, md, plain):
        m.destroy()
    order.destroy()


def test_set_bits_out_of_range_is_an_error(ctx, pkg):
    m = ctx.matrix(10)
    with pytest.raises(pkg.capi.CfpqError) as e:
        m.set_bits([1, 10], [2, 3])
    assert e.value.code == pkg.capi.ERR_INVALID
    m.destroy()


def _write(wl, tmp_path):
    gp, rp = str(tmp_path / "grammar.txt"), str(tmp_path / "graph.txt")
    wl.write(gp, rp)
    return gp, rp


def _oracle_run(oracle, gp, rp):
    with oracle.Problem(gp, rp) as p:
        p.closure(oracle.M4RM, 0)
        return p.results(), [p.matrix(i) for i in range(len(p.names))], p.names


def _check_query(ctx, pkg, oracle, wl, tmp_path, order="auto", **kw):
    gp, rp = _write(wl, tmp_path)
    exp_lines, exp_mats, names = _oracle_run(oracle, gp, rp)
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph, order=order)
    try:
        res = q.run(**kw)
        assert res.lines == exp_lines
        assert q.grammar.nonterminals == names
        for i, m in enumerate(q.mats):
            assert np.array_equal(m.download_rows(), exp_mats[i]), names[i]
            if q.order is None:
                check_tile_stats(m, exp_mats[i])
        return res
    finally:
        q.close()


@pytest.mark.parametrize("kw", [dict(driver="engine", use_graph=True), dict(driver="engine", use_graph=False),
                                dict(driver="worklist", variant="plain"),
                                dict(driver="worklist", variant="lop3"),
                                dict(driver="engine", variant="m4r"),
                                dict(driver="worklist", variant="m4r")])
def test_closure_brackets_full_size(ctx, pkg, oracle, tmp_path, kw):
    wl = pkg.workloads.brackets_query()  # N=1024, 4096 edges
    res = _check_query(ctx, pkg, oracle, wl, tmp_path, **kw)
    if kw["driver"] == "engine":
        assert res.stats["iterations"] > 1


@pytest.mark.parametrize("order", ["auto", None])
@pytest.mark.parametrize("n,seed", [(512, 3), (2048, 4), (8192, 1)])
def test_closure_same_generation(ctx, pkg, oracle, tmp_path, n, seed, order):
    wl = pkg.workloads.ontology_query(n, seed)
    _check_query(ctx, pkg, oracle, wl, tmp_path, order=order)


@pytest.mark.parametrize("variant", ["lop3", "m4r"])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_closure_random_cnf(ctx, pkg, oracle, tmp_path, seed, variant):
    labels = ["x", "y", "z"]
    g = pkg.workloads.uniform_graph(700, 1400, labels, seed)
    gram = pkg.workloads.random_cnf(8, 20, labels, seed)
    wl = pkg.workloads.Workload("random_cnf", gram, g, {})
    _check_query(ctx, pkg, oracle, wl, tmp_path, variant=variant)


@pytest.mark.parametrize("loop", ["device", "graph", "host"])
@pytest.mark.parametrize("variant", ["lop3", "m4r"])
def test_closure_loop_modes(ctx, pkg, oracle, tmp_path, loop, variant):
    """The persistent kernel (device), the CUDA-graph loop and the host loop
    sequence the same plan / product code and agree with the oracle."""
    labels = ["x", "y", "z"]
    g = pkg.workloads.uniform_graph(900, 2000, labels, 11)
    gram = pkg.workloads.random_cnf(8, 20, labels, 11)
    wl = pkg.workloads.Workload("random_cnf", gram, g, {})
    res = _check_query(ctx, pkg, oracle, wl, tmp_path, variant=variant, use_graph=loop)
    assert res.stats["iterations"] > 1
    if loop == "device":
        assert res.stats["kernel_launches"] == 2  # mark + one persistent launch


def test_closure_iteration_limit_then_full(ctx, pkg, oracle, tmp_path):
    """A closure cut off by max_iterations leaves the context usable: the
    next full closure of the same query is exact."""
    wl = pkg.workloads.ontology_query(2048, 7)
    gp, rp = _write(wl, tmp_path)
    exp_lines, _, _ = _oracle_run(oracle, gp, rp)
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        for loop in ("device", "graph", "host"):
            q.load()
            st = ctx.closure(wl.grammar.rules, q.mats, use_graph=loop, max_iterations=2)
            assert st["iterations"] == 2
            assert q.run(use_graph=loop).lines == exp_lines
    finally:
        q.close()


def test_closure_epsilon_and_self_loops(ctx, pkg, oracle, tmp_path):
    gram = "S\nS S S\nS A S\nA a\nB S B\nB b\n"
    g = pkg.workloads.uniform_graph(150, 200, ["a", "b"], 9)
    wl = pkg.workloads.Workload("eps", gram, g, {})
    _check_query(ctx, pkg, oracle, wl, tmp_path)


def test_closure_repeated_runs_are_identical(ctx, pkg, oracle, tmp_path):
    wl = pkg.workloads.ontology_query(1024, 5)
    gp, rp = _write(wl, tmp_path)
    exp_lines, _, _ = _oracle_run(oracle, gp, rp)
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        for _ in range(3):
            assert q.run().lines == exp_lines
    finally:
        q.close()


def test_plan_reuse_across_interleaved_work(ctx, pkg, oracle, tmp_path):
    """Closures of two prepared queries, interleaved with a product that
    reuses the context's tables, stay exact (the cached plan of the last
    closure is only reused for the same rules and matrices)."""
    wl1 = pkg.workloads.ontology_query(1024, 5)
    labels = ["x", "y", "z"]
    wl2 = pkg.workloads.Workload("random_cnf", pkg.workloads.random_cnf(8, 20, labels, 4),
                                 pkg.workloads.uniform_graph(700, 1400, labels, 4), {})
    exps = []
    for i, wl in enumerate((wl1, wl2)):
        d = tmp_path / f"q{i}"
        d.mkdir()
        exps.append(_oracle_run(oracle, *_write(wl, d))[0])
    q1 = pkg.query.PreparedQuery(ctx, wl1.grammar, wl1.graph)
    q2 = pkg.query.PreparedQuery(ctx, wl2.grammar, wl2.graph)
    a, b, c = ctx.matrix(300), ctx.matrix(300), ctx.matrix(300)
    try:
        for loop in ("device", "graph", "device"):
            assert q1.run(use_graph=loop).lines == exps[0]
            assert q1.run(use_graph=loop).lines == exps[0]
            assert q2.run(use_graph=loop).lines == exps[1]
            a.set_diagonal()
            b.set_diagonal()
            ctx.add_mul(c, a, b, "lop3")
            assert q2.run(use_graph=loop).lines == exps[1]
            assert q1.run(use_graph=loop).lines == exps[0]
    finally:
        q1.close()
        q2.close()
        for m in (a, b, c):
            m.destroy()


def test_clear_many(ctx, pkg):
    rng = np.random.default_rng(3)
    mats = [ctx.matrix(n) for n in (1, 64, 200, 1000)]
    order = ctx.order(rng.permutation(333).astype(np.uint32))
    mats.append(ctx.matrix(333, order))
    try:
        for m in mats:
            n = m.n
            k = max(1, n * 3)
            m.set_bits(rng.integers(0, n, k).astype(np.uint32), rng.integers(0, n, k).astype(np.uint32))
            assert m.hash_count()[1] > 0
        ctx.clear_many(mats)
        for m in mats:
            assert m.hash_count() == (0, 0)
            assert not m.download_rows().any()
            occ, nnz = m.tile_stats()
            assert not occ.any() and not nnz.any()
    finally:
        for m in mats:
            m.destroy()
        order.destroy()


def test_batch_matches_single_queries(ctx, pkg, oracle, tmp_path):
    wls = [w for w in pkg.workloads.batch_queries(24, seed=5, n_min=64, n_max=900)]
    qs, exps = [], []
    for i, wl in enumerate(wls):
        d = tmp_path / f"q{i}"
        d.mkdir()
        gp, rp = _write(wl, d)
        exps.append(_oracle_run(oracle, gp, rp)[0])
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
        q.load()
        qs.append(q)
    try:
        for loop in ("device", "graph"):
            for q in qs:
                q.load()
            stats, iters, done = ctx.closure_batch([(q.grammar.rules, q.mats) for q in qs], use_graph=loop)
            for q, exp in zip(qs, exps):
                got = dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats)))
                assert got == exp
            assert stats["iterations"] >= int(iters.max())
            assert (done >= 0).all()
    finally:
        for q in qs:
            q.close()


def test_batch_active_queries(ctx, pkg, oracle, tmp_path):
    """Batches plan only the queries still changing (persistent loop): empty
    queries in the mix, and an iteration limit followed by a full closure.
    Iteration counts are not compared with each query closed alone: products
    of one iteration may already see bits other products set in it, so the
    count depends on scheduling; the fixpoint does not."""
    wls = pkg.workloads.batch_queries(12, seed=11, n_min=64, n_max=700)
    qs, exps = [], []
    for i, wl in enumerate(wls):
        d = tmp_path / f"q{i}"
        d.mkdir()
        gp, rp = _write(wl, d)
        exps.append(_oracle_run(oracle, gp, rp)[0])
        qs.append(pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph))
    spare = ctx.matrix(128)
    try:
        batch = [(q.grammar.rules, q.mats) for q in qs]
        batch.insert(3, ([], []))          # no matrices
        batch.insert(7, ([], [spare]))     # a matrix, no rules
        for limit in (2, 0):
            for q in qs:
                q.load()
            st, it, done = ctx.closure_batch(batch, use_graph="device", max_iterations=limit)
            assert int(it[3]) == 0 and int(it[7]) == 0
            if limit:
                assert int(it.max()) <= limit
                continue
            assert 1 <= int(it.min(initial=99, where=it > 0)) and int(it.max()) < st["iterations"]
            for q, exp in zip(qs, exps):
                assert dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats))) == exp
        for q in qs:  # after the limited run the next closure restarts from scratch
            q.load()
        ctx.closure_batch(batch, use_graph="device", max_iterations=3)
        ctx.closure_batch(batch, use_graph="device")
        for q, exp in zip(qs, exps):
            assert dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats))) == exp
    finally:
        spare.destroy()
        for q in qs:
            q.close()


def test_interleaved_loads_and_clears(ctx, pkg):
    """Edge loads and clears of alternating matrix sets (host and device edge
    arrays, the library keeping the small tables of the last load on the
    device) leave every matrix exactly as a first load does."""
    import torch

    wls = [pkg.workloads.ontology_query(700, 3), pkg.workloads.brackets_query(), pkg.workloads.ontology_query(700, 4)]
    qs = [pkg.query.PreparedQuery(ctx, w.grammar, w.graph) for w in wls]
    try:
        first = []
        for q in qs:
            q.load()
            first.append(ctx.hash_count_many(q.mats))
        for order in ([0, 1, 2], [2, 2, 0], [1, 0, 1]):
            for i in order:
                qs[i].load()
                assert ctx.hash_count_many(qs[i].mats) == first[i]
            for i in order:  # device-resident edge arrays
                g = qs[i].graph
                dev = [torch.from_numpy(a.view(np.int32)).cuda() for a in (g.src, g.label, g.dst)]
                ctx.clear_many(qs[i].mats)
                ctx.load_edges_device(qs[i].mats, dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(),
                                      g.nedges, qs[i].off, qs[i].lm)
                for e in qs[i].grammar.epsilon:
                    qs[i].mats[e].set_diagonal()
                assert ctx.hash_count_many(qs[i].mats) == first[i]
        ctx.clear_many(qs[0].mats)
        assert all(c == 0 for _, c in ctx.hash_count_many(qs[0].mats))
        assert ctx.hash_count_many(qs[1].mats) == first[1]
    finally:
        for q in qs:
            q.close()


def test_item_trace(ctx, pkg, oracle, tmp_path):
    """LOG_ITEMS records every work item of a persistent closure once, and
    tracing does not change the result."""
    wl = pkg.workloads.ontology_query(1024, 2)
    gp, rp = _write(wl, tmp_path)
    exp = _oracle_run(oracle, gp, rp)[0]
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        q.load()
        st = ctx.closure(wl.grammar.rules, q.mats, use_graph="device", log_products=pkg.capi.LOG_ITEMS)
        assert dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats))) == exp
        log = ctx.item_log()
        plans, tr = log[log["list"] == 2], log[log["list"] < 2]
        assert len(tr) == st["work_items"] > 0
        assert len(plans) == st["iterations"] * len(np.unique(plans["cta"]))  # every CTA plans every iteration
        assert (tr["end_ns"] >= tr["start_ns"]).all()
        assert (tr["iteration"] < st["iterations"]).all()
        assert (tr["product"] < 2 * len(wl.grammar.rules)).all()
        assert (tr["klo"] < tr["khi"]).all() and (tr["khi"] <= (1024 + 63) // 64).all()
        assert set(np.unique(tr["list"])) <= {0, 1}
        assert (plans["end_ns"] >= plans["start_ns"]).all()
        q.load()
        ctx.closure(wl.grammar.rules, q.mats, use_graph="device")
        assert len(ctx.item_log()) == 0
    finally:
        q.close()


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_CASES = sorted(d for d in os.listdir(GOLDEN) if os.path.isdir(os.path.join(GOLDEN, d)))


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_engine_matches_golden(ctx, pkg, oracle, case):
    """The engine (through the C ABI) and the b200GPU drop-in executable
    reproduce every committed golden answer."""
    d = os.path.join(GOLDEN, case)
    gp, rp = os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")
    expected = oracle.parse_answer(open(os.path.join(d, "expected.txt")).read())
    grammar, graph = pkg.query.CnfGrammar.from_file(gp), pkg.query.EdgeGraph.from_file(rp)
    res = pkg.query.run_query(ctx, grammar, graph)
    assert res.lines == expected
    exe = os.path.join(os.path.dirname(pkg.capi.LIB_PATH), "..", "bin", "b200GPU")
    got, _ = oracle.run_executable(exe, gp, rp)
    assert got == expected


def test_b200gpu_executable(pkg, oracle, tmp_path):
    """The drop-in executable on a random graph and an ontology graph: the
    engine with the vertex order its backend suggests at upload (default),
    without it (CFPQ_ORDER=0), and the reference's worklist with the plain
    product on ordered matrices; every answer equals the oracle's."""
    exe = os.path.join(os.path.dirname(pkg.capi.LIB_PATH), "..", "bin", "b200GPU")
    for wl in (pkg.workloads.brackets_query(n=512, nedges=2048, seed=3), pkg.workloads.ontology_query(2048, 2)):
        d = tmp_path / wl.name
        d.mkdir()
        gp, rp = _write(wl, d)
        exp, _, _ = _oracle_run(oracle, gp, rp)
        for env in ({}, {"CFPQ_ORDER": "0"}, {"CFPQ_DRIVER": "worklist", "CFPQ_VARIANT": "plain"}):
            got, (total, algo) = oracle.run_executable(exe, gp, rp, env={**os.environ, **env})
            assert got == exp, (wl.name, env)
            assert total >= algo >= 0


@pytest.mark.parametrize("exe", ["naiveGPU", "m4riGPU"])
def test_reference_gpu_backends_agree(pkg, oracle, tmp_path, exe):
    """The reference's own CUDA backends (built from its sources for sm_100a)
    give the same answers as the oracle on inputs whose rules never alias
    head and body (the reference naive backend's aliased path reads an
    uninitialised temporary, cuda/naive-gpu/Multiplication.cu:151-158)."""
    path = oracle.ref_executable(exe)
    if path is None:
        pytest.skip(f"oracle/_ref/{exe} not built")
    for wl in (pkg.workloads.brackets_query(), pkg.workloads.ontology_query(2048, 2)):
        d = tmp_path / wl.name
        d.mkdir()
        gp, rp = _write(wl, d)
        exp, _, _ = _oracle_run(oracle, gp, rp)
        got, _ = oracle.run_executable(path, gp, rp)
        assert got == exp
