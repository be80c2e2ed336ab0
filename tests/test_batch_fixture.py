"""The 512-query batch fixture (tests/golden/batch512_seed1.txt, printed by the
reference's m4riCPU): it matches the generator's inputs, and the CPU oracle
reproduces it on a sample of queries (no GPU)."""
import importlib.util
import os

import pytest

from conftest import GOLDEN

FIXTURE = os.path.join(GOLDEN, "batch512_seed1.txt")


def _maker():
    spec = importlib.util.spec_from_file_location("make_batch_golden", os.path.join(GOLDEN, "make_batch_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def batch(pkg):
    mk = _maker()
    return mk, mk.read_fixture(FIXTURE), mk.batch_workloads()


def test_fixture_covers_every_query(batch):
    mk, fx, wls = batch
    assert sorted(fx) == list(range(mk.NQ)) == list(range(len(wls)))
    for i, wl in enumerate(wls):
        g = wl.graph
        assert (fx[i]["n"], fx[i]["edges"], fx[i]["family"]) == (g.n, g.nedges, wl.name), i
        assert fx[i]["digest"] == mk.edges_digest(g), i
        assert sorted(fx[i]["lines"]) == sorted(wl.grammar.nonterminals, key=lambda s: s.encode()), i


def test_oracle_reproduces_fixture_sample(batch, oracle, tmp_path):
    """Both oracle products (naive row gather and restated M4RM) give the
    fixture's lines on the smallest queries of each grammar family."""
    _, fx, wls = batch
    picked = []
    for fam in ("brackets", "same_generation", "random_cnf"):
        idx = sorted((i for i, w in enumerate(wls) if w.name == fam), key=lambda i: wls[i].graph.n)
        picked += idx[:3]
    for i in picked:
        d = tmp_path / f"q{i}"
        d.mkdir()
        gp, rp = str(d / "grammar.txt"), str(d / "graph.txt")
        wls[i].write(gp, rp)
        for method in (oracle.NAIVE, oracle.M4RM):
            with oracle.Problem(gp, rp) as p:
                p.closure(method, 0)
                assert p.results() == fx[i]["lines"], (i, method)
