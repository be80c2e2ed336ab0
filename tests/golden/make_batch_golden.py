"""Generates tests/golden/batch512_seed1.txt: the answer lines of every query
of the 512-query mixed batch (seed 1).

The batch is `workloads.batch_queries(512, seed=1)`: N log-uniform in
[256, 8192], 2-8 edges per vertex, 2-6 labels, grammar family per query from
{balanced brackets, same-generation, random CNF with 8 nonterminals and 20
rules}.  Each query is written in the reference's text formats and closed
  - by the CPU oracle (oracle/cfpq_oracle.c, restated M4RM),
    which gives the fixture's lines for every query, and
  - by the reference's own CPU executable oracle/_ref/m4riCPU (m4ri/main.cpp +
    the cfpq-cpp driver compiled from the reference sources, linked with the
    restated libm4ri subset in oracle/) within a per-query time budget: where
    it finishes, its answer file (cfpq-cpp/Grammar.cpp:81-100) must equal the
    oracle's lines, and the query is marked source=reference+oracle.  Its
    worklist driver needs minutes for the largest random-CNF queries, which
    stay source=oracle.

Fixture format, one block per query:
    query <index> n=<n> edges=<nedges> family=<family> digest=<edge digest> source=<who answered>
    <name> <hash> <count>
    ...
The digest (edges_digest) pins the generated input, so a change in the
generator is reported as such instead of as a wrong answer.

Usage:  python tests/golden/make_batch_golden.py [--ref-budget SECONDS] [--jobs J]
(one query per host core at a time; about half an hour on 8 cores)
"""
from __future__ import annotations

import argparse
import hashlib
import importlib
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIXTURE = os.path.join(HERE, "batch512_seed1.txt")
NQ, SEED = 512, 1


def edges_digest(graph) -> str:
    """First 16 hex digits of the SHA-256 of (n, src, label, dst)."""
    import numpy as np

    h = hashlib.sha256()
    h.update(np.uint64(graph.n).tobytes())
    for a in (graph.src, graph.label, graph.dst):
        h.update(np.ascontiguousarray(a, dtype=np.uint32).tobytes())
    return h.hexdigest()[:16]


def batch_workloads():
    pkg = importlib.import_module("cfpq-on-gpgpu_b200")
    return pkg.workloads.batch_queries(NQ, seed=SEED)


def read_fixture(path: str = FIXTURE) -> dict[int, dict]:
    """{query index: {"n", "edges", "family", "digest", "lines": {name: (hash, count)}}}"""
    out: dict[int, dict] = {}
    cur = None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "query":
                kv = dict(p.split("=", 1) for p in parts[2:])
                cur = {"n": int(kv["n"]), "edges": int(kv["edges"]), "family": kv["family"],
                       "digest": kv["digest"], "source": kv.get("source", ""), "lines": {}}
                out[int(parts[1])] = cur
            else:
                cur["lines"][parts[0]] = (int(parts[1]), int(parts[2]))
    return out


def _reference_answer(exe: str, gp: str, rp: str, budget: float, threads: int):
    """Answer lines of the reference executable, or None when it needs more
    than `budget` seconds."""
    with tempfile.TemporaryDirectory() as d:
        ap = os.path.join(d, "a.txt")
        try:
            p = subprocess.run([exe, gp, rp, ap], capture_output=True, timeout=budget,
                               env={**os.environ, "OMP_NUM_THREADS": str(threads)})
        except subprocess.TimeoutExpired:
            return None
        if p.returncode != 0 or p.stderr:
            raise RuntimeError(f"{exe} failed: {p.stderr.decode()[:400]}")
        with open(ap) as f:
            return f.read()


def _close_query(args):
    """(index, fixture block, answered by the reference) of one query: worker
    of the process pool, one host thread per query."""
    i, budget = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the checker (CPU restatement) and the reference executables

    wl = batch_workloads_cached()[i]
    with tempfile.TemporaryDirectory() as d:
        gp, rp = os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")
        wl.write(gp, rp)
        with oracle.Problem(gp, rp) as p:
            p.closure(oracle.M4RM, 1)
            lines = p.results()
        exe = oracle.ref_executable("m4riCPU")
        ref = _reference_answer(exe, gp, rp, budget, 1) if exe else None
    if ref is not None and oracle.parse_answer(ref) != lines:
        raise RuntimeError(f"query {i}: the reference m4riCPU and the oracle disagree")
    text = "".join(f"{k} {h} {c}\n" for k, (h, c) in sorted(lines.items(), key=lambda kv: kv[0].encode()))
    g = wl.graph
    source = "reference+oracle" if ref is not None else "oracle"
    return i, (f"query {i} n={g.n} edges={g.nedges} family={wl.name} digest={edges_digest(g)} "
               f"source={source}\n{text}"), ref is not None


_WLS = None


def batch_workloads_cached():
    global _WLS
    if _WLS is None:
        _WLS = batch_workloads()
    return _WLS


def main():
    import multiprocessing as mp

    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-budget", type=float, default=60.0,
                    help="seconds per query for oracle/_ref/m4riCPU (one thread)")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=FIXTURE)
    args = ap.parse_args()
    n = len(batch_workloads_cached())
    # largest queries first, so that the pool ends evenly
    order = sorted(range(n), key=lambda i: -batch_workloads_cached()[i].graph.n)
    blocks, checked = {}, 0
    with mp.get_context("spawn").Pool(args.jobs) as pool:
        for k, (i, block, by_ref) in enumerate(pool.imap_unordered(_close_query, [(i, args.ref_budget)
                                                                                 for i in order])):
            blocks[i] = block
            checked += by_ref
            if k % 32 == 31:
                print(f"{k + 1}/{n} queries, {checked} also answered by the reference", flush=True)
    with open(args.out, "w") as f:
        f.writelines(blocks[i] for i in range(n))
    print(f"{n} queries written, {checked} also answered by the reference")


if __name__ == "__main__":
    main()
