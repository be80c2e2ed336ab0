"""Generates the golden fixtures under tests/golden/.

Each fixture is a directory with grammar.txt, graph.txt and expected.txt (the
reference's answer format: "name hash count" per nonterminal in name order,
cfpq-cpp/Grammar.cpp:81-100) plus source.txt saying where the answer came from.

  known_*      closed-form answers: the expected matrices are built here from
               the mathematics of each case (not by any closure code) and the
               answer lines by a direct transcription of the reference's
               printing loop.
  m4ricpu_*    answers printed by the reference's own CPU executable
               (m4ri/main.cpp + cfpq-cpp driver compiled from the reference
               sources, oracle/_ref/m4riCPU; its libm4ri dependency is the
               restated subset in oracle/), on seeded inputs written here.
  naivegpu_*   answers printed by the reference's naive CUDA executable
               (cuda/naive-gpu compiled from the reference sources for sm_100a,
               oracle/_ref/naiveGPU) on a B200, same inputs (--ref-gpu; needs a
               GPU).

Usage:  python tests/golden/make_golden.py [--ref-cpu] [--ref-gpu] [--out DIR]
"""
from __future__ import annotations

import argparse
import importlib
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

MOD = 1000000007


def answer_lines(names: list[str], n: int, sets: dict[str, set]) -> str:
    """The reference printing loop (Grammar.cpp:83-99) transcribed literally."""
    out = []
    for name in sorted(names, key=lambda s: s.encode()):
        bits = sets.get(name, set())
        h, count = 0, 0
        for row in range(n):
            line = 0
            for col in range(n):
                line *= 11
                if (row, col) in bits:
                    count += 1
                    line += 1
                line %= MOD
            h = (h * 13 + line) % MOD
        out.append(f"{name} {h} {count}\n")
    return "".join(out)


def write_case(out_dir: str, name: str, grammar: str, edges: list[tuple[int, str, int]], expected: str,
               source: str) -> None:
    d = os.path.join(out_dir, name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "grammar.txt"), "w") as f:
        f.write(grammar)
    with open(os.path.join(d, "graph.txt"), "w") as f:
        f.writelines(f"{a} {l} {b}\n" for a, l, b in edges)
    with open(os.path.join(d, "expected.txt"), "w") as f:
        f.write(expected)
    with open(os.path.join(d, "source.txt"), "w") as f:
        f.write(source + "\n")


BRACKETS = "S A B\nS A S1\nS1 S B\nA a\nB b\n"


def known_cases(out_dir: str) -> None:
    # 1. a^k b^k on a path: 0 -a-> 1 ... -a-> k -b-> ... -b-> 2k
    k = 9
    edges = [(i, "a", i + 1) for i in range(k)] + [(i, "b", i + 1) for i in range(k, 2 * k)]
    n = 2 * k + 1
    sets = {
        "A": {(i, i + 1) for i in range(k)},
        "B": {(i, i + 1) for i in range(k, 2 * k)},
        "S": {(k - m, k + m) for m in range(1, k + 1)},
        "S1": {(k - m, k + m + 1) for m in range(1, k)},
    }
    write_case(out_dir, "known_brackets_path", BRACKETS, edges, answer_lines(["S", "A", "B", "S1"], n, sets),
               "closed form: S = {(k-m, k+m)}, S1 = {(k-m, k+m+1)} on the path a^k b^k, k=9")
    # 2. epsilon + self-referencing rule: S -> eps | S S; labels unused by the grammar
    n = 37
    edges = [(i, "z", (i * 7 + 3) % n) for i in range(n)]
    write_case(out_dir, "known_epsilon_identity", "S\nS S S\n", edges,
               answer_lines(["S"], n, {"S": {(i, i) for i in range(n)}}),
               "closed form: S = identity (epsilon diagonal; S S adds nothing)")
    # 3. complete graph, S -> S S | a: every pair
    n = 40
    edges = [(i, "a", j) for i in range(n) for j in range(n)]
    write_case(out_dir, "known_full_graph_a_plus", "S S S\nS a\n", edges,
               answer_lines(["S"], n, {"S": {(i, j) for i in range(n) for j in range(n)}}),
               "closed form: complete graph with label a, S = a+ relates all n^2 pairs")
    # 4. a-cycle of length p and b-cycle of length q sharing vertex 0 (gcd(p,q)=1):
    #    S(u, v) iff some m >= 1 has u + m = 0 (mod p) on the a-cycle and v is
    #    the vertex m steps along the b-cycle -- by the Chinese remainder
    #    theorem every (a-cycle vertex, b-cycle vertex) pair qualifies.
    p, q = 3, 4
    bcyc = [0] + list(range(p, p + q - 1))
    edges = [(i, "a", (i + 1) % p) for i in range(p)] + [(bcyc[j], "b", bcyc[(j + 1) % q]) for j in range(q)]
    n = p + q - 1
    s_set = {(u, v) for u in range(p) for v in bcyc}
    s1_set = {(u, bcyc[(bcyc.index(v) + 1) % q]) for (u, v) in s_set}
    sets = {"S": s_set, "S1": s1_set, "A": {(i, (i + 1) % p) for i in range(p)},
            "B": {(bcyc[j], bcyc[(j + 1) % q]) for j in range(q)}}
    write_case(out_dir, "known_two_cycles", BRACKETS, edges, answer_lines(["S", "A", "B", "S1"], n, sets),
               "closed form: a-cycle p=3 and b-cycle q=4 sharing vertex 0; S = a-cycle x b-cycle (CRT), "
               "S1 = S followed by one b step")
    # 5. same generation on a complete binary tree (child subClassOf parent + inverses):
    #    only co-parents of a child are related, i.e. S = {(x, x) : x internal}
    depth = 4
    nt = 2 ** (depth + 1) - 1
    edges = []
    for c in range(1, nt):
        par = (c - 1) // 2
        edges += [(c, "subClassOf", par), (par, "subClassOf_r", c)]
    gram = "S SCR S1\nS1 S SC\nS SCR SC\nSCR subClassOf_r\nSC subClassOf\n"
    internal = {x for x in range(nt) if 2 * x + 1 < nt}
    sets = {"S": {(x, x) for x in internal},
            "S1": {(x, (x - 1) // 2) for x in internal if x > 0},
            "SC": {(c, (c - 1) // 2) for c in range(1, nt)},
            "SCR": {((c - 1) // 2, c) for c in range(1, nt)}}
    write_case(out_dir, "known_same_generation_tree", gram, edges,
               answer_lines(["S", "S1", "SC", "SCR"], nt, sets),
               "closed form: same-generation on a binary tree of depth 4; S = diagonal of internal nodes, "
               "S1 = (internal non-root node, its parent)")


def seeded_inputs():
    pkg = importlib.import_module("cfpq-on-gpgpu_b200")
    W = pkg.workloads
    cases = {
        "brackets_n256": W.brackets_query(n=256, nedges=1024, seed=11),
        "brackets_n1024": W.brackets_query(n=1024, nedges=4096, seed=1),
        "same_generation_n1024": W.ontology_query(1024, 5),
    }
    labels = ["x", "y", "z"]
    g = W.uniform_graph(512, 1100, labels, 21)
    cases["random_cnf_n512"] = W.Workload("random_cnf", W.random_cnf(8, 20, labels, 21), g, {})
    return cases


def run_reference(exe: str, out_dir: str, prefix: str, source: str, check_against: str | None = None) -> None:
    """Run a reference executable on the seeded inputs.  With check_against, an
    answer that differs from the `check_against`_<case> answer in out_dir is a
    reference defect: it goes to ../golden_defects instead of the fixtures."""
    for name, wl in seeded_inputs().items():
        with tempfile.TemporaryDirectory() as d:
            gp, rp, ap = (os.path.join(d, x) for x in ("g.txt", "r.txt", "a.txt"))
            wl.write(gp, rp)
            p = subprocess.run([exe, gp, rp, ap], capture_output=True, timeout=1800)
            if p.returncode != 0 or p.stderr:
                raise RuntimeError(f"{exe} failed: {p.stderr.decode()[:400]}")
            case = os.path.join(out_dir, f"{prefix}_{name}")
            if check_against:
                ref_answer = os.path.join(out_dir, f"{check_against}_{name}", "expected.txt")
                if os.path.exists(ref_answer) and open(ref_answer).read() != open(ap).read():
                    case = os.path.join(os.path.dirname(os.path.abspath(out_dir)), "golden_defects",
                                        f"{prefix}_{name}")
                    source += " -- DIFFERS from the least fixpoint (see golden_defects)"
            os.makedirs(case, exist_ok=True)
            shutil.copy(gp, os.path.join(case, "grammar.txt"))
            shutil.copy(rp, os.path.join(case, "graph.txt"))
            shutil.copy(ap, os.path.join(case, "expected.txt"))
            with open(os.path.join(case, "source.txt"), "w") as f:
                f.write(source + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--ref-cpu", action="store_true")
    ap.add_argument("--ref-gpu", action="store_true")
    args = ap.parse_args()
    known_cases(args.out)
    ref = os.path.join(ROOT, "oracle", "_ref")
    if args.ref_cpu:
        run_reference(os.path.join(ref, "m4riCPU"), args.out, "m4ricpu",
                      "reference m4riCPU (m4ri/main.cpp + cfpq-cpp, restated libm4ri subset)")
    if args.ref_gpu:
        run_reference(os.path.join(ref, "naiveGPU"), args.out, "naivegpu",
                      "reference naiveGPU (cuda/naive-gpu + cfpq-cpp) built for sm_100a, run on a B200",
                      check_against="m4ricpu")


if __name__ == "__main__":
    main()
