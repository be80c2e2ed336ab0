"""Seeded synthetic CFPQ workloads in the reference's text formats.

The reference's own datasets (data/graphs/{RDF,SG,WorstCase,FullGraph}, data/bio)
are Git-LFS pointers without content, so these generators stand in for them.
Every generator is deterministic in its seed (numpy MT19937).

  brackets_query      N=1024, labels {a,b}, 4096 uniform edges, balanced-bracket
                      CNF  S -> A B | A S1, S1 -> S B, A -> a, B -> b
  ontology_query      N=8192 ontology-like graph: subClassOf edges form a random
                      DAG of depth <= 12 over classes, type edges from instances to
                      classes by preferential attachment (scale-free), mean
                      out-degree 3, plus the inverse of every edge (4 labels);
                      same-generation grammar
                        S -> sc^-1 S sc | t^-1 S t | sc^-1 sc | t^-1 t
                      in CNF with 7 nonterminals (S, two helpers, four label
                      nonterminals)
  batch_queries       512 queries, N log-uniform in [256, 8192], 2-8 edges per
                      vertex, 2-6 labels, grammar family drawn per query from
                      {brackets, same-generation, random CNF with 8 nonterminals
                      and 20 binary rules}
  chain_query         N=65536, mean out-degree 2, 90 % of edges with |u-v| <= 64
                      and 10 % uniform, 6 labels, random CNF with 10 nonterminals
                      and 24 binary rules plus one terminal rule per label
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .query import CnfGrammar, EdgeGraph

BRACKETS_GRAMMAR = "S A B\nS A S1\nS1 S B\nA a\nB b\n"

SAME_GENERATION_GRAMMAR = (
    "S SCR S1\n"
    "S1 S SC\n"
    "S TR S2\n"
    "S2 S T\n"
    "S SCR SC\n"
    "S TR T\n"
    "SCR subClassOf_r\n"
    "SC subClassOf\n"
    "TR type_r\n"
    "T type\n"
)


@dataclasses.dataclass
class Workload:
    name: str
    grammar_text: str
    graph: EdgeGraph
    params: dict

    @property
    def grammar(self) -> CnfGrammar:
        return CnfGrammar.from_text(self.grammar_text)

    def write(self, grammar_path: str, graph_path: str) -> None:
        with open(grammar_path, "w") as f:
            f.write(self.grammar_text)
        self.graph.write(graph_path)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.MT19937(seed))


def _graph(src, lab, dst, labels, n) -> EdgeGraph:
    return EdgeGraph(np.asarray(src, dtype=np.uint32), np.asarray(lab, dtype=np.uint32),
                     np.asarray(dst, dtype=np.uint32), list(labels), int(n))


def _pin_last_vertex(src: np.ndarray, dst: np.ndarray, n: int, rng: np.random.Generator) -> None:
    """Make sure vertex n-1 has an edge so that the loaders derive exactly n."""
    if src.size and max(int(src.max()), int(dst.max())) < n - 1:
        dst[rng.integers(0, src.size)] = n - 1


def uniform_graph(n: int, nedges: int, labels: list[str], seed: int) -> EdgeGraph:
    rng = _rng(seed)
    src = rng.integers(0, n, nedges, dtype=np.int64)
    dst = rng.integers(0, n, nedges, dtype=np.int64)
    lab = rng.integers(0, len(labels), nedges, dtype=np.int64)
    _pin_last_vertex(src, dst, n, rng)
    return _graph(src, lab, dst, labels, n)


def brackets_query(n: int = 1024, nedges: int = 4096, seed: int = 1) -> Workload:
    g = uniform_graph(n, nedges, ["a", "b"], seed)
    return Workload("brackets", BRACKETS_GRAMMAR, g, {"n": n, "edges": nedges, "seed": seed})


def ontology_graph(n: int, seed: int, mean_degree: float = 3.0, class_fraction: float = 0.25,
                   depth: int = 12) -> EdgeGraph:
    """subClassOf DAG of depth <= `depth` levels + preferential type edges, with inverses."""
    rng = _rng(seed)
    nc = max(depth, int(n * class_fraction))
    ni = n - nc
    # class levels: level sizes grow geometrically with depth
    w = 1.6 ** np.arange(depth)
    sizes = np.maximum(1, np.floor(w / w.sum() * nc)).astype(np.int64)
    sizes[-1] += nc - sizes.sum()
    level = np.repeat(np.arange(depth), sizes)
    starts = np.concatenate([[0], np.cumsum(sizes)])
    sc_src, sc_dst = [], []
    child_count = np.zeros(nc, dtype=np.float64)
    for c in range(nc):
        L = level[c]
        if L == 0:
            continue
        lo, hi = starts[L - 1], starts[L]
        k = 1 if rng.random() < 0.8 else 2
        k = min(k, hi - lo)
        p = child_count[lo:hi] + 1.0
        parents = rng.choice(np.arange(lo, hi), size=k, replace=False, p=p / p.sum())
        for par in parents:
            sc_src.append(c)
            sc_dst.append(par)
            child_count[par] += 1
    # instances: scale-free out-degree (Zipf), targets by preferential
    # attachment.  An instance is typed with a home class and classes of the
    # home's neighbourhood in the hierarchy (its siblings, then ancestor levels
    # with their siblings), as materialised RDF types are.
    parent_of = [[] for _ in range(nc)]
    children = [[] for _ in range(nc)]
    for c, par in zip(sc_src, sc_dst):
        parent_of[c].append(par)
        children[par].append(c)
    n_type = max(ni, int(round(mean_degree * n)) - len(sc_src))
    deg = rng.zipf(2.2, size=ni).astype(np.float64)
    # 1.35: compensates for degrees truncated at the size of the neighbourhood
    deg = np.maximum(1, np.round(deg * (1.35 * n_type / deg.sum()))).astype(np.int64)
    t_src, t_dst = [], []
    indeg = np.ones(nc, dtype=np.float64)
    for i in range(ni):
        p = indeg / indeg.sum()
        home = int(rng.choice(nc, p=p))
        targets = {home}
        want = int(deg[i])
        # neighbourhood: siblings, then each ancestor level with its siblings
        pool = []
        level_nodes = [home]
        while level_nodes and len(pool) < 2 * want:
            parents = list(dict.fromkeys(p_ for x in level_nodes for p_ in parent_of[x]))
            sib = [y for p_ in parents for y in children[p_]]
            pool.extend(sib)
            pool.extend(parents)
            level_nodes = parents
        pool = [x for x in dict.fromkeys(pool) if x != home]
        if pool and want > 1:
            w_ = indeg[pool]
            k = min(want - 1, len(pool))
            extra = rng.choice(np.asarray(pool), size=k, replace=False, p=w_ / w_.sum())
            targets.update(int(x) for x in extra)
        tg = np.fromiter(targets, dtype=np.int64)
        indeg[tg] += 1
        t_src.extend([nc + i] * tg.size)
        t_dst.extend(tg.tolist())
    perm = rng.permutation(n)
    sc_src = perm[np.asarray(sc_src, dtype=np.int64)]
    sc_dst = perm[np.asarray(sc_dst, dtype=np.int64)]
    t_src = perm[np.asarray(t_src, dtype=np.int64)]
    t_dst = perm[np.asarray(t_dst, dtype=np.int64)]
    labels = ["subClassOf", "type", "subClassOf_r", "type_r"]
    src = np.concatenate([sc_src, t_src, sc_dst, t_dst])
    dst = np.concatenate([sc_dst, t_dst, sc_src, t_src])
    lab = np.concatenate([np.zeros(sc_src.size), np.ones(t_src.size), np.full(sc_src.size, 2),
                          np.full(t_src.size, 3)]).astype(np.int64)
    _pin_last_vertex(src, dst, n, rng)
    return _graph(src, lab, dst, labels, n)


def ontology_query(n: int = 8192, seed: int = 1) -> Workload:
    g = ontology_graph(n, seed)
    return Workload("same_generation", SAME_GENERATION_GRAMMAR, g, {"n": n, "seed": seed})


def random_cnf(n_nonterminals: int, n_rules: int, labels: list[str], seed: int) -> str:
    """Random CNF: one terminal rule per label (spread over the nonterminals),
    `n_rules` distinct binary rules; every nonterminal heads at least one rule
    or derives a label so that none is trivially empty."""
    rng = _rng(seed)
    names = ["S"] + [f"N{i}" for i in range(1, n_nonterminals)]
    lines = []
    lab_nt = rng.permutation(n_nonterminals)[:len(labels)] if len(labels) <= n_nonterminals else \
        rng.integers(0, n_nonterminals, len(labels))
    for l, nt in zip(labels, lab_nt):
        lines.append(f"{names[nt]} {l}")
    seen = set()
    heads = list(rng.permutation(n_nonterminals))
    while len(seen) < n_rules:
        h = int(heads.pop()) if heads else int(rng.integers(0, n_nonterminals))
        b1, b2 = (int(x) for x in rng.integers(0, n_nonterminals, 2))
        if (h, b1, b2) in seen:
            continue
        seen.add((h, b1, b2))
        lines.append(f"{names[h]} {names[b1]} {names[b2]}")
    return "\n".join(lines) + "\n"


def chain_graph(n: int, mean_degree: float, local_fraction: float, window: int, labels: list[str],
                seed: int) -> EdgeGraph:
    rng = _rng(seed)
    m = int(round(mean_degree * n))
    src = rng.integers(0, n, m, dtype=np.int64)
    local = rng.random(m) < local_fraction
    off = rng.integers(1, window + 1, m) * np.where(rng.random(m) < 0.5, -1, 1)
    dst = np.where(local, np.clip(src + off, 0, n - 1), rng.integers(0, n, m))
    lab = rng.integers(0, len(labels), m, dtype=np.int64)
    _pin_last_vertex(src, dst, n, rng)
    return _graph(src, lab, dst, labels, n)


def chain_query(n: int = 65536, seed: int = 1, n_nonterminals: int = 10, n_rules: int = 24) -> Workload:
    labels = [f"l{i}" for i in range(6)]
    g = chain_graph(n, 2.0, 0.9, 64, labels, seed)
    gram = random_cnf(n_nonterminals, n_rules, labels, seed + 1000003)
    return Workload("chain_random_cnf", gram, g, {"n": n, "seed": seed, "nonterminals": n_nonterminals,
                                                   "rules": n_rules})


def batch_queries(count: int = 512, seed: int = 1, n_min: int = 256, n_max: int = 8192) -> list[Workload]:
    rng = _rng(seed)
    out = []
    for q in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        density = float(rng.uniform(2.0, 8.0))
        nlab = int(rng.integers(2, 7))
        family = int(rng.integers(0, 3))
        qseed = int(rng.integers(1, 2**31 - 1))
        if family == 0:
            labels = ["a", "b"] + [f"x{i}" for i in range(nlab - 2)]
            g = uniform_graph(n, int(density * n), labels, qseed)
            out.append(Workload("brackets", BRACKETS_GRAMMAR, g,
                                {"n": n, "density": density, "labels": nlab, "seed": qseed}))
        elif family == 1:
            g = ontology_graph(n, qseed, mean_degree=density / 2.0)
            out.append(Workload("same_generation", SAME_GENERATION_GRAMMAR, g,
                                {"n": n, "density": density, "labels": 4, "seed": qseed}))
        else:
            labels = [f"l{i}" for i in range(nlab)]
            g = uniform_graph(n, int(density * n), labels, qseed)
            gram = random_cnf(8, 20, labels, qseed + 7)
            out.append(Workload("random_cnf", gram, g, {"n": n, "density": density, "labels": nlab,
                                                        "seed": qseed}))
    return out
