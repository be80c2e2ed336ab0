"""Query plumbing above the C ABI: grammar / graph text formats and one call
that runs a CFPQ query on the device.

The text formats and their semantics are the reference's:
  grammar  cfpq-cpp/Grammar.cpp:17-51  one rule per line: "A" (epsilon),
           "A x" (terminal), "A B C" (A -> B C); nonterminals numbered in order
           of first appearance; a line with more than 3 tokens only registers
           its head; empty lines are skipped.
  graph    cfpq-cpp/Graph.cpp:11-20    "from label to" triples; n = max id + 1.
  results  cfpq-cpp/Grammar.cpp:81-100 "name hash count" per nonterminal in
           name order.
The closure itself runs in libcfpq_b200.so; nothing here computes a product.
"""
from __future__ import annotations

import dataclasses
import time
from typing import Sequence

import numpy as np

from . import capi


@dataclasses.dataclass
class CnfGrammar:
    nonterminals: list[str]
    rules: list[tuple[int, int, int]]
    terminal_to_nts: dict[str, list[int]]
    epsilon: list[int]

    @classmethod
    def from_text(cls, text: str) -> "CnfGrammar":
        idx: dict[str, int] = {}
        names: list[str] = []

        def index(name: str) -> int:
            if name not in idx:
                idx[name] = len(names)
                names.append(name)
            return idx[name]

        rules, t2n, eps = [], {}, []
        for line in text.split("\n"):
            tok = line.split()
            if not tok:
                continue
            head = index(tok[0])
            if len(tok) == 1:
                eps.append(head)
            elif len(tok) == 2:
                t2n.setdefault(tok[1], []).append(head)
            elif len(tok) == 3:
                b1 = index(tok[1])
                b2 = index(tok[2])
                rules.append((head, b1, b2))
        return cls(names, rules, t2n, eps)

    @classmethod
    def from_file(cls, path: str) -> "CnfGrammar":
        with open(path) as f:
            return cls.from_text(f.read())


@dataclasses.dataclass
class EdgeGraph:
    src: np.ndarray      # uint32
    label: np.ndarray    # uint32 index into labels
    dst: np.ndarray      # uint32
    labels: list[str]
    n: int

    @property
    def nedges(self) -> int:
        return int(self.src.size)

    @classmethod
    def from_file(cls, path: str, threads: int = 0) -> "EdgeGraph":
        """Parse with the library's parallel loader (cfpq_graph_load)."""
        src, lab, dst, labels, n = capi.load_graph_file(path, threads)
        return cls(src, lab, dst, labels, n)

    def write(self, path: str) -> None:
        lab = np.asarray(self.labels, dtype=object)[self.label] if self.nedges else []
        with open(path, "w") as f:
            for a, l, b in zip(self.src.tolist(), lab, self.dst.tolist()):
                f.write(f"{a} {l} {b}\n")


def write_grammar(path: str, text: str) -> None:
    with open(path, "w") as f:
        f.write(text)


@dataclasses.dataclass
class QueryResult:
    lines: dict[str, tuple[int, int]]   # name -> (hash, count)
    stats: dict
    load_ms: float
    closure_ms: float
    result_ms: float

    def answer_text(self) -> str:
        return "".join(f"{k} {h} {c}\n" for k, (h, c) in sorted(self.lines.items(), key=lambda kv: kv[0].encode()))


def label_map(grammar: CnfGrammar, graph: EdgeGraph) -> tuple[np.ndarray, np.ndarray]:
    """CSR map graph label id -> nonterminal matrices deriving it."""
    off, mats = [0], []
    for name in graph.labels:
        nts = grammar.terminal_to_nts.get(name, [])
        mats.extend(nts)
        off.append(len(mats))
    return np.asarray(off, dtype=np.uint32), np.asarray(mats, dtype=np.uint32)


class PreparedQuery:
    """Matrices of one query allocated on the device (reusable across runs).

    order: "auto" relabels vertices with the library's heuristic when it finds
    one (results are reported in original vertex ids either way), None keeps
    vertex v at index v, or an explicit permutation array."""

    def __init__(self, ctx: capi.Context, grammar: CnfGrammar, graph: EdgeGraph, order="auto"):
        self.ctx, self.grammar, self.graph = ctx, grammar, graph
        self.order = None
        if isinstance(order, str) and order == "auto":
            perm = capi.suggest_order(graph.n, graph.src, graph.label, graph.dst, ctx.lib)
            if not np.array_equal(perm, np.arange(graph.n, dtype=np.uint32)):
                self.order = ctx.order(perm)
        elif order is not None:
            self.order = ctx.order(np.asarray(order, dtype=np.uint32))
        self.mats = [ctx.matrix(graph.n, self.order) for _ in grammar.nonterminals]
        self.off, self.lm = label_map(grammar, graph)

    def load(self) -> None:
        """Clear and initialise from the edge list (one H2D copy, one scatter)."""
        self.ctx.clear_many(self.mats)
        if self.graph.nedges and self.mats:
            self.ctx.load_edges(self.mats, self.graph.src, self.graph.label, self.graph.dst, self.off, self.lm)
        for e in self.grammar.epsilon:
            self.mats[e].set_diagonal()

    def close(self) -> None:
        for m in self.mats:
            m.destroy()
        self.mats = []
        if self.order is not None:
            self.order.destroy()
            self.order = None

    def run(self, driver="engine", variant="auto", use_graph=True) -> QueryResult:
        t0 = time.perf_counter()
        self.load()
        self.ctx.synchronize()
        t1 = time.perf_counter()
        st = self.ctx.closure(self.grammar.rules, self.mats, driver=driver, variant=variant, use_graph=use_graph)
        t2 = time.perf_counter()
        hc = self.ctx.hash_count_many(self.mats)
        t3 = time.perf_counter()
        lines = {name: hc[i] for i, name in enumerate(self.grammar.nonterminals)}
        return QueryResult(lines, st, (t1 - t0) * 1e3, (t2 - t1) * 1e3, (t3 - t2) * 1e3)


def run_query(ctx: capi.Context, grammar: CnfGrammar, graph: EdgeGraph, **kw) -> QueryResult:
    q = PreparedQuery(ctx, grammar, graph)
    try:
        return q.run(**kw)
    finally:
        q.close()


def parse_answer(text: str) -> dict[str, tuple[int, int]]:
    out = {}
    for line in text.splitlines():
        if line.strip():
            name, h, c = line.split()
            out[name] = (int(h), int(c))
    return out
