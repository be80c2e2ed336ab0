"""Query sharding for batched closures on several GPUs (one process per GPU).

Independent queries need no collective on the data path: each rank closes its
own share with one cfpq_closure_batch, and only the per-query result lines and
timings are gathered on the host afterwards.  Shares are balanced by
longest-processing-time-first over an estimate of the dense-equivalent work of
a query (n^3 bit-MACs per rule term).
"""
from __future__ import annotations

import heapq
from typing import Sequence


def query_cost(n: int, n_rules: int) -> float:
    """Dense-equivalent work estimate of one closure iteration: 2 terms x rules x n^3."""
    return 2.0 * max(int(n_rules), 1) * float(n) ** 3


def lpt_assign(costs: Sequence[float], nranks: int) -> list[list[int]]:
    """Longest-processing-time-first: queries in decreasing cost, each to the
    least loaded rank (ties: lowest rank, then lowest index first).  Returns
    the query indices of every rank, in increasing order."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(nranks)]
    shares: list[list[int]] = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shares]


def gather_lines(dist, local: dict[int, dict]) -> dict[int, dict]:
    """All ranks' {query index: result lines} merged (torch.distributed, any backend)."""
    if dist is None:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, local)
    merged: dict[int, dict] = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"query {k} closed on two ranks")
            merged[k] = v
    return merged
