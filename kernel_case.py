#!/usr/bin/env python
"""Single-kernel cases for profiling the product variants in isolation.

  python kernel_case.py dense --variant tc --n 8192 --density 0.3 --reps 3
  python kernel_case.py closure --n 8192 --reps 3
  python kernel_case.py batch --queries 64 --reps 2
  python kernel_case.py chain --n 16384 --reps 1
  python kernel_case.py lines --n 8192 --reps 20

`dense` runs C |= A * B on two seeded random n x n bit matrices (every tile
populated) `reps` times with one variant; `closure` runs the same-generation
ontology query (seeded, n vertices) `reps` times; `batch` closes a seeded
mixed batch of `queries` queries (N log-uniform in [256, 8192]) with one
cfpq_closure_batch per repetition; `chain` closes the chain workload (mean
out-degree 2, 90% local edges, random CNF with 10 nonterminals and 24 rules)
at n vertices with the selector (variant AUTO, every size selects); `lines`
closes the same-generation query once and then computes the result lines of
its matrices (cfpq_hash_count_many: one hash launch, one synchronisation)
`reps` times (`--empty`: of the same matrices cleared after the closure,
so every block finds no tile).  Each prints one JSON line
with the device time of every repetition (CUDA events on the library's
stream), so the same command can run with and without a profiler.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["dense", "closure", "batch", "chain", "lines"])
    ap.add_argument("--queries", type=int, default=64)
    ap.add_argument("--variant", default="lop3", choices=["plain", "lop3", "m4r", "tc"])
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--density", type=float, default=0.3)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--empty", action="store_true", help="lines: hash the query's matrices after clearing them")
    ap.add_argument("--no-graph", action="store_true",
                    help="closure, chain, batch: host-launched iterations, no CUDA graph or persistent kernel "
                         "(every kernel a separate launch, as a profiler needs)")
    args = ap.parse_args()

    import numpy as np
    import torch

    pkg = importlib.import_module("cfpq-on-gpgpu_b200")
    ctx = pkg.capi.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    times = []
    out = {"case": args.case, "n": args.n, "reps": args.reps}
    if args.case == "dense":
        rng = np.random.default_rng(args.seed)
        n, wpr = args.n, (args.n + 63) // 64
        mats = []
        for _ in range(2):
            bits = rng.random((n, wpr * 64)) < args.density
            bits[:, n:] = False
            m = ctx.matrix(n)
            m.upload_rows(np.packbits(bits, axis=1, bitorder="little").view(np.uint64).reshape(n, wpr))
            mats.append(m)
        c = ctx.matrix(n)
        for _ in range(args.reps):
            c.clear()
            ctx.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.add_mul(c, mats[0], mats[1], args.variant)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        out.update(variant=args.variant, density=args.density, hash_count=list(c.hash_count()),
                   tbitmac_per_s=[n ** 3 / (t / 1e3) / 1e12 for t in times])
        for m in mats + [c]:
            m.destroy()
    elif args.case == "batch":
        wls = pkg.workloads.batch_queries(args.queries, seed=args.seed)
        qs = [pkg.query.PreparedQuery(ctx, w.grammar, w.graph) for w in wls]
        for _ in range(args.reps):
            for q in qs:
                q.load()
            ctx.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, iters, _ = ctx.closure_batch([(q.grammar.rules, q.mats) for q in qs],
                                             use_graph="host" if args.no_graph else True)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        out.update(queries=args.queries, iterations=int(iters.max()), items=st["work_items"],
                   dense_bitops=st["dense_bitops"], tile_triples=st["tile_triples"], variant_items=st["variant_items"])
        for q in qs:
            q.close()
    elif args.case == "chain":
        wl = pkg.workloads.chain_query(args.n, args.seed)
        ctx.selector_configure(min_tiles=1)
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
        for _ in range(args.reps):
            q.load()
            ctx.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = ctx.closure(wl.grammar.rules, q.mats, variant="auto", use_graph=not args.no_graph)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        out.update(iterations=st["iterations"], tile_triples=st["tile_triples"], variant_items=st["variant_items"],
                   lines={k: list(v) for k, v in zip(wl.grammar.nonterminals, ctx.hash_count_many(q.mats))})
        q.close()
    elif args.case == "lines":
        wl = pkg.workloads.ontology_query(args.n, args.seed)
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
        q.run()
        if args.empty:
            ctx.clear_many(q.mats)
        for _ in range(args.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lines = ctx.hash_count_many(q.mats)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        out.update(lines={k: list(v) for k, v in zip(wl.grammar.nonterminals, lines)})
        q.close()
    else:
        wl = pkg.workloads.ontology_query(args.n, args.seed)
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
        for _ in range(args.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = q.run(variant="auto" if args.variant == "lop3" else args.variant, use_graph=not args.no_graph)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        out.update(variant=args.variant, lines={k: list(v) for k, v in res.lines.items()})
        q.close()
    out["ms"] = times
    print(json.dumps(out))
    ctx.close()


if __name__ == "__main__":
    main()
