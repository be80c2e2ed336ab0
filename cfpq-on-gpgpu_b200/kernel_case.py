#!/usr/bin/env python
"""Single-kernel cases for profiling the product variants in isolation.

  python cfpq-on-gpgpu_b200/kernel_case.py dense --variant tc --n 8192 --density 0.3 --reps 3
  python cfpq-on-gpgpu_b200/kernel_case.py closure --n 8192 --reps 3

`dense` runs C |= A * B on two seeded random n x n bit matrices (every tile
populated) `reps` times with one variant; `closure` runs the same-generation
ontology query (seeded, n vertices) `reps` times.  Each prints one JSON line
with the device time of every repetition (CUDA events on the library's
stream), so the same command can run with and without a profiler.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["dense", "closure"])
    ap.add_argument("--variant", default="lop3", choices=["plain", "lop3", "m4r", "tc"])
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--density", type=float, default=0.3)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-graph", action="store_true", help="closure: host-launched iterations, no CUDA graph")
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
