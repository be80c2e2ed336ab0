#!/usr/bin/env python
"""CFPQ closure benchmark on B200.

Workload (one step = one whole CFPQ query on one GPU): the same-generation
query on a seeded ontology-like graph, N = 8192 vertices, 4 labels
(subClassOf, type and their inverses), mean out-degree ~3, subClassOf DAG of
depth <= 12, CNF grammar with 7 nonterminals and 6 binary rules.  Synthetic
data (the reference's RDF datasets are not available).

  value  closures/s with the edge list resident in HBM: every step clears the
         nonterminal matrices, scatters the edges on the device and runs the
         closure to its fixpoint (CUDA-graph loop); device time from CUDA
         events on the library's stream; L2 flushed (256 MiB write) between
         steps; max over ranks.
  e2e    the same through the C ABI from pinned host buffers: H2D of the edge
         list, closure, and the D2H of the result lines (hash, count per
         nonterminal) inside the timed region.

Multi-GPU (torchrun): one process per GPU, each closes its own seeded query
(query-partitioned replicas, weak scaling, no data-path collective).

--impl reference times the reference's CPU path on the host cores: the
reference's own m4riCPU driver (cfpq-cpp + m4ri backend sources) linked with
the restated libm4ri subset (oracle/_ref/m4riCPU), all host threads.
"""
from __future__ import annotations

import argparse
import datetime
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_VERTICES = 8192


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-profile", action="store_true")
    ap.add_argument("--no-selector-eval", action="store_true",
                    help="skip the learned-selector evaluation (trains the cost model on logged product timings "
                         "and reports its regret and batch closure time on fresh queries; about a minute)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the plain-GPU-form, reference-GPU, brackets and 512-query batch measurements")
    ap.add_argument("--no-chain", action="store_true",
                    help="skip the N=65536 chain closure (about three minutes)")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch every kernel from the host instead of the CUDA-graph loop (profilers cannot "
                         "capture kernel nodes of graphs with conditional nodes)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def committed_traffic() -> dict:
    """ncu DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per
    launch of the dominant kernels on the bench workload (profiles/traffic.json,
    copied from an ncu capture)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def reference_arm(args, world, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # reference / oracle executables only

    pkg = importlib.import_module("cfpq-on-gpgpu_b200")
    wl = pkg.workloads.ontology_query(N_VERTICES, args.seed)
    exe = oracle.ref_executable("m4riCPU")
    threads = os.cpu_count() or 1
    env = {**os.environ, "OMP_NUM_THREADS": str(threads)}
    with tempfile.TemporaryDirectory() as d:
        gp, rp = os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")
        wl.write(gp, rp)
        if exe is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/m4riCPU not built"}))
            return
        times = []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            _, (total, algo) = oracle.run_executable(exe, gp, rp, env=env)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(algo / 1e3 if algo > 0 else dt)
    total_s = sum(times)
    value = len(times) / total_s
    line = {
        "impl": "reference", "metric": "CFPQ closure throughput (same-generation query, N=8192)",
        "value": value, "unit": "closures/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64 (bit-packed Boolean)", "data": "synthetic",
        "config": {"workload": "same_generation_ontology_n8192", "n": N_VERTICES, "seed": args.seed,
                   "edges": wl.graph.nedges},
        "cpu_baseline": {"value": value, "unit": "closures/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(times)} full closures of the workload (algorithm time printed by "
                                   "the reference m4riCPU main, restated libm4ri M4RM, OpenMP)"},
        "e2e": {"value": value, "unit": "closures/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def cpu_baseline(wl, budget_s=12.0, budget_1thread_s=8.0) -> dict:
    """The reference's CPU path on this host's cores: all threads (the
    reported value) and one thread (a bounded sample beside it)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    exe = oracle.ref_executable("m4riCPU")
    nproc = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        gp, rp = os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")
        wl.write(gp, rp)

        def sample(threads, budget):
            times, answer = [], None
            t_start = time.perf_counter()
            while time.perf_counter() - t_start < budget or not times:
                if exe:
                    answer, (_, algo) = oracle.run_executable(exe, gp, rp,
                                                              env={**os.environ, "OMP_NUM_THREADS": str(threads)})
                    times.append(max(algo, 1) / 1e3)
                else:
                    with oracle.Problem(gp, rp) as p:
                        times.append(p.closure(oracle.M4RM, threads) / 1e3)
                        answer = p.results()
                if len(times) >= 50:
                    break
            return times, answer

        times, answer = sample(nproc, budget_s)
        times1, answer1 = sample(1, budget_1thread_s) if nproc > 1 else (times, answer)
    kind = "reference" if exe else "port"
    what = "reference m4riCPU main + restated libm4ri" if exe else "oracle M4RM port"
    return {"value": len(times) / sum(times), "unit": "closures/s", "cores": nproc, "kind": kind,
            "nproc": nproc,
            "sample": f"{len(times)} full closures of the same workload, algorithm time, {what}",
            "one_thread": {"value": len(times1) / sum(times1), "unit": "closures/s", "cores": 1,
                           "sample": f"{len(times1)} full closures, OMP_NUM_THREADS=1",
                           "same_answer": answer1 == answer},
            "answer": answer}


def _event_ms(torch, stream, fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r = fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1), r


def tile_model_bytes(ctx, q, grammar, iterations: int) -> dict:
    """Algorithmic bytes of a closure under the tile model: per product term
    of every iteration, (occupied P tiles + occupied Q tiles in the rows that
    P's occupied columns select + 2 x output tiles that some (P, Q) tile pair
    reaches) x 512 B (one 64x64-bit tile).  P / Q are the full matrix or the
    previous iteration's delta as the semi-naive term reads them.  The
    per-iteration tile occupancy comes from closures stopped after k = 0..K
    iterations (tile statistics downloaded after each; not timed)."""
    import numpy as np

    occ = []
    for k in range(iterations + 1):
        q.load()
        if k:
            ctx.closure(grammar.rules, q.mats, max_iterations=k)
        occ.append([m.tile_stats()[1].astype(np.int64) for m in q.mats])
    q.load()
    tiles = {"p": 0, "q": 0, "c": 0}
    terms = 0
    for t in range(iterations):
        cur = occ[t]
        delta = [cur[i] > occ[t - 1][i] for i in range(len(cur))] if t else None
        for head, b1, b2 in grammar.rules:
            pairs = [(cur[b1] > 0, cur[b2] > 0)] if t == 0 else [(delta[b1], cur[b2] > 0), (cur[b1] > 0, delta[b2])]
            for P, Q in pairs:
                if not P.any():
                    continue
                cols = P.any(axis=0)
                tiles["p"] += int(P.sum())
                tiles["q"] += int(Q[cols].sum())
                tiles["c"] += int(((P.astype(np.float32) @ Q.astype(np.float32)) > 0).sum())
                terms += 1
    return {"bytes": 512 * (tiles["p"] + tiles["q"] + 2 * tiles["c"]), "terms": terms,
            "occupied_p_tiles": tiles["p"], "occupied_q_tiles": tiles["q"], "touched_c_tiles": tiles["c"]}


def read_batch_fixture() -> dict:
    """Answer lines of the 512-query batch (seed 1) from tests/golden/batch512_seed1.txt
    (oracle M4RM for every query, the reference m4riCPU where it finished)."""
    out, cur = {}, None
    path = os.path.join(ROOT, "tests", "golden", "batch512_seed1.txt")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if parts and parts[0] == "query":
                cur = out.setdefault(int(parts[1]), {})
            elif parts:
                cur[parts[0]] = (int(parts[1]), int(parts[2]))
    return out


def plain_gpu_form(ctx, q, grammar, torch, stream, reps=2) -> dict:
    """The plain single-variant GPU form on the same workload: the reference's
    worklist driver (one product at a time, changed flag read back after each)
    with the plain dense product kernel (no tiles, no skipping, no batching)."""
    best, st = None, None
    for _ in range(reps):
        q.load()
        ctx.synchronize()
        ms, st = _event_ms(torch, stream, lambda: ctx.closure(grammar.rules, q.mats, driver="worklist",
                                                               variant="plain"))
        best = ms if best is None else min(best, ms)
    return {"ms": best, "closures_per_s": 1e3 / best, "products": st["products"],
            "form": "worklist driver + plain dense kernel (variant PLAIN)"}


def reference_gpu_forms(wl, lines_expected) -> dict:
    """The reference's own GPU executables (naiveGPU, m4riGPU built from its
    sources for sm_100a) and this repository's drop-in executable b200GPU
    (cfpq-cpp Grammar/Graph driver with the B200Matrix backend, the plugin
    boundary) on the same files: "total algo" milliseconds printed by each
    main (the harness contract), median of 3 runs for b200GPU."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    out = {}
    with tempfile.TemporaryDirectory() as d:
        gp, rp = os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")
        wl.write(gp, rp)
        ours = os.path.join(ROOT, "cfpq-on-gpgpu_b200", "bin", "b200GPU")
        if os.path.exists(ours):
            runs = []
            for _ in range(3):
                answer, (total, algo) = oracle.run_executable(ours, gp, rp, timeout=600)
                runs.append((total, algo, answer == lines_expected))
            runs.sort()
            total, algo, _ = runs[1]
            out["b200GPU"] = {"algo_ms": algo, "total_ms": total, "matches_ours": all(r[2] for r in runs),
                              "note": "this repository's drop-in executable: the reference's harness contract "
                                      "(process start, file parsing, device init and upload included in total)"}
        for name in ("naiveGPU", "m4riGPU"):
            exe = oracle.ref_executable(name)
            if exe is None:
                out[name] = {"unavailable": "not built"}
                continue
            try:
                answer, (total, algo) = oracle.run_executable(exe, gp, rp, timeout=600)
                out[name] = {"algo_ms": algo, "total_ms": total, "matches_ours": answer == lines_expected}
            except Exception as e:  # a reference failure is reported, not fatal
                out[name] = {"error": str(e)[:200]}
    return out


def batch_bench(pkg, ctx, torch, stream, rank, world, dist, nq=512, seed=1, steps=3) -> dict:
    """Batched queries (512 independent queries, N log-uniform in [256, 8192],
    three grammar families): every step closes the rank's LPT share of the
    batch with one cfpq_closure_batch (all products of all unfinished queries
    per iteration in one grouped launch).  Matrices are loaded before each
    step (not timed); queries/s = all queries / the slowest rank's time."""
    wls = pkg.workloads.batch_queries(nq, seed=seed)
    costs = [pkg.shard.query_cost(w.graph.n, len(w.grammar.rules)) for w in wls]
    mine = pkg.shard.lpt_assign(costs, world)[rank]
    qs = [pkg.query.PreparedQuery(ctx, wls[i].grammar, wls[i].graph) for i in mine]
    times, done, iters = [], None, None
    try:
        for step in range(steps + 1):
            for q in qs:
                q.load()
            ctx.synchronize()
            ms, (st, it, dn) = _event_ms(torch, stream, lambda: ctx.closure_batch(
                [(q.grammar.rules, q.mats) for q in qs]))
            if step > 0:  # step 0 warms up (plan cache, graph)
                times.append(ms)
                done, iters = dn, it
        t = max(times)
        if dist:
            tt = torch.tensor([t], dtype=torch.float64, device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        local_lines = {i: dict(zip(wls[i].grammar.nonterminals, ctx.hash_count_many(q.mats)))
                       for i, q in zip(mine, qs)}
        # the same queries closed one cfpq_closure at a time on the same
        # context (the unbatched baseline): sum of the closures' device times
        seq = 0.0
        seq_ok = True
        for i, q in zip(mine, qs):
            q.load()
            ctx.synchronize()
            seq += _event_ms(torch, stream, lambda: ctx.closure(q.grammar.rules, q.mats))[0]
            seq_ok &= dict(zip(q.grammar.nonterminals, ctx.hash_count_many(q.mats))) == local_lines[i]
        if dist:
            tt = torch.tensor([seq, float(seq_ok)], dtype=torch.float64, device="cuda")
            dist.all_reduce(tt[:1], op=dist.ReduceOp.MAX)
            dist.all_reduce(tt[1:], op=dist.ReduceOp.MIN)
            seq, seq_ok = float(tt[0].item()), bool(tt[1].item())
        lines = pkg.shard.gather_lines(dist, local_lines)
        import numpy as np

        expected = read_batch_fixture() if seed == 1 and nq == 512 else {}
        parity = (len(expected) == nq and all(lines.get(i) == expected[i] for i in range(nq))) if expected else None
        return {"queries": nq, "ms": t, "queries_per_s": nq / (t / 1e3),
                "p50_query_ms": float(np.percentile(done, 50)), "p99_query_ms": float(np.percentile(done, 99)),
                "max_iterations": int(iters.max()), "products": st["products"], "ranks": world,
                "sharding": "LPT on 2 * rules * n^3 per query, no data-path collective",
                "queries_closed": len(lines),
                "parity_vs_cpu": parity,
                "parity_reference": "tests/golden/batch512_seed1.txt: every query's answer lines from the CPU "
                                    "oracle (restated M4RM), also printed by the reference m4riCPU wherever it "
                                    "finished within its time budget",
                "sequential_ms": seq, "sequential_matches_batch": seq_ok,
                "batch_speedup_vs_sequential": seq / t if t > 0 else None,
                "sequential": "the same queries, one cfpq_closure each on the same context (default options), "
                              "sum of device times; loads not timed",
                "per_query_ms": "completion time of each query inside its rank's batch (device timer)"}
    finally:
        for q in qs:
            q.close()


def chain_cpu_check(wl, q, rows_per_rule=16, seed=65536) -> dict:
    """CPU side of the N=65536 chain workload: the closure property of the
    device's fixpoint checked with the oracle on a row sample -- for every
    rule C -> A B, rows R of C | A * B equal rows R of C (a dense CPU closure
    at this size takes hours).  All host threads."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the checker

    n = q.mats[0].n
    rng = np.random.default_rng(seed)
    rows = np.unique(np.concatenate([rng.choice(n, rows_per_rule - 2, replace=False), [0, n - 1]]))
    rows = rows.astype(np.uint32)
    t0 = time.perf_counter()
    host = [m.download_rows() for m in q.mats]
    ok, bad = True, []
    for r, (head, b1, b2) in enumerate(wl.grammar.rules):
        got = oracle.add_mul_rows(host[head], host[b1], host[b2], n, rows, os.cpu_count() or 1)
        if not np.array_equal(got, host[head][rows]):
            ok = False
            bad.append(r)
    return {"closure_property_holds": ok, "rules": len(wl.grammar.rules), "rows_per_rule": int(rows.size),
            "failing_rules": bad, "cpu_s": time.perf_counter() - t0,
            "check": "for every rule C -> A B: rows of C | A*B (oracle row gather) == rows of C at the fixpoint"}


def reference_naive_product_ms(n: int, log2_inv_density: int = 1, reps: int = 1) -> dict:
    """The reference's naive GPU product (gpu_lib::matrix_product_add_wrapper,
    built from its sources for sm_100a under oracle/_ref/naiveGPU-product) on
    random n x n matrices of density 2^-log2_inv_density."""
    exe = os.path.join(ROOT, "oracle", "_ref", "naiveGPU-product")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/naiveGPU-product not built"}
    try:
        p = subprocess.run([exe, str(n), str(log2_inv_density), str(reps), "7"], capture_output=True, text=True,
                           timeout=900)
    except subprocess.TimeoutExpired:
        return {"error": "timed out after 900 s"}
    if p.returncode != 0:
        return {"error": (p.stdout + p.stderr)[-300:]}
    return {"ms": float(p.stdout.split()[1]), "density": 2.0 ** -log2_inv_density}


def chain_bench(pkg, ctx, torch, stream, n=65536, seed=1) -> dict:
    """The large chain workload: N = 65536 (512 MiB per matrix), mean
    out-degree 2, 90% of edges with |u-v| <= 64 and 10% uniform, 6 labels,
    random CNF with 10 nonterminals and 24 binary rules; one closure with the
    selector choosing LOP3 / Four Russians / tensor cores per term and
    iteration (device time, CUDA events), its closure property checked on the
    CPU on a row sample, and per-product times at this n on random matrices of
    density 0.5 for every engine variant, the plain single-variant form and
    the reference's naive GPU product."""
    import numpy as np

    wl = pkg.workloads.chain_query(n, seed)
    before = ctx.selector_config()
    ctx.selector_configure(min_tiles=1)  # a single query selects per term
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    out = {"n": n, "seed": seed, "edges": wl.graph.nedges, "nonterminals": len(wl.grammar.nonterminals),
           "rules": len(wl.grammar.rules)}
    try:
        q.load()
        ctx.synchronize()
        ms, st = _event_ms(torch, stream, lambda: ctx.closure(wl.grammar.rules, q.mats, variant="auto"))
        out.update({"closure_s": ms / 1e3, "iterations": st["iterations"], "products": st["products"],
                    "tile_triples": st["tile_triples"],
                    "executed_tbitmac_per_s": st["tile_triples"] * 64 ** 3 / (ms / 1e3) / 1e12,
                    "dense_equiv_tbitmac_per_s": st["dense_bitops"] / (ms / 1e3) / 1e12,
                    "variant_items": {"lop3": st["variant_items"][2], "m4r": st["variant_items"][3],
                                      "tc": st["variant_items"][4]},
                    "result": {k: list(v) for k, v in zip(wl.grammar.nonterminals, ctx.hash_count_many(q.mats))}})
        out["parity"] = chain_cpu_check(wl, q)
    finally:
        q.close()
        ctx.selector_configure(**{k: before[k] for k in ("mode", "min_tiles", "tc_min_tiles")})
    # per-product times on random density-0.5 operands
    rng = np.random.default_rng(seed)
    wpr = n // 64
    a, b, c = ctx.matrix(n), ctx.matrix(n), ctx.matrix(n)
    try:
        for m in (a, b):
            m.upload_rows(rng.integers(0, 2 ** 63, size=(n, wpr), dtype=np.uint64)
                          | (rng.integers(0, 2, size=(n, wpr), dtype=np.uint64) << np.uint64(63)))
        per = {}
        ref_hash = None
        for variant in ("tc", "m4r", "lop3", "plain"):
            c.clear()
            ctx.synchronize()
            t, _ = _event_ms(torch, stream, lambda: ctx.add_mul(c, a, b, variant))
            h = c.hash_count()
            ref_hash = ref_hash or h
            per[variant] = {"ms": t, "tbitmac_per_s": n ** 3 / (t / 1e3) / 1e12, "same_result": h == ref_hash}
        out["per_product_random_d05"] = per
    finally:
        for m in (a, b, c):
            m.destroy()
    out["per_product_random_d05"]["reference_naiveGPU"] = reference_naive_product_ms(n)
    ref_ms = out["per_product_random_d05"]["reference_naiveGPU"].get("ms")
    best = min(v["ms"] for k, v in out["per_product_random_d05"].items() if k in ("tc", "m4r", "lop3"))
    out["per_product_speedup"] = {"vs_plain_form": per["plain"]["ms"] / best,
                                  "vs_reference_naiveGPU": ref_ms / best if ref_ms else None}
    return out


def brackets_small(pkg, ctx, torch, stream, reps=20) -> dict:
    """Balanced brackets on a random graph, N = 1024, 4096 edges."""
    wl = pkg.workloads.brackets_query()
    q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
    try:
        ms = []
        for _ in range(reps + 3):
            q.load()
            ctx.synchronize()
            ms.append(_event_ms(torch, stream, lambda: ctx.closure(wl.grammar.rules, q.mats))[0])
        t = statistics.median(ms[3:])
        return {"n": 1024, "edges": wl.graph.nedges, "ms": t, "closures_per_s": 1e3 / t}
    finally:
        q.close()


def _logged_records(pkg, ctx, queries):
    """CFPQ_LOG_PRODUCTS run of a batch (exhaustive timing of every candidate
    variant of every term in every iteration); records and their keys."""
    for q in queries:
        q.load()
    ctx.closure_batch([(q.grammar.rules, q.mats) for q in queries], log_products=pkg.capi.LOG_PRODUCTS)
    return ctx.product_log()


def _regret(recs, choice) -> float:
    """sum of the chosen variants' times / sum of the fastest timed variant's - 1."""
    import numpy as np

    t = recs["usec"][:, 2:5].astype(np.float64)
    timed = t > 0
    best = np.where(timed, t, np.inf).min(axis=1)
    idx = np.asarray(choice) - 2
    chosen = t[np.arange(len(t)), idx]
    ok = timed[np.arange(len(t)), idx] & np.isfinite(best)
    return float(chosen[ok].sum() / best[ok].sum() - 1.0)


def selector_eval(pkg, ctx, torch, stream, n_train=32, n_eval=32) -> dict:
    """The learned selector (cfg5 shape): train the cost model on product
    timings logged from brackets (N=1024), same-generation (N=8192) and a
    32-query batch of the mixed-query shape, then evaluate on a fresh-seed
    32-query batch: regret against exhaustive per-term timing for the
    heuristic, the MLP and each fixed variant, and the batch closure time
    with each selector."""
    import numpy as np

    # logging: tensor cores are a candidate for terms of n >= 4096
    ctx.selector_configure(mode="heuristic", min_tiles=1, tc_min_tiles=64)
    cfg = ctx.selector_config()
    train = []
    t0 = time.perf_counter()
    for wl in (pkg.workloads.brackets_query(), pkg.workloads.ontology_query(8192, 7)):
        q = pkg.query.PreparedQuery(ctx, wl.grammar, wl.graph)
        train.append(_logged_records(pkg, ctx, [q]))
        q.close()
    tr_wls = pkg.workloads.batch_queries(n_train, seed=101, n_max=8192)
    tr_qs = [pkg.query.PreparedQuery(ctx, w.grammar, w.graph) for w in tr_wls]
    train.append(_logged_records(pkg, ctx, tr_qs))
    for q in tr_qs:
        q.close()
    train = np.concatenate(train)
    log_s = time.perf_counter() - t0
    rep = ctx.selector_train(train, epochs=3000, learning_rate=3e-3, weight_decay=1e-4, seed=1)
    ev_wls = pkg.workloads.batch_queries(n_eval, seed=202, n_max=8192)
    ev_qs = [pkg.query.PreparedQuery(ctx, w.grammar, w.graph) for w in ev_wls]
    out = {"train_records": int(len(train)), "logging_s": log_s, "train": rep, "config": cfg}
    try:
        ctx.selector_configure(mode="heuristic", min_tiles=1, tc_min_tiles=64)
        rec_h = _logged_records(pkg, ctx, ev_qs)
        ctx.selector_configure(mode="mlp", min_tiles=1, tc_min_tiles=64, conf_margin=0.0)
        rec_m = _logged_records(pkg, ctx, ev_qs)
        key = lambda r: (int(r["query"]), int(r["rule"]), int(r["term"]), int(r["iteration"]))
        hmap = {key(r): int(r["variant"]) for r in rec_h}
        common = np.array([key(r) in hmap for r in rec_m])
        rm = rec_m[common]
        heur = [hmap[key(r)] for r in rm]
        tc_ok = rm["usec"][:, 4] > 0
        out["eval_records"] = int(len(rm))
        out["regret"] = {
            "mlp": _regret(rm, rm["variant"]),
            "heuristic": _regret(rm, heur),
            "fixed_lop3": _regret(rm, np.full(len(rm), 2)),
            "fixed_m4r": _regret(rm, np.full(len(rm), 3)),
            "tc_where_possible": _regret(rm, np.where(tc_ok, 4, 2)),
        }
        out["mlp_decided_fraction"] = float(((rm["flags"] >> 8) & 1).mean())
        # batch closure time of the fresh queries with each selector (the
        # default tensor-core size limit, n >= 16384, keeps these terms on the
        # word-level kernels: the choice is LOP3 or M4R per term and iteration)
        # in the persistent loop (8-warp kernel, the default) and in the CUDA-
        # graph loop (the plan + product kernels whose timings the model was
        # trained on)
        times, times_graph = {}, {}
        for label, kw in (("fixed_lop3", dict(mode="fixed")),
                          ("heuristic", dict(mode="heuristic", min_tiles=1, tc_min_tiles=256)),
                          ("mlp", dict(mode="mlp", min_tiles=1, tc_min_tiles=256, conf_margin=0.0))):
            ctx.selector_configure(**kw)
            for loop, dest in (("device", times), ("graph", times_graph)):
                ms = []
                for _ in range(3):
                    for q in ev_qs:
                        q.load()
                    ctx.synchronize()
                    ms.append(_event_ms(torch, stream, lambda: ctx.closure_batch(
                        [(q.grammar.rules, q.mats) for q in ev_qs], use_graph=loop))[0])
                dest[label] = min(ms)
        out["batch_closure_ms"] = times
        out["batch_closure_ms_graph_loop"] = times_graph
    finally:
        for q in ev_qs:
            q.close()
        ctx.selector_configure(mode="heuristic", min_tiles=256, tc_min_tiles=256)
    return out


def dense_product_kernels(ctx, capi, torch, stream, n=8192, density=0.3, reps=3):
    """One dense product C |= A*B (n=8192, every tile populated) per variant:
    the word-level rooflines.  Dense-equivalent work n^3 bit-MACs; LOP3 bound
    = 32 bit-MACs per logic instruction at the calibrated logic rate."""
    import numpy as np

    rng = np.random.default_rng(5)
    wpr = n // 64
    rows = [np.packbits(rng.random((n, n)) < density, axis=1, bitorder="little").view(np.uint64).reshape(n, wpr)
            for _ in range(2)]
    a, b, c = ctx.matrix(n), ctx.matrix(n), ctx.matrix(n)
    a.upload_rows(rows[0])
    b.upload_rows(rows[1])
    cal = ctx.calibrate()
    out = {"n": n, "density": density, "calibrated_logic_ops_per_s": cal["logic_ops_per_s"],
           "calibrated_logic_ops_per_clk_sm": cal["logic_ops_per_clk_sm"], "variants": {}}
    for variant in ("tc", "lop3", "m4r", "plain"):
        ms = []
        for _ in range(reps if variant != "plain" else 1):
            c.clear()
            ctx.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.add_mul(c, a, b, variant)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        t = min(ms)
        rate = n ** 3 / (t / 1e3)
        out["variants"][variant] = {"ms": t, "tbitmac_per_s": rate / 1e12,
                                    "frac_of_lop3_bound": rate / cal["bitmac_per_s"]}
    for m in (a, b, c):
        m.destroy()
    return out


def ours_arm(args, world, rank, local):
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod
    pkg = importlib.import_module("cfpq-on-gpgpu_b200")
    capi, query = pkg.capi, pkg.query
    wl = pkg.workloads.ontology_query(N_VERTICES, args.seed + rank)
    grammar, graph = wl.grammar, wl.graph
    ctx = capi.Context(local)
    q = query.PreparedQuery(ctx, grammar, graph)
    stream = torch.cuda.ExternalStream(ctx.stream)
    # device-resident edge list (value) and pinned host copy (e2e)
    d_src = torch.from_numpy(graph.src.view(np.int32)).cuda()
    d_lab = torch.from_numpy(graph.label.view(np.int32)).cuda()
    d_dst = torch.from_numpy(graph.dst.view(np.int32)).cuda()
    h_src = torch.from_numpy(graph.src.view(np.int32)).pin_memory().numpy().view(np.uint32)
    h_lab = torch.from_numpy(graph.label.view(np.int32)).pin_memory().numpy().view(np.uint32)
    h_dst = torch.from_numpy(graph.dst.view(np.int32)).pin_memory().numpy().view(np.uint32)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2

    launches = {"n": 0}
    device_ms: list[float] = []

    dev_edges = (d_src.data_ptr(), d_lab.data_ptr(), d_dst.data_ptr())

    def step_value():
        # cfpq_intersection: clear + edge scatter + epsilon diagonals +
        # closure, enqueued back to back, one synchronisation
        st, _ = ctx.intersection(grammar.rules, q.mats, *dev_edges, q.off, q.lm, epsilon=grammar.epsilon,
                                 nedges=graph.nedges, use_graph=not args.no_graph, lines=False)
        launches["n"] += st["kernel_launches"]  # input kernels + closure, as the library counts them
        device_ms.append(st["device_ms"])
        return st

    def step_e2e():
        # the same from pinned host edges, with the result lines copied back
        return ctx.intersection(grammar.rules, q.mats, h_src, h_lab, h_dst, q.off, q.lm, epsilon=grammar.epsilon,
                                use_graph=not args.no_graph, lines=True)

    def timed(fn, k):
        times, last = [], None
        # events created (and their CUDA events allocated by a first record)
        # before the timed loop, so that no event creation falls inside a step
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for e0, e1 in evs:
            e0.record(stream)
            e1.record(stream)
        torch.cuda.synchronize()
        for e0, e1 in evs:
            e0.record(stream)
            last = fn()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            flush.zero_()
            torch.cuda.synchronize()
        return times, last

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # correctness gate on this rank's instance: device result == host result of the first closure
    for _ in range(args.warmup):
        step_value()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    launches["n"] = 0
    device_ms.clear()
    times, st = timed(step_value, args.steps)
    clocks = sampler.stop()
    barrier()
    total_ms = max_over_ranks(sum(times))
    gpu_launches = launches["n"]
    phases = ctx.phase_log()  # per-iteration (plan, products) us of the last persistent closure
    value = world * args.steps / (total_ms / 1e3)

    # end to end through the C ABI with host buffers
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    barrier()
    e2e_times, (st_e2e, lines) = timed(step_e2e, args.steps)
    barrier()
    e2e_total = max_over_ranks(sum(e2e_times))
    e2e_value = world * args.steps / (e2e_total / 1e3)
    h2d = 3 * 4 * graph.nedges + 4 * (q.off.size + q.lm.size)
    d2h = 16 * len(q.mats)

    # roofline of the dominant kernel, the persistent closure kernel (one
    # launch per step, its duration the library's event pair around it):
    # bound by the logic-instruction issue rate (32 bit-MACs per LOP3 on a
    # 32-bit lane), measured on the executed tile triples (64^3 bit-MACs
    # each); HBM beside it with the tile model's algorithmic bytes
    peaks = measured_peaks()
    cal = ctx.calibrate()
    dev_ms = statistics.mean(device_ms) if device_ms else 0.0
    executed = st["tile_triples"] * 64 ** 3
    achieved = executed / (dev_ms / 1e3) / 1e12 if dev_ms > 0 else 0.0
    peak = cal["bitmac_per_s"] / 1e12
    tr = committed_traffic().get("k_closure_persistent", {}).get("dram_bytes_per_launch")
    model = tile_model_bytes(ctx, q, grammar, st["iterations"])
    hbm_achieved = model["bytes"] / (dev_ms / 1e3) / 1e9 if dev_ms > 0 else 0.0
    roofline = {"kernel": "k_closure_persistent" if len(phases) else "closure iteration kernels",
                "bound": "lop3_issue", "achieved": achieved, "peak": peak, "unit": "Tbit-MAC/s",
                "frac": achieved / peak if peak else None, "traffic": tr,
                "peak_source": f"calibrated on this GPU (cfpq_calibrate: register-only 3-input logic chains, "
                               f"{cal['logic_ops_per_clk_sm']:.1f} ops/clk/SM x 32 bit-MACs per op)",
                "avg_launch_ms": dev_ms, "executed_bitmac_per_launch": executed,
                "executed": "tile_triples x 64^3 (tile pairs skipped as empty are not counted)",
                "hbm": {"bound": "hbm", "algorithmic_bytes_per_launch": model["bytes"], "achieved": hbm_achieved,
                        "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": hbm_achieved / peaks["hbm_gbs"],
                        "traffic": tr, "peak_source": peaks["source"],
                        "algorithmic_bytes": "per product term: (occupied P tiles + occupied Q tiles in the "
                                             "rows P's columns select + 2 x output tiles reached) x 512 B",
                        "tile_model": model},
                "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch "
                                "(profiles/traffic.json); the operands stay in L2 across iterations",
                "note": "latency-bound: a few hundred short work items per iteration; see phase_us_per_iteration "
                        "and the dense_product_kernels rooflines"}
    if not args.no_profile:
        # per-kernel times of the multi-kernel iteration (host loop, every launch bracketed by events)
        ctx.clear_many(q.mats)
        ctx.load_edges_device(q.mats, d_src.data_ptr(), d_lab.data_ptr(), d_dst.data_ptr(), graph.nedges,
                              q.off, q.lm)
        ctx.closure(grammar.rules, q.mats, use_graph=False, log_products=capi.LOG_KERNELS)
        prof = ctx.kernel_profile()
        roofline["multi_kernel_path_ms"] = {"plan": prof["plan_ms"], "product": prof["product_ms"],
                                            "advance_end": prof["advance_ms"]}

    batch = None if args.no_extras else batch_bench(pkg, ctx, torch, stream, rank, world, dist)

    out = None
    if rank == 0:
        out = {
            "metric": "CFPQ closure throughput (same-generation query, N=8192)",
            "value": value, "unit": "closures/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 (bit-packed Boolean)",
            "data": "synthetic (seeded ontology-like graph, MT19937)",
            "config": {"workload": "same_generation_ontology_n8192", "n": N_VERTICES, "edges": graph.nedges,
                       "nonterminals": len(grammar.nonterminals), "rules": len(grammar.rules),
                       "seed": args.seed, "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"query-partitioned x{world}",
                       "launch": "host loop" if args.no_graph else
                       ("one persistent cooperative kernel per closure" if len(phases) else
                        "CUDA graph (conditional while node)")},
            "clocks": clocks,
            "e2e": {"value": e2e_value, "unit": "closures/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": gpu_launches,
            "roofline": roofline,
            "closure": {"iterations": st["iterations"], "products": st["products"], "work_items": st["work_items"],
                        "tile_triples": st["tile_triples"], "device_ms_last": st["device_ms"],
                        "dense_equiv_gbitops": st["dense_bitops"] / (total_ms / args.steps / 1e3) / 1e9,
                        "loop": "persistent kernel" if len(phases) else "CUDA graph",
                        "phase_us_per_iteration": {"plan": float(phases[:, 0].mean()),
                                                   "products": float(phases[:, 1].mean())} if len(phases) else None,
                        "result": {k: list(v) for k, v in zip(grammar.nonterminals, lines)}},
        }
        if not args.no_profile:
            out["dense_product_kernels"] = dense_product_kernels(ctx, capi, torch, stream)
        if not args.no_extras:
            expected = {k: tuple(v) for k, v in zip(grammar.nonterminals, lines)}
            pf = plain_gpu_form(ctx, q, grammar, torch, stream)
            pf["engine_speedup"] = value / pf["closures_per_s"]
            out["plain_gpu_form"] = pf
            out["reference_gpu"] = reference_gpu_forms(wl, expected)
            out["brackets_n1024"] = brackets_small(pkg, ctx, torch, stream)
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(wl)
            answer = cb.pop("answer")
            out["cpu_baseline"] = cb
            out["closure"]["parity_vs_cpu"] = answer == {k: tuple(v) for k, v in zip(grammar.nonterminals, lines)}
        if batch is not None:
            out["batch_512"] = batch
        if world == 1 and not args.no_extras and not args.no_selector_eval:
            out["selector_eval"] = selector_eval(pkg, ctx, torch, stream)
        if world == 1 and not args.no_extras and not args.no_chain:
            out["chain_65536"] = chain_bench(pkg, ctx, torch, stream)
        print(json.dumps(out))
    q.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()


def main():
    args = parse_args()
    world, rank, local = dist_env()
    if args.impl == "reference":
        reference_arm(args, world, rank)
        return
    ours_arm(args, world, rank, local)


if __name__ == "__main__":
    main()
