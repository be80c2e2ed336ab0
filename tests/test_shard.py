"""Query sharding of batched closures: LPT balance, and a world-size-2 gloo run
on CPU where each rank closes its share with the CPU oracle and the gathered
result equals the single-process one."""
import importlib
import os
import socket
import tempfile

import pytest
import torch.multiprocessing as mp


def _shard():
    return importlib.import_module("cfpq-on-gpgpu_b200.shard")


def test_lpt_balances_and_covers():
    shard = _shard()
    costs = [shard.query_cost(n, 6) for n in (8192, 256, 4096, 4096, 1024, 300, 7000, 512, 2048)]
    shares = shard.lpt_assign(costs, 3)
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in shares]
    # LPT bound: max load <= 4/3 of the optimum, optimum >= max(total / m, largest job)
    opt_lb = max(sum(costs) / 3, max(costs))
    assert max(loads) <= 4 / 3 * opt_lb + 1e-6
    assert shard.lpt_assign([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.lpt_assign([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle

    pkg = importlib.import_module("cfpq-on-gpgpu_b200")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        wls = pkg.workloads.batch_queries(10, seed=3, n_min=64, n_max=300)
        costs = [pkg.shard.query_cost(w.graph.n, len(w.grammar.rules)) for w in wls]
        mine = pkg.shard.lpt_assign(costs, world)[rank]
        local = {}
        for i in mine:
            d = os.path.join(outdir, f"r{rank}_q{i}")
            os.makedirs(d)
            gp, rp = os.path.join(d, "g.txt"), os.path.join(d, "r.txt")
            wls[i].write(gp, rp)
            with oracle.Problem(gp, rp) as p:
                p.closure(oracle.M4RM, 1)
                local[i] = p.results()
        merged = pkg.shard.gather_lines(dist, local)
        if rank == 0:
            import json

            with open(os.path.join(outdir, "merged.json"), "w") as f:
                json.dump({str(k): {n: list(v) for n, v in lines.items()} for k, lines in merged.items()}, f)
    finally:
        dist.destroy_process_group()


def test_two_rank_batch_matches_single_process(oracle, pkg, tmp_path):
    import json

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    merged = json.load(open(tmp_path / "merged.json"))
    wls = pkg.workloads.batch_queries(10, seed=3, n_min=64, n_max=300)
    assert sorted(int(k) for k in merged) == list(range(10))
    for i, wl in enumerate(wls):
        d = tempfile.mkdtemp(dir=tmp_path)
        gp, rp = os.path.join(d, "g.txt"), os.path.join(d, "r.txt")
        wl.write(gp, rp)
        with oracle.Problem(gp, rp) as p:
            p.closure(oracle.M4RM, 1)
            exp = p.results()
        assert {n: tuple(v) for n, v in merged[str(i)].items()} == exp
