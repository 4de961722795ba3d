"""The multi-GPU path is replicas only: N independent runs, one per rank, no data-path
collective; timings are the maximum over ranks. These CPU tests run that host logic as two
`gloo` ranks (spawned processes, rendezvous on 127.0.0.1)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime
    import torch
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # max over ranks of a per-rank time
        t = bench.max_over_ranks(dist, 1.5 + rank, device="cpu")
        bench.rank_barrier(dist, device="cpu")
        # each rank's ensemble replica: same droplet distribution, its own noise seeds
        w = bench.WORKLOADS["quench_ensemble_128"]
        inst = bench.ensemble_instances(w, rank)
        seeds = torch.tensor([d["seed"] for d in inst], dtype=torch.int64)
        gathered = [torch.zeros_like(seeds) for _ in range(world)]
        dist.all_gather(gathered, seeds)
        radii = torch.tensor([d["droplet_radius_cells"] for d in inst])
        rg = [torch.zeros_like(radii) for _ in range(world)]
        dist.all_gather(rg, radii)
        out[rank] = (t, [g.tolist() for g in gathered], [r.tolist() for r in rg])
    finally:
        dist.destroy_process_group()


def test_replicas_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    for r in range(2):
        t, seeds, radii = out[r]
        assert t == 2.5                       # the slower rank's time
        assert set(seeds[0]).isdisjoint(seeds[1])
        assert radii[0] == radii[1]           # weak scaling: identical work per rank


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        pass
    a = A()
    a.ref_grid, a.steps, a.warmup, a.gpus, a.workload = 16, 1, 0, 2, bench.DEFAULT_WORKLOAD
    assert bench.run_reference_arm(a, bench.WORKLOADS[bench.DEFAULT_WORKLOAD]) == 0
    assert capsys.readouterr().out == ""
