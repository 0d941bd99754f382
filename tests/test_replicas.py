"""Multi-GPU replicas on the CPU: job placement (the gpulock device choice)
and the one-process-per-GPU plumbing run as world-size-2 gloo ranks."""
import json
import os
import socket

import pytest

from zk_gpu_b200.replicas import ReplicaGroup, place_job, rank_seed


def test_place_job_fewest_running_then_room():
    cap = [100, 100, 100]
    assert place_job(10, [2, 1, 1], [0, 0, 0], cap) == 1          # fewest running, lowest index
    assert place_job(10, [2, 1, 1], [0, 95, 0], cap) == 2         # device 1 has no room
    assert place_job(10, [0, 0, 0], [91, 91, 90], cap) == 2
    assert place_job(10, [0, 0, 0], [91, 91, 91], cap) == -1      # nobody can take it: wait
    assert place_job(0, [0], [100], [100]) == 0
    assert place_job(101, [0, 0], [0, 0], [100, 100]) == -1       # larger than any device


def test_place_job_spreads_a_stream():
    running, used, cap = [0, 0, 0, 0], [0, 0, 0, 0], [10**9] * 4
    seen = []
    for _ in range(8):
        d = place_job(1000, running, used, cap)
        running[d] += 1
        used[d] += 1000
        seen.append(d)
    assert seen == [0, 1, 2, 3, 0, 1, 2, 3]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import numpy as np
    from oracle import pyoracle as zo
    g = ReplicaGroup("gloo", timeout_s=60)
    try:
        assert (g.rank, g.world) == (rank, world)
        # each replica transforms its own seeded input; rank 0 reports
        seed = rank_seed(100, rank)
        a = zo.rand_fr(1 << 8, seed)
        w = zo.omega(8)
        ok = np.array_equal(zo.best_fft(a, w, 8), zo.naive_dft(a, w))
        g.barrier()
        res = {"max": g.max(1.5 + rank), "sum": g.sum(1.0 + rank), "all_ok": g.all_ok(ok),
               "one_fails": g.all_ok(rank == 0), "seed": seed}
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        g.close()


def test_two_gloo_replicas(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["max"] == 2.5
        assert r["sum"] == 3.0
        assert r["all_ok"] is True
        assert r["one_fails"] is False
    assert res[0]["seed"] != res[1]["seed"]
