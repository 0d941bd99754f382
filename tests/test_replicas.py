"""Multi-GPU replicas on the CPU: job placement (the gpulock device choice),
the placement layer over per-device servers (stand-in servers, no GPU), and
the one-process-per-GPU plumbing run as world-size-2 gloo ranks."""
import json
import os
import random
import socket
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import pytest

from zk_gpu_b200.replicas import MultiGpuServer, ReplicaGroup, place_job, rank_seed


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


class FakeServer:
    """Stand-in for one device's zk.Server: a job 'runs' from submit for a
    random 1-5 ms (the reference test sleeps 1-5 s per task), or until its
    `hold` event is set; it records the bytes in flight on the device."""

    def __init__(self, device, capacity, fail_kinds=()):
        self.device, self.capacity, self.fail_kinds = device, capacity, set(fail_kinds)
        self.mu = threading.Lock()
        self.jobs, self.next = {}, 0
        self.in_flight = self.peak = 0
        self.closed = False

    def submit(self, job, keep=None):
        with self.mu:
            t = self.next
            self.next += 1
            self.in_flight += job["bytes"]
            self.peak = max(self.peak, self.in_flight)
            self.jobs[t] = (job, time.monotonic(), random.uniform(0.001, 0.005))
            return t

    def wait(self, t, timeout_ms=0):
        job, t0, dur = self.jobs[t]
        if job.get("hold") is not None:
            job["hold"].wait()
        else:
            time.sleep(max(0.0, t0 + dur - time.monotonic()))
        with self.mu:
            self.in_flight -= job["bytes"]
            del self.jobs[t]
        if job.get("kind") in self.fail_kinds:
            raise RuntimeError(f"job failed on device {self.device}")
        return (time.monotonic() - t0) * 1e3

    def add_bases(self, bases):
        return 0

    def close(self):
        self.closed = True


def _multi(ndev=4, capacity=11000, **kw):
    fakes = {}

    def factory(d):
        fakes[d] = FakeServer(d, capacity, **kw)
        return fakes[d]

    srv = MultiGpuServer(list(range(ndev)), hbm_budget=capacity, server_factory=factory,
                         footprint=lambda j: j["bytes"])
    return srv, fakes


def test_hundred_concurrent_tasks_release_everything():
    """src/gpulock.rs:272-302 (test_gpulock): 100 tasks from a worker pool on
    LOCKER_4GPU (4 devices x 11000 MB), each needing 10, 3300 or 6700 MB;
    afterwards every device's used memory and running count are back at 0."""
    random.seed(7)
    srv, fakes = _multi()

    def task(i):
        job = {"bytes": random.choice([10, 3300, 6700]), "kind": "x"}
        t = srv.submit(job, timeout_s=30)
        lat = srv.wait(t)
        return lat

    with ThreadPoolExecutor(max_workers=16) as ex:
        lats = list(ex.map(task, range(100)))
    assert len(lats) == 100 and all(v >= 0 for v in lats)
    c = srv.counters()
    assert c["used"] == [0, 0, 0, 0] and c["running"] == [0, 0, 0, 0] and c["in_flight"] == 0
    assert sum(c["placed"]) == 100 and all(p > 0 for p in c["placed"])
    for f in fakes.values():
        assert f.peak <= f.capacity and f.in_flight == 0
    srv.close()
    assert all(f.closed for f in fakes.values())


def test_budget_released_without_wait():
    srv, fakes = _multi(ndev=2, capacity=1000)
    tickets = [srv.submit({"bytes": 400}, timeout_s=10) for _ in range(6)]  # > 2 x 1000 bytes in total
    deadline = time.monotonic() + 10
    while srv.counters()["in_flight"] and time.monotonic() < deadline:
        time.sleep(0.002)
    c = srv.counters()
    assert c["used"] == [0, 0] and c["running"] == [0, 0]
    # results stay available until taken
    assert all(srv.wait(t) >= 0 for t in tickets)
    srv.close()


def test_submit_blocks_until_room_then_times_out():
    srv, fakes = _multi(ndev=1, capacity=100)
    hold = threading.Event()
    t1 = srv.submit({"bytes": 80, "hold": hold})
    with pytest.raises(TimeoutError):
        srv.submit({"bytes": 80}, timeout_s=0.05)
    got = []
    th = threading.Thread(target=lambda: got.append(srv.submit({"bytes": 80}, timeout_s=10)))
    th.start()
    time.sleep(0.02)
    assert not got  # still blocked: the device is full
    hold.set()
    th.join(10)
    assert got and srv.wait(t1) >= 0 and srv.wait(got[0]) >= 0
    assert srv.counters()["used"] == [0]
    with pytest.raises(ValueError):
        srv.submit({"bytes": 101})
    srv.close()


def test_failed_job_releases_and_reraises():
    srv, fakes = _multi(ndev=2, capacity=1000, fail_kinds=("bad",))
    tb = srv.submit({"bytes": 500, "kind": "bad"})
    tg = srv.submit({"bytes": 500, "kind": "good"})
    with pytest.raises(RuntimeError):
        srv.wait(tb)
    assert srv.wait(tg) >= 0
    assert srv.counters()["used"] == [0, 0]
    with pytest.raises(KeyError):
        srv.wait(tb)  # already taken
    srv.close()
