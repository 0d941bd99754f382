"""Multi-GPU replicas: the hot path does not shard (a 2^26 transform or a
2^22 MSM fits one GPU's HBM many times over), so N GPUs run N independent
replicas.  Two pieces live here:

* ``ReplicaGroup`` — the per-process plumbing of a one-process-per-GPU run
  (``torch.distributed``; NCCL on GPUs, gloo on CPU): rank identity, seeds
  that differ per rank, a barrier, and the max/sum over ranks used to time a
  job on the device as the slowest rank.  No data-path collective exists.
* ``place_job`` / ``MultiGpuServer`` — device-id placement of jobs over the
  local GPUs, the role of ``GpuLock::acquire_gpu`` (src/gpulock.rs:131-200)
  and ``config::get_gpu`` (src/config.rs:97-127): the device with the fewest
  running jobs is tried, and a job is admitted there only while that
  device's memory counter has room for the job's footprint.
"""
from __future__ import annotations

import datetime
import os


def rank_env() -> tuple:
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def rank_seed(base: int, rank: int) -> int:
    """Seeds differ per rank so replicas do not process identical inputs."""
    return base + 7919 * rank


class ReplicaGroup:
    """Process-group plumbing for N replicas (world 1: no process group)."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 120.0):
        self.rank, self.world, self.local_rank = rank_env()
        self.dist = None
        self.device = device
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.dist is None:
            return float(x)
        import torch
        dev = self.device if (self.device is not None and self.dist.get_backend() == "nccl") else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        """max over ranks (job time = the slowest replica's device time)"""
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)

    def all_ok(self, ok: bool) -> bool:
        """True iff every rank passed (e.g. every replica's parity check)"""
        return self._reduce(0.0 if ok else 1.0, self.dist.ReduceOp.MAX if self.dist else None) == 0.0

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def place_job(footprint: int, running: list, used: list, capacity: list) -> int:
    """Device for a job of `footprint` bytes, or -1 if none can take it now.

    The device with the fewest running jobs is tried first (ties: the lowest
    index, where the reference shuffles); a device admits the job only if its
    used bytes plus the footprint stay within its capacity.  The reference
    tests ``mem_total > mem_used`` before adding (src/gpulock.rs:178), which
    can overshoot by one job; this check cannot."""
    order = sorted(range(len(running)), key=lambda d: (running[d], d))
    for d in order:
        if used[d] + footprint <= capacity[d]:
            return d
    return -1


class MultiGpuServer:
    """One serving loop (zk.Server) per local GPU; each job goes to a device
    chosen by place_job, the role of GpuLock::acquire_gpu / release_gpu
    (src/gpulock.rs:133-226).

    Two ledgers exist on purpose, at two levels.  This object's per-device
    counters (bytes placed, jobs running) decide WHICH device takes a job,
    before the job is queued anywhere, as GpuLock's mem_used / running_tasks
    do.  Each device's Server then enforces its HBM budget at execution time
    (its admission queue also holds the resident bases, which the placement
    ledger does not see) and decides WHEN the job starts.

    Thread safety: every counter is read and written under one condition
    variable.  Release happens on completion, not in wait(): a reaper thread
    per device waits for that device's jobs in submission order (a Server
    retires jobs in admission order, which is submission order) and gives
    their bytes back at once, so a job that is never waited on does not hold
    its budget; its result stays available to wait() until taken.
    submit() blocks while no device has room (the reference's acquire_gpu
    blocks the same way), up to an optional timeout.

    Bases added here are made resident on every device.  `server_factory`
    (device -> server object with submit / wait / close / add_bases) lets
    tests run the placement logic against stand-in servers without a GPU."""

    def __init__(self, devices: list, hbm_budget: int = 150 * 10**9, max_wave_jobs: int = 256,
                 server_factory=None, footprint=None):
        import collections
        import threading
        if server_factory is None:
            from . import Server

            def server_factory(d):
                return Server(d, hbm_budget, max_wave_jobs)
        if footprint is None:
            from . import job_footprint as footprint
        self._footprint = footprint
        self.devices = list(devices)
        self.servers = [server_factory(d) for d in self.devices]
        self.capacity = [hbm_budget] * len(self.devices)
        self.used = [0] * len(self.devices)
        self.running = [0] * len(self.devices)
        self.placed = [0] * len(self.devices)
        self._cv = threading.Condition()
        self._where = {}       # ticket -> (device index, server ticket, bytes)
        self._results = {}     # ticket -> (exception or None, latency ms)
        self._queues = [collections.deque() for _ in self.devices]
        self._next = 0
        self._closing = False
        self._reapers = [threading.Thread(target=self._reap, args=(i,), daemon=True)
                         for i in range(len(self.devices))]
        for t in self._reapers:
            t.start()

    def add_bases(self, bases) -> int:
        ids = {s.add_bases(bases) for s in self.servers}
        assert len(ids) == 1, "base ids diverged across devices"
        return ids.pop()

    def submit(self, job, keep=None, timeout_s: float | None = None) -> int:
        """Place the job and queue it on that device's server; returns a
        ticket.  Blocks while no device has room; raises TimeoutError after
        timeout_s, and ValueError for a job larger than every device."""
        fp = int(self._footprint(job))
        if fp > max(self.capacity):
            raise ValueError(f"job footprint {fp} exceeds every device's budget")
        with self._cv:
            if self._closing:
                raise RuntimeError("MultiGpuServer is closed")
            ok = self._cv.wait_for(lambda: place_job(fp, self.running, self.used, self.capacity) >= 0,
                                   timeout=timeout_s)
            if not ok:
                raise TimeoutError("no device had room for the job in time")
            d = place_job(fp, self.running, self.used, self.capacity)
            t = self.servers[d].submit(job, keep)  # non-blocking; raises on rejection
            self.used[d] += fp
            self.running[d] += 1
            self.placed[d] += 1
            ticket = self._next
            self._next += 1
            self._where[ticket] = (d, t, fp)
            self._queues[d].append(ticket)
            self._cv.notify_all()
        return ticket

    def _reap(self, d: int):
        while True:
            with self._cv:
                self._cv.wait_for(lambda: self._queues[d] or self._closing)
                if not self._queues[d]:
                    return
                ticket = self._queues[d][0]
                _, t, fp = self._where[ticket]
            try:
                res = (None, self.servers[d].wait(t))
            except Exception as ex:  # the job failed on its device: report it to wait()
                res = (ex, None)
            with self._cv:
                self._queues[d].popleft()
                del self._where[ticket]
                self.used[d] -= fp
                self.running[d] -= 1
                self._results[ticket] = res
                self._cv.notify_all()

    def wait(self, ticket: int, timeout_ms: int = 0) -> float:
        """Latency (ms) of a job, once it completed; re-raises its failure."""
        with self._cv:
            if ticket not in self._results and ticket not in self._where:
                raise KeyError(f"unknown ticket {ticket}")
            ok = self._cv.wait_for(lambda: ticket in self._results,
                                   timeout=None if timeout_ms == 0 else timeout_ms / 1e3)
            if not ok:
                raise TimeoutError(f"job {ticket} still running")
            ex, lat = self._results.pop(ticket)
        if ex is not None:
            raise ex
        return lat

    def counters(self) -> dict:
        with self._cv:
            return {"used": list(self.used), "running": list(self.running), "placed": list(self.placed),
                    "in_flight": len(self._where)}

    def close(self):
        """Finish the jobs in flight, stop the reapers, close the servers."""
        with self._cv:
            self._closing = True
            self._cv.notify_all()
        for t in self._reapers:
            t.join()
        for s in self.servers:
            s.close()
