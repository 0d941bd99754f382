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
    """One serving loop (zk.Server) per local GPU, jobs placed by place_job.
    Bases added here are made resident on every device."""

    def __init__(self, devices: list, hbm_budget: int = 150 * 10**9, max_wave_jobs: int = 4096):
        from . import Server
        self.devices = list(devices)
        self.servers = [Server(d, hbm_budget, max_wave_jobs) for d in self.devices]
        self.capacity = [hbm_budget] * len(self.devices)
        self.used = [0] * len(self.devices)
        self.running = [0] * len(self.devices)
        self._where = {}
        self._next = 0

    def add_bases(self, bases) -> int:
        ids = {s.add_bases(bases) for s in self.servers}
        assert len(ids) == 1, "base ids diverged across devices"
        return ids.pop()

    def submit(self, job, keep=None) -> int:
        """Returns a ticket; raises RuntimeError when no device has room
        (the caller waits for a completion and retries)."""
        from . import job_footprint
        fp = job_footprint(job)
        d = place_job(fp, self.running, self.used, self.capacity)
        if d < 0:
            raise RuntimeError("no device has room for this job now")
        t = self.servers[d].submit(job, keep)
        self.used[d] += fp
        self.running[d] += 1
        ticket = self._next
        self._next += 1
        self._where[ticket] = (d, t, fp)
        return ticket

    def wait(self, ticket: int, timeout_ms: int = 0) -> float:
        d, t, fp = self._where.pop(ticket)
        try:
            return self.servers[d].wait(t, timeout_ms)
        finally:
            self.used[d] -= fp
            self.running[d] -= 1

    def close(self):
        for s in self.servers:
            s.close()
