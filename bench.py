#!/usr/bin/env python3
"""Benchmark of the halo2/BN256 prover hot path on B200.

Workload (one "step"): the halo2 coset LDE on 2^24 Fr values — ifft on the
2^24 domain (x n^-1), multiply coefficient i by 7^i, zero-pad to 2^26 and
NTT on the extended 2^26 domain — seeded uniform Fr inputs, bit-exact
arithmetic.  Metric: Fr NTT Melem/s at 2^24 = 2^24 input elements / step
time.  Inputs (512 MiB) and outputs (2 GiB) exceed the 126 MB L2, so no
flush is needed between steps.

  value  : device-resident pipeline (zkgpu_lagrange_to_extended_dev), CUDA
           events on the launching stream, max over ranks.
  e2e    : the same pipeline through the host-buffer C ABI
           (zkgpu_lagrange_to_extended) from pinned host memory, H2D + D2H
           inside the timed region.
  extras : forward NTT 2^24 Melem/s (device resident).

Multi-GPU: independent replicas, one per rank ("weak" scaling); no
collective on the data path.  `--impl reference` times the reference's CPU
path (the oracle's restatement of halo2 best_fft / ifft / distribute_powers)
on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
MONT_R = 1 << 256
LOG_N, LOG_EXT = 24, 26


# ---------------------------------------------------------------------------
# Fr constants (host arithmetic on Python ints)
# ---------------------------------------------------------------------------
def mont(x: int) -> np.ndarray:
    v = x * MONT_R % R_MOD
    return np.array([(v >> (64 * i)) & (2**64 - 1) for i in range(4)], dtype=np.uint64)


def root_of_unity(log_n: int) -> int:
    w = pow(7, (R_MOD - 1) >> 28, R_MOD)
    for _ in range(28 - log_n):
        w = w * w % R_MOD
    return w


def lde_constants(k: int, e: int):
    w = root_of_unity(k)
    return dict(omega=mont(w), omega_inv=mont(pow(w, -1, R_MOD)), divisor=mont(pow(1 << k, -1, R_MOD)),
                g=mont(7), omega_ext=mont(root_of_unity(k + e)))


def rand_fr(n: int, seed: int) -> np.ndarray:
    """n uniform elements of [0, r) (used directly as Montgomery forms)."""
    rng = np.random.default_rng(seed)
    r_limbs = [(R_MOD >> (64 * i)) & (2**64 - 1) for i in range(4)]
    out = rng.integers(0, 2**64, size=(n, 4), dtype=np.uint64)
    out[:, 3] &= np.uint64((1 << 62) - 1)

    def below_r(a):
        lt = np.zeros(a.shape[0], bool)
        eq = np.ones(a.shape[0], bool)
        for w in (3, 2, 1, 0):
            lt |= eq & (a[:, w] < np.uint64(r_limbs[w]))
            eq &= a[:, w] == np.uint64(r_limbs[w])
        return lt

    bad = ~below_r(out)
    while bad.any():
        repl = rng.integers(0, 2**64, size=(int(bad.sum()), 4), dtype=np.uint64)
        repl[:, 3] &= np.uint64((1 << 62) - 1)
        out[bad] = repl
        bad = ~below_r(out)
    return out


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.stamped: list = []  # (perf_counter, csv line)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            # nvidia-smi's start-up (NVML init) disturbs a running GPU context:
            # let it settle before anything is timed
            deadline = time.perf_counter() + 5.0
            while not self.stamped and time.perf_counter() < deadline:
                time.sleep(0.02)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.stamped.append((time.perf_counter(), line.strip()))

    def window(self, t0: float, t1: float):
        """keep only samples taken inside [t0, t1] (the timed region)"""
        inside = [ln for (t, ln) in self.stamped if t0 <= t <= t1]
        self.lines = inside if inside else [ln for (_, ln) in self.stamped[-3:]]

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference arm: the CPU path on host cores
# ---------------------------------------------------------------------------
def cpu_lde_sample(k: int = 22, e: int = 2, seed: int = 5):
    """halo2 CPU LDE (oracle restatement of best_fft/ifft/distribute_powers) on
    a 2^k -> 2^(k+e) sample; returns (seconds, threads)."""
    from oracle import pyoracle as O
    threads = os.cpu_count() or 1
    c = lde_constants(k, e)
    vals = rand_fr(1 << k, seed)
    t0 = time.perf_counter()
    coeffs = O.ifft(vals, c["omega_inv"], k, c["divisor"], threads)
    O.coeff_to_extended(coeffs, k, k + e, c["g"], c["omega_ext"], threads)
    return time.perf_counter() - t0, threads


def lde_work(k: int, e: int) -> float:
    """algorithmic Fr products of the LDE (radix-2 convention)"""
    return (2**k / 2) * k + 2**k + 2**k + (2 ** (k + e) / 2) * (k + e)


def cpu_melem_s(t_sample: float, k: int = 22, e: int = 2) -> float:
    # scale the sample's time to the full 2^24 -> 2^26 workload by algorithmic work
    t_full = t_sample * lde_work(LOG_N, LOG_EXT - LOG_N) / lde_work(k, e)
    return (2**LOG_N) / t_full / 1e6


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return 0
    ts = []
    threads = 1
    for i in range(args.warmup + args.steps):
        t, threads = cpu_lde_sample()
        if i >= args.warmup:
            ts.append(t)
    t = statistics.median(ts)
    v = cpu_melem_s(t)
    sample = ("halo2 LDE 2^22 -> 2^24 per step (oracle port of best_fft/ifft/distribute_powers, OpenMP), "
              "time scaled to 2^24 -> 2^26 by algorithmic work")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "Melem/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32x8 (Fr Montgomery)", "data": "synthetic",
        "config": CONFIG,
        "cpu_baseline": {"value": round(v, 3), "unit": "Melem/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(v, 3), "unit": "Melem/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


METRIC = "Fr NTT Melem/s @2^24 (halo2 coset LDE 2^24 -> 2^26)"
CONFIG = {"workload": "halo2 coset LDE: ifft 2^24, x7^i, zero-pad, NTT 2^26 (Fr, Montgomery)", "log_n": LOG_N,
          "log_ext": LOG_EXT, "l2_flush": "inputs 512 MiB and outputs 2 GiB exceed L2", "parallelism": "replicas"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import zk_gpu_b200 as zk

    from zk_gpu_b200.replicas import ReplicaGroup

    dev = local_rank
    torch.cuda.set_device(dev)
    # N GPUs = N independent replicas: no data-path collective, only the
    # barrier and the max over ranks of the device-timed step
    group = ReplicaGroup("nccl", device=torch.device("cuda", dev), timeout_s=120)
    barrier, max_over_ranks = group.barrier, group.max

    c = lde_constants(LOG_N, LOG_EXT - LOG_N)
    n, N = 1 << LOG_N, 1 << LOG_EXT
    vals_np = rand_fr(n, 1234 + rank)
    d_vals = torch.from_numpy(vals_np.view(np.int64)).to(f"cuda:{dev}")
    d_ext = torch.empty((N, 4), dtype=torch.int64, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)

    imad_ps, modmul_ps = zk.int_peak(dev)

    # autotuner (untimed): NTT plans for the LDE's two sizes, the MSM window
    # for 2^22, and batched-transform plans for 2^10..2^20
    tune = {"ms": 0.0}
    if args.tune_load:
        tune["loaded"] = zk.tune_load(args.tune_load, device=dev)
    elif not args.no_tune:
        # single transforms 2^21..2^24 (the LDE's 2^24, the serving mix's large
        # NTT / LDE sizes) and 2^26; MSM windows for every size the bench runs
        tune["ms"] += zk.autotune(zk.TUNE_NTT, 21, LOG_N, device=dev)
        tune["ms"] += zk.autotune(zk.TUNE_NTT, LOG_EXT, LOG_EXT, device=dev)
        tune["ms"] += zk.autotune(zk.TUNE_MSM, 14, 22, device=dev)
        tune["ms"] += zk.autotune(zk.TUNE_NTT_BATCHED, 10, 20, device=dev)
    tune["ntt_plans"] = {str(k): zk.get_ntt_plan(k, device=dev) for k in list(range(10, 25)) + [LOG_EXT]}
    tune["msm_windows"] = {str(k): zk.get_msm_window(k, device=dev) for k in range(14, 23)}
    tune["msm_window_2p22"] = zk.get_msm_window(22, device=dev)
    tune["ms"] = round(tune["ms"], 1)
    if args.tune_save:
        zk.tune_save(args.tune_save, device=dev)

    def step():
        zk.lagrange_to_extended_dev(d_vals, d_ext, LOG_N, LOG_EXT, c["omega_inv"], c["divisor"], c["g"],
                                    c["omega_ext"], stream=stream)

    with ClockSampler(dev) as clk:
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 3)):
                step()
        stream.synchronize()

        # ---- timed region: device-resident pipeline ----
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        zk.prof_reset()
        zk.prof_enable(True)
        zk.launch_count(reset=True)
        barrier()
        torch.cuda.synchronize()
        t_begin = time.perf_counter()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        stream.synchronize()
        t_end = time.perf_counter()
    clk.window(t_begin, t_end)
    torch.cuda.synchronize()
    barrier()
    launches = zk.launch_count()
    zk.prof_enable(False)
    prof = zk.prof_read()
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms)
    value = world * n / (ms * 1e-3) / 1e6

    # ---- forward NTT 2^24 (sub-metric) ----
    d_a = d_vals.clone()
    for _ in range(3):
        zk.ntt_dev(d_a, LOG_N, c["omega"], stream=stream)
    stream.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        zk.ntt_dev(d_a, LOG_N, c["omega"], stream=stream)
    e1.record(stream)
    stream.synchronize()
    ntt_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    del d_a

    # ---- MSM 2^22 (sub-metric): 10% of scalars < 2^16, resident bases ----
    n_msm = 1 << 22
    sc = rand_fr(n_msm, 4242 + rank)
    sc[: n_msm // 10] = small_fr(n_msm // 10, 4343 + rank)
    d_sc = torch.from_numpy(sc.view(np.int64)).to(f"cuda:{dev}")
    d_bs = gen_bases(zk, torch, n_msm, 4141 + rank, dev)
    d_out = torch.zeros(12, dtype=torch.int64, device=f"cuda:{dev}")
    zk.msm_dev(d_sc, d_bs, d_out, stream=stream)
    stream.synchronize()
    msm_steps = max(3, min(args.steps, 10))
    zk.prof_reset()
    zk.prof_enable(True)
    e0.record(stream)
    for _ in range(msm_steps):
        zk.msm_dev(d_sc, d_bs, d_out, stream=stream)
    e1.record(stream)
    stream.synchronize()
    zk.prof_enable(False)
    msm_prof = zk.prof_read()
    msm_ms = max_over_ranks(e0.elapsed_time(e1) / msm_steps)
    del d_sc, d_bs

    batched = bench_batched(zk, torch, dev, stream, args.steps)
    serving = bench_serving(zk, torch, dev) if not args.no_serving else None

    # ---- e2e through the host-buffer C ABI, pinned host memory ----
    h_vals = torch.from_numpy(vals_np.view(np.int64)).pin_memory()
    h_ext = torch.empty((N, 4), dtype=torch.int64).pin_memory()
    hv = h_vals.numpy().view(np.uint64)
    he = h_ext.numpy().view(np.uint64)

    def e2e_step():
        rc = zk.lib().zkgpu_lagrange_to_extended(dev, hv.ctypes.data, LOG_N, he.ctypes.data, LOG_EXT,
                                                 c["omega_inv"].ctypes.data, c["divisor"].ctypes.data,
                                                 c["g"].ctypes.data, c["omega_ext"].ctypes.data)
        if rc != 0:
            raise RuntimeError(f"zkgpu_lagrange_to_extended failed: {rc}")

    e2e_step()
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(2, min(args.steps, 10))
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps)
    e2e_value = world * n / e2e_s / 1e6

    # ---- roofline of the dominant kernel ----
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"]) if prof else None
    roof = None
    if dom:
        name, d = dom
        achieved_imad = d["work"] * 256 / (d["ms"] * 1e-3)          # 256 IMAD issues per Fr product
        per_launch_bytes = d["bytes"] / d["launches"]
        roof = {"bound": "imad", "kernel": name, "achieved": round(achieved_imad / 1e12, 3),
                "peak": round(imad_ps / 1e12, 3), "unit": "TIMAD/s",
                "frac": round(achieved_imad / imad_ps, 4), "traffic": (round(TRAFFIC_RATIO[name] * per_launch_bytes) if name in TRAFFIC_RATIO else None),
                "traffic_source": TRAFFIC_SOURCE.get(name),
                "algorithmic_bytes_per_launch": per_launch_bytes,
                "hbm_gbs": round(d["bytes"] / (d["ms"] * 1e-3) / 1e9, 1),
                "hbm_frac_of_measured": round(d["bytes"] / (d["ms"] * 1e-3) / 1e9 / HBM_GBS, 4),
                "kernel_ms_per_launch": round(d["ms"] / d["launches"], 4),
                "peak_source": "measured live: zkgpu_int_peak (mad.lo.cc/madc.hi.cc chains, all SMs)",
                "modmul_rate_measured_gps": round(modmul_ps / 1e9, 2)}

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Melem/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32x8 (Fr Montgomery, integer)", "data": "synthetic (seeded uniform Fr)",
        "config": CONFIG, "clocks": clk.summary(), "gpu_launches": int(launches),
        "e2e": {"value": round(e2e_value, 3), "unit": "Melem/s", "h2d_bytes_per_step": n * 32,
                "d2h_bytes_per_step": N * 32, "api": "zkgpu_lagrange_to_extended (host buffers, pinned)"},
        "roofline": roof,
        "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 3)} for k, v in prof.items()},
        "extra": {"ntt_fwd_2p24_melem_s": round(world * n / (ntt_ms * 1e-3) / 1e6, 2),
                  "ntt_fwd_2p24_ms": round(ntt_ms, 4),
                  "msm_2p22_mpts_s": round(world * n_msm / (msm_ms * 1e-3) / 1e6, 2),
                  "msm_2p22_ms": round(msm_ms, 3),
                  "msm_inputs": "bases k_i*(1,2) for seeded uniform Fr k_i (device fixed-base multiplication); "
                                "scalars uniform Fr, 10% replaced by uniform < 2^16",
                  "msm_kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 3)} for k, v in msm_prof.items()},
                  "msm_roofline": msm_roofline(msm_prof, imad_ps, n_msm, msm_ms),
                  "batched_ntt": batched,
                  "autotune": tune,
                  "serving": serving},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t, threads = cpu_lde_sample()
        line["cpu_baseline"] = {"value": round(cpu_melem_s(t), 3), "unit": "Melem/s", "cores": threads,
                                "kind": "port",
                                "sample": "halo2 LDE 2^22 -> 2^24 once (oracle port, OpenMP on all host threads), "
                                          "time scaled to 2^24 -> 2^26 by algorithmic work"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    group.barrier()
    group.close()
    return 0


def bench_batched(zk, torch, dev: int, stream, steps: int, njobs: int = 512, seed: int = 77):
    """512 NTT jobs, log2 size uniform in {10..20}, random forward/inverse and
    coset flag: one persistent graph launch per run vs one call per job."""
    rng = np.random.default_rng(seed)
    sizes = [int(k) for k in rng.integers(10, 21, njobs)]
    gen = torch.Generator(device=f"cuda:{dev}")
    gen.manual_seed(seed)
    consts = {}
    jobs = []
    for k in sizes:
        if k not in consts:
            w = root_of_unity(k)
            consts[k] = (mont(w), mont(pow(w, -1, R_MOD)), mont(pow(1 << k, -1, R_MOD)),
                         mont(7 * root_of_unity(k + 2) % R_MOD))
        w, wi, ninv, c = consts[k]
        # uniform 252-bit values (< r), generated on the device
        t = torch.randint(0, 2**62, (1 << k, 4), dtype=torch.int64, device=f"cuda:{dev}", generator=gen)
        t[:, 3] &= (1 << 60) - 1
        inverse, coset = bool(rng.integers(0, 2)), bool(rng.integers(0, 2))
        j = {"tensor": t, "log_n": k, "omega": wi if inverse else w}
        if inverse:
            j["scale"] = ninv
        if coset:
            j["coset"] = c
        jobs.append(j)
    elems = sum(1 << k for k in sizes)
    batch = zk.NttBatch(jobs, device=dev)
    for _ in range(2):
        batch.run(stream)
    stream.synchronize()
    batch.check()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    runs = max(3, min(steps, 10))
    zk.launch_count(reset=True)
    e0.record(stream)
    for _ in range(runs):
        batch.run(stream)
    e1.record(stream)
    stream.synchronize()
    batch_launches = zk.launch_count() / runs
    batch.check()
    batch_ms = e0.elapsed_time(e1) / runs

    def one_call_per_job():
        for j in jobs:
            zk.ntt_dev(j["tensor"], j["log_n"], j["omega"], coset=j.get("coset"), post_scale=j.get("scale"),
                       stream=stream)

    one_call_per_job()
    stream.synchronize()
    zk.launch_count(reset=True)
    e0.record(stream)
    for _ in range(runs):
        one_call_per_job()
    e1.record(stream)
    stream.synchronize()
    single_launches = zk.launch_count() / runs
    single_ms = e0.elapsed_time(e1) / runs
    info = batch.info()
    batch.close()
    return {"jobs": njobs, "elements": elems, "batched_ms": round(batch_ms, 3),
            "batched_jobs_s": round(njobs / (batch_ms * 1e-3), 1),
            "batched_melem_s": round(elems / (batch_ms * 1e-3) / 1e6, 1),
            "one_call_per_job_ms": round(single_ms, 3),
            "one_call_per_job_jobs_s": round(njobs / (single_ms * 1e-3), 1),
            "speedup": round(single_ms / batch_ms, 3),
            "launches_per_run": {"batched": batch_launches, "one_call_per_job": single_launches},
            "work_items": info["tiles"], "passes": info["passes"], "grid": info["grid"],
            "inputs": "uniform 252-bit values (< r) from torch.randint on the device"}


def serving_trace(njobs: int, rate: float, seed: int = 99):
    """(arrival_s, kind, log_size) per job: Poisson arrivals; 70% NTT / coset
    LDE (log2 size uniform 12..22, half each), 30% MSM (log2 points 14..20)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, njobs))
    out = []
    for i in range(njobs):
        u = rng.random()
        if u < 0.35:
            out.append((float(t[i]), "ntt", int(rng.integers(12, 23))))
        elif u < 0.70:
            out.append((float(t[i]), "lde", int(rng.integers(12, 23))))
        else:
            out.append((float(t[i]), "msm", int(rng.integers(14, 21))))
    return out


def bench_serving(zk, torch, dev: int, njobs: int = 1000, rate: float = 2000.0, wave_jobs: int = 64):
    """Serving loop (continuous batching) vs one call per job on the same GPU,
    same arrival trace; host buffers pinned, shared per size class (read-only
    inputs; outputs of identical jobs are identical)."""
    import ctypes
    trace = serving_trace(njobs, rate)
    pools = {}

    def pinned(rows, cols):
        t = torch.empty((rows, cols), dtype=torch.int64).pin_memory()
        return t, t.numpy().view(np.uint64)

    consts = {}
    for k in range(12, 25):
        w = root_of_unity(k)
        consts[k] = dict(omega=mont(w), omega_inv=mont(pow(w, -1, R_MOD)), divisor=mont(pow(1 << k, -1, R_MOD)))
    g7 = mont(7)
    for _, kind, k in trace:
        key = (kind, k)
        if key in pools:
            continue
        if kind == "msm":
            ti, a = pinned(1 << k, 4)
            a[:] = rand_fr(1 << k, k)
            to, o = pinned(1, 12)
        else:
            ti, a = pinned(1 << k, 4)
            a[:] = rand_fr(1 << k, 1000 + k)
            to, o = pinned(1 << (k + 2 if kind == "lde" else k), 4)
        pools[key] = (ti, a, to, o)
    nb = 1 << 20
    bases = gen_bases(zk, torch, nb, 4545, dev).cpu().numpy().view(np.uint64)

    def make_job(kind, k):
        ti, a, to, o = pools[(kind, k)]
        if kind == "ntt":
            return zk.ntt_job(a, o, k, consts[k]["omega"])
        if kind == "lde":
            return zk.lde_job(a, o, k, k + 2, consts[k]["omega_inv"], consts[k]["divisor"], g7,
                              consts[k + 2]["omega"])
        return zk.msm_job(a, o, 1 << k, bid)

    def pct(x, q):
        return float(np.percentile(np.asarray(x), q)) if len(x) else None

    # ---- serving loop ----
    srv = zk.Server(device=dev, hbm_budget=150 * 10**9, max_wave_jobs=wave_jobs)
    bid = srv.add_bases(bases)

    def run_server(open_loop: bool):
        lats = [None] * len(trace)
        tickets = [None] * len(trace)
        done_evt = threading.Event()

        def waiter():
            for i in range(len(trace)):
                while tickets[i] is None:
                    time.sleep(0.0002)
                lats[i] = srv.wait(tickets[i]) / 1e3
            done_evt.set()

        th = threading.Thread(target=waiter)
        th.start()
        t0 = time.perf_counter()
        jobs_keep = []
        for i, (at, kind, k) in enumerate(trace):
            if open_loop:
                d = t0 + at - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            j = make_job(kind, k)
            jobs_keep.append(j)
            tickets[i] = srv.submit(j)
        done_evt.wait()
        th.join()
        span = time.perf_counter() - t0
        return lats, span

    run_server(False)  # warm-up: tables, pools, allocator
    lat_s, span_s = run_server(True)
    lat_sc, span_sc = run_server(False)
    st = srv.stats()
    # ---- one call per job (synchronous, one job at a time, same residency) ----
    stream = torch.cuda.Stream(device=dev)
    d_bases = torch.from_numpy(bases.view(np.int64)).to(f"cuda:{dev}")
    d_out = torch.zeros(12, dtype=torch.int64, device=f"cuda:{dev}")

    def one_call(kind, k):
        ti, a, to, o = pools[(kind, k)]
        with torch.cuda.stream(stream):
            if kind == "ntt":
                d = ti.to(f"cuda:{dev}", non_blocking=True)
                zk.ntt_dev(d, k, consts[k]["omega"], stream=stream)
                to.copy_(d, non_blocking=True)
            elif kind == "lde":
                d = ti.to(f"cuda:{dev}", non_blocking=True)
                e = torch.empty((1 << (k + 2), 4), dtype=torch.int64, device=f"cuda:{dev}")
                zk.lagrange_to_extended_dev(d, e, k, k + 2, consts[k]["omega_inv"], consts[k]["divisor"], g7,
                                            consts[k + 2]["omega"], stream=stream)
                to.copy_(e, non_blocking=True)
            else:
                d = ti.to(f"cuda:{dev}", non_blocking=True)
                zk.msm_dev(d, d_bases[: 1 << k], d_out, stream=stream)
                to.copy_(d_out.view(1, 12), non_blocking=True)
        stream.synchronize()

    def run_plain(open_loop: bool):
        lats = []
        t0 = time.perf_counter()
        for at, kind, k in trace:
            if open_loop:
                d = t0 + at - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            arrive = t0 + at if open_loop else t0
            one_call(kind, k)
            lats.append(time.perf_counter() - arrive)
        return lats, time.perf_counter() - t0

    for kind, k in pools:
        one_call(kind, k)
    lat_p, span_p = run_plain(True)
    lat_pc, span_pc = run_plain(False)
    srv.close()

    # device time of each job alone (inputs resident, no copies; best of 3),
    # summed over the trace: the compute floor of any schedule on one GPU
    dev_ms = {}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for kind, k in pools:
        ti, a, to, o = pools[(kind, k)]
        d = ti.to(f"cuda:{dev}")
        e = torch.empty((1 << (k + 2), 4), dtype=torch.int64, device=f"cuda:{dev}") if kind == "lde" else None
        best = 1e30
        for _ in range(4):
            ev0.record(stream)
            if kind == "ntt":
                zk.ntt_dev(d, k, consts[k]["omega"], stream=stream)
            elif kind == "lde":
                zk.lagrange_to_extended_dev(d, e, k, k + 2, consts[k]["omega_inv"], consts[k]["divisor"], g7,
                                            consts[k + 2]["omega"], stream=stream)
            else:
                zk.msm_dev(d, d_bases[: 1 << k], d_out, stream=stream)
            ev1.record(stream)
            stream.synchronize()
            best = min(best, ev0.elapsed_time(ev1))
        dev_ms[(kind, k)] = best
        del d, e
    trace_dev_s = sum(dev_ms[(kind, k)] for _, kind, k in trace) / 1e3
    by_kind = {kd: round(sum(dev_ms[(kind, k)] for _, kind, k in trace if kind == kd) / 1e3, 3)
               for kd in ("ntt", "lde", "msm")}
    n = len(trace)
    # host<->device bytes the trace moves, against the pinned-copy bandwidth
    # of this box measured the same way (1 GiB, CUDA events)
    h2d = sum((1 << k) * 32 for _, kind, k in trace)
    d2h = sum(96 if kind == "msm" else (1 << (k + 2 if kind == "lde" else k)) * 32 for _, kind, k in trace)
    pcie = pcie_bandwidth(torch, dev)
    pcie.update({"trace_h2d_gb": round(h2d / 1e9, 2), "trace_d2h_gb": round(d2h / 1e9, 2),
                 "batched_closed_loop_d2h_gbs": round(d2h / span_sc / 1e9, 2),
                 "batched_closed_loop_h2d_gbs": round(h2d / span_sc / 1e9, 2),
                 "one_call_closed_loop_d2h_gbs": round(d2h / span_pc / 1e9, 2)})
    return {
        "jobs": n, "offered_rate_jobs_s": rate, "mix": "35% NTT 2^12-2^22, 35% coset LDE x4 2^12-2^22, "
                                                         "30% MSM 2^14-2^20 (resident bases)",
        "open_loop": {
            "batched": {"jobs_s": round(n / span_s, 1), "p50_ms": round(pct(lat_s, 50) * 1e3, 3),
                        "p99_ms": round(pct(lat_s, 99) * 1e3, 3)},
            "one_call_per_job": {"jobs_s": round(n / span_p, 1), "p50_ms": round(pct(lat_p, 50) * 1e3, 3),
                                 "p99_ms": round(pct(lat_p, 99) * 1e3, 3)}},
        "closed_loop_saturation": {
            "batched_jobs_s": round(n / span_sc, 1), "one_call_per_job_jobs_s": round(n / span_pc, 1),
            "speedup": round(span_pc / span_sc, 3),
            "batched_p99_ms": round(pct(lat_sc, 99) * 1e3, 3), "one_call_p99_ms": round(pct(lat_pc, 99) * 1e3, 3)},
        "server": {"waves": st["waves"], "batch_launches": st["batch_launches"], "hbm_peak_gb":
                   round(st["hbm_peak"] / 1e9, 2), "rejected": st["rejected"], "failed": st["failed"]},
        "pcie": pcie,
        "device_floor": {"trace_device_s": round(trace_dev_s, 3), "by_kind_s": by_kind,
                         "jobs_s_at_floor": round(n / trace_dev_s, 1),
                         "batched_closed_loop_frac_of_floor": round(trace_dev_s / span_sc, 3)},
    }


def pcie_bandwidth(torch, dev: int, nbytes: int = 1 << 30) -> dict:
    """Pinned host<->device copy bandwidth: H2D alone, D2H alone, and both at
    once on two streams (GB/s, best of 3, CUDA events)."""
    h_in = torch.empty(nbytes // 8, dtype=torch.int64).pin_memory()
    h_out = torch.empty(nbytes // 8, dtype=torch.int64).pin_memory()
    d_a = torch.empty(nbytes // 8, dtype=torch.int64, device=f"cuda:{dev}")
    d_b = torch.zeros(nbytes // 8, dtype=torch.int64, device=f"cuda:{dev}")
    s1, s2 = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)

    def timed(fn) -> float:
        best = 1e30
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
        return best

    def h2d():
        with torch.cuda.stream(s1):
            d_a.copy_(h_in, non_blocking=True)

    def d2h():
        with torch.cuda.stream(s2):
            h_out.copy_(d_b, non_blocking=True)

    def both():
        h2d()
        d2h()

    t_h, t_d, t_b = timed(h2d), timed(d2h), timed(both)
    del d_a, d_b
    return {"pinned_h2d_gbs": round(nbytes / t_h / 1e9, 1), "pinned_d2h_gbs": round(nbytes / t_d / 1e9, 1),
            "pinned_duplex_gbs": round(2 * nbytes / t_b / 1e9, 1)}


def small_fr(n: int, seed: int, bits: int = 16) -> np.ndarray:
    """n uniform canonical values < 2^bits, in Montgomery form"""
    rng = np.random.default_rng(seed)
    vals = rng.integers(0, 1 << bits, size=n, dtype=np.uint64)
    out = np.empty((n, 4), np.uint64)
    m = 2**64 - 1
    for i, v in enumerate(vals.tolist()):
        x = v * MONT_R % R_MOD
        out[i] = [(x >> (64 * j)) & m for j in range(4)]
    return out


def msm_roofline(prof: dict, imad_ps: float, n: int, total_ms: float):
    """Whole-MSM roofline: fixed work convention 16 windows x 1 bucket add per
    point x 6 Fq products (batch-affine cost) x 256 IMAD per product."""
    work = n * 16 * 6
    achieved = work * 256 / (total_ms * 1e-3)
    out = {"bound": "imad", "achieved": round(achieved / 1e12, 3), "peak": round(imad_ps / 1e12, 3),
           "unit": "TIMAD/s", "frac": round(achieved / imad_ps, 4), "work_fq_products": work}
    b = prof.get("msm_bucket")
    if b:
        out["bucket_kernel_ms_per_launch"] = round(b["ms"] / b["launches"], 3)
        out["bucket_kernel_share"] = round(b["ms"] / sum(v["ms"] for v in prof.values()), 3)
    return out


HBM_GBS = 6543.1
# DRAM bytes (read + write) per launch over algorithmic bytes, from one ncu
# capture of the same kernel on a smaller case (traffic grows with the
# elements processed): ntt_pass_kernel<6> on a 2^24 transform, plan 6+6+6+6,
# launches 1.583 / 1.611 GB and 1.034 / 1.082 GB.
TRAFFIC_RATIO = {"ntt_pass_b6": 0.97}
TRAFFIC_SOURCE = {"ntt_pass_b6": "ncu dram__bytes_read.sum + dram__bytes_write.sum of ntt_pass_kernel<6> on a "
                                 "2^24 transform (plan 6+6+6+6), scaled by algorithmic bytes"}


def _load_peaks():
    global HBM_GBS
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            HBM_GBS = float(json.load(open(p))["hbm_gbs"])
        except Exception:
            pass


def run_case(args):
    """Small single-kernel-family cases for profiler captures (inputs larger
    than L2, a few hundred MB on the device): `ntt22` = forward NTT of 2^22,
    `lde20` = LDE 2^20 -> 2^22, `msm20` = MSM of 2^20 points."""
    import torch
    import zk_gpu_b200 as zk
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.case in ("ntt22", "lde20", "ntt24"):
        k = {"ntt22": 22, "lde20": 20, "ntt24": 24}[args.case]
        if args.plan:  # pass widths for the transform of this case (the extended one for lde20)
            zk.set_ntt_plan(k + 2 if args.case == "lde20" else k, [int(b) for b in args.plan.split(",")])
        c = lde_constants(k, 2)
        d = torch.from_numpy(rand_fr(1 << k, 7).view(np.int64)).cuda()
        ext = torch.empty(((1 << (k + 2)), 4), dtype=torch.int64, device="cuda") if args.case == "lde20" else None

        def step():
            if ext is None:
                zk.ntt_dev(d, k, c["omega"], stream=stream)
            else:
                zk.lagrange_to_extended_dev(d, ext, k, k + 2, c["omega_inv"], c["divisor"], c["g"],
                                            c["omega_ext"], stream=stream)
    elif args.case == "msm20":
        n = 1 << 20
        s = torch.from_numpy(rand_fr(n, 8).view(np.int64)).cuda()
        b = gen_bases(zk, torch, n, 4141, 0)
        out = torch.zeros(12, dtype=torch.int64, device="cuda")

        def step():
            zk.msm_dev(s, b, out, stream=stream)
    step()
    stream.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    stream.synchronize()
    print(json.dumps({"case": args.case, "steps": args.steps, "status": "ok",
                      "ms_per_step": round(e0.elapsed_time(e1) / args.steps, 4)}))
    return 0


def gen_bases(zk, torch, n: int, seed: int, dev: int):
    """n affine G1 bases k_i * (1, 2) for seeded uniform Fr k_i, generated on
    the device by the library's fixed-base multiplication (device tensor)."""
    k = torch.from_numpy(rand_fr(n, seed).view(np.int64)).to(f"cuda:{dev}")
    out = torch.empty((n, 8), dtype=torch.int64, device=f"cuda:{dev}")
    zk.g1_mul_fixed_dev(k, out)
    del k
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-loop sub-benchmark")
    ap.add_argument("--no-tune", action="store_true", help="use the built-in NTT plans and MSM windows")
    ap.add_argument("--case", choices=["ntt22", "ntt24", "lde20", "msm20"], default=None,
                    help="run a small profiling case instead of the benchmark")
    ap.add_argument("--plan", default=None, help="with --case: NTT pass widths, e.g. 6,6,6,6")
    ap.add_argument("--tune-save", default=None, help="write the autotuner's choices to this file")
    ap.add_argument("--tune-load", default=None, help="load autotuner choices from this file instead of tuning")
    args = ap.parse_args()
    _load_peaks()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
