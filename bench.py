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
def cpu_lde_sample(k: int = LOG_N, e: int = LOG_EXT - LOG_N, seed: int = 5):
    """halo2 CPU LDE (oracle restatement of best_fft/ifft/distribute_powers) on
    a 2^k -> 2^(k+e) input, the full benchmark size by default; returns
    (seconds, threads)."""
    from oracle import pyoracle as O
    threads = os.cpu_count() or 1
    c = lde_constants(k, e)
    vals = rand_fr(1 << k, seed)
    t0 = time.perf_counter()
    coeffs = O.ifft(vals, c["omega_inv"], k, c["divisor"], threads)
    O.coeff_to_extended(coeffs, k, k + e, c["g"], c["omega_ext"], threads)
    return time.perf_counter() - t0, threads


def cpu_ntt16_ms(calls: int = 20) -> tuple:
    """The single forward NTT 2^16 on the host (oracle restatement of halo2
    best_fft, OpenMP on all host threads): median ms of `calls` calls."""
    from oracle import pyoracle as O
    threads = os.cpu_count() or 1
    a = rand_fr(1 << 16, 1616)
    w = mont(root_of_unity(16))
    ts = []
    for _ in range(calls):
        t0 = time.perf_counter()
        O.best_fft(a, w, 16, threads)
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts)) * 1e3, threads


def lde_work(k: int, e: int) -> float:
    """algorithmic Fr products of the LDE (radix-2 convention)"""
    return (2**k / 2) * k + 2**k + 2**k + (2 ** (k + e) / 2) * (k + e)


def cpu_melem_s(t_sample: float, k: int = LOG_N, e: int = LOG_EXT - LOG_N) -> float:
    # a smaller sample's time scales to the full 2^24 -> 2^26 workload by
    # algorithmic work (the default sample is the full workload: factor 1)
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
    sample = ("one full halo2 LDE 2^24 -> 2^26 per step (oracle port of best_fft/ifft/distribute_powers, "
              "OpenMP on all host threads)")
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
    torch.cuda.synchronize()

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
    torch.cuda.synchronize()
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
    ntt16 = bench_ntt16(zk, torch, dev, stream)

    # ---- MSM 2^22 (sub-metric): 10% of scalars < 2^16, resident bases ----
    n_msm = 1 << 22
    sc = rand_fr(n_msm, 4242 + rank)
    sc[: n_msm // 10] = small_fr(n_msm // 10, 4343 + rank)
    d_sc = torch.from_numpy(sc.view(np.int64)).to(f"cuda:{dev}")
    d_bs = gen_bases(zk, torch, n_msm, 4141 + rank, dev)
    d_out = torch.zeros(12, dtype=torch.int64, device=f"cuda:{dev}")
    torch.cuda.synchronize()
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

    # ---- e2e through the host-buffer C ABI ----
    e2e = bench_e2e(zk, torch, dev, vals_np, c, n, N, args.steps, barrier, max_over_ranks, world)

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
        if name in PIPE_FRACS:
            roof["pipes"] = PIPE_FRACS[name]

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Melem/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32x8 (Fr Montgomery, integer)", "data": "synthetic (seeded uniform Fr)",
        "config": CONFIG, "clocks": clk.summary(), "gpu_launches": int(launches),
        "e2e": e2e,
        "roofline": roof,
        "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 3)} for k, v in prof.items()},
        "extra": {"ntt_fwd_2p24_melem_s": round(world * n / (ntt_ms * 1e-3) / 1e6, 2),
                  "ntt_fwd_2p24_ms": round(ntt_ms, 4),
                  "ntt_fwd_2p16": ntt16,
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
        t16, _ = cpu_ntt16_ms()
        line["cpu_baseline"] = {"value": round(cpu_melem_s(t), 3), "unit": "Melem/s", "cores": threads,
                                "kind": "port",
                                "sample": "one full halo2 LDE 2^24 -> 2^26 (oracle port, OpenMP on all host threads)",
                                "ntt_fwd_2p16_ms": round(t16, 3)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    group.barrier()
    group.close()
    return 0


def bench_e2e(zk, torch, dev: int, vals_np, c, n: int, N: int, steps: int, barrier, max_over_ranks, world: int,
              callers: int = 3):
    """The LDE through the public host-buffer call zkgpu_lagrange_to_extended:
    every step copies its 2^24 inputs host->device and its 2^26 outputs
    device->host inside the call.

    One synchronous call cannot overlap its own copies with its compute (the
    ifft's first pass needs every input, the extended NTT's last pass
    completes every output at once), so the copies of one call overlap only
    the work of other calls.  The reference's callers are concurrent
    (THREAD_POOL workers, src/threadpool.rs:50-69); here `callers` host
    threads each run steps back to back on their own pinned buffers (each
    thread gets its own stream inside the library) and the value is all their
    steps over the wall time.  The single-caller figure and the same call on
    pageable (unpinned) host buffers are reported beside it."""
    import threading as th

    def call(hv, he):
        rc = zk.lib().zkgpu_lagrange_to_extended(dev, hv.ctypes.data, LOG_N, he.ctypes.data, LOG_EXT,
                                                 c["omega_inv"].ctypes.data, c["divisor"].ctypes.data,
                                                 c["g"].ctypes.data, c["omega_ext"].ctypes.data)
        if rc != 0:
            raise RuntimeError(f"zkgpu_lagrange_to_extended failed: {rc}")

    bufs = []
    for i in range(callers):
        h_vals = torch.from_numpy(vals_np.view(np.int64)).pin_memory()
        h_ext = torch.empty((N, 4), dtype=torch.int64).pin_memory()
        bufs.append((h_vals, h_ext, h_vals.numpy().view(np.uint64), h_ext.numpy().view(np.uint64)))
    steps_each = max(2, min(steps, 8))

    def timed(fn_list) -> float:
        errs = []

        def run(fn):
            try:
                fn()
            except Exception as ex:  # surfaced below
                errs.append(ex)
        for fn in fn_list:  # warm-up: tables, pools, first touch of the buffers
            fn()
        barrier()
        t0 = time.perf_counter()
        ts = [th.Thread(target=run, args=(fn,)) for fn in fn_list]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        dt = time.perf_counter() - t0
        if errs:
            raise errs[0]
        return max_over_ranks(dt)

    def loop(hv, he, k):
        return lambda: [call(hv, he) for _ in range(k)]

    # single caller, pinned
    t_one = timed([loop(bufs[0][2], bufs[0][3], steps_each)])
    one_value = world * n * steps_each / t_one / 1e6
    # concurrent callers, pinned
    t_many = timed([loop(b[2], b[3], steps_each) for b in bufs])
    many_value = world * n * steps_each * callers / t_many / 1e6
    # single caller, pageable host memory (a plain numpy array, as a Rust Vec)
    pg_steps = max(2, steps_each // 2)
    pv = np.array(vals_np, copy=True)
    pe = np.empty((N, 4), np.uint64)
    t_pg = timed([loop(pv, pe, pg_steps)])
    pg_value = world * n * pg_steps / t_pg / 1e6
    # outputs of the concurrent callers and of the pageable call equal the single caller's
    ok = all(np.array_equal(b[3], bufs[0][3]) for b in bufs[1:]) and np.array_equal(pe, bufs[0][3])
    del bufs
    if not ok:
        raise RuntimeError("e2e: outputs of concurrent / pageable calls differ")
    return {"value": round(many_value, 3), "unit": "Melem/s", "h2d_bytes_per_step": n * 32,
            "d2h_bytes_per_step": N * 32,
            "api": "zkgpu_lagrange_to_extended (host buffers, pinned), %d concurrent callers" % callers,
            "callers": callers, "steps_per_caller": steps_each,
            "single_caller": {"value": round(one_value, 3), "ms_per_step": round(t_one / steps_each * 1e3, 2)},
            "pageable_single_caller": {"value": round(pg_value, 3), "ms_per_step": round(t_pg / pg_steps * 1e3, 2)},
            "outputs_agree": bool(ok)}


def bench_ntt16(zk, torch, dev: int, stream, reps: int = 200, calls: int = 50):
    """The single forward NTT of 2^16 elements (seeded uniform Fr): device
    time per call over back-to-back calls (input and tables stay in L2: 2 MiB
    of data), and the end-to-end time of the reference's own entry point
    `parallel_fft_api` on a pageable host array (copies in and out inside),
    median of `calls` calls, checked against the device call's output."""
    k, n = 16, 1 << 16
    omega = mont(root_of_unity(k))
    a = rand_fr(n, 1616)
    d = torch.from_numpy(a.view(np.int64)).to(f"cuda:{dev}")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    for _ in range(3):
        zk.ntt_dev(d, k, omega, stream=stream)
    stream.synchronize()
    e0.record(stream)
    for _ in range(reps):
        zk.ntt_dev(d, k, omega, stream=stream)
    e1.record(stream)
    stream.synchronize()
    dev_ms = e0.elapsed_time(e1) / reps
    ref = torch.from_numpy(a.view(np.int64)).to(f"cuda:{dev}")
    zk.ntt_dev(ref, k, omega, stream=stream)
    stream.synchronize()
    ref = ref.cpu().numpy().view(np.uint64)
    times, ok = [], True
    for i in range(calls + 3):
        buf = a.copy()
        t0 = time.perf_counter()
        st = zk.parallel_fft_api(dev, buf, omega, None, n, k, 0)
        dt = time.perf_counter() - t0
        ok = ok and st == 0 and np.array_equal(buf, ref)
        if i >= 3:
            times.append(dt)
    host_ms = float(np.median(times)) * 1e3
    return {"device_ms": round(dev_ms, 4), "device_melem_s": round(n / (dev_ms * 1e-3) / 1e6, 1),
            "parallel_fft_api_ms": round(host_ms, 4), "parallel_fft_api_melem_s": round(n / (host_ms * 1e-3) / 1e6, 1),
            "host_buffer": "pageable numpy array, in place (the reference's callers pass a Vec)",
            "outputs_agree": bool(ok)}


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
    orig = [j["tensor"].clone() for j in jobs]
    torch.cuda.synchronize()  # inputs are made on torch's stream; the runs below use `stream`
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
    # verification: every batched output against the one-call-per-job output
    # of the same job on the same (restored) seeded input, compared on the GPU
    torch.cuda.synchronize()
    for j, o in zip(jobs, orig):
        j["tensor"].copy_(o)
    torch.cuda.synchronize()
    batch.run(stream)
    stream.synchronize()
    batch.check()
    got = [j["tensor"].clone() for j in jobs]
    for j, o in zip(jobs, orig):
        j["tensor"].copy_(o)
    torch.cuda.synchronize()
    one_call_per_job()
    stream.synchronize()
    torch.cuda.synchronize()
    verified = sum(bool(torch.equal(g, j["tensor"])) for g, j in zip(got, jobs))
    del got
    info = batch.info()
    batch.close()
    if verified != njobs:
        raise RuntimeError(f"batched NTT: {njobs - verified} of {njobs} jobs differ from one call per job")
    return {"jobs": njobs, "elements": elems, "batched_ms": round(batch_ms, 3),
            "verified": f"{verified}/{njobs} equal to one call per job",
            "batched_jobs_s": round(njobs / (batch_ms * 1e-3), 1),
            "batched_melem_s": round(elems / (batch_ms * 1e-3) / 1e6, 1),
            "one_call_per_job_ms": round(single_ms, 3),
            "one_call_per_job_jobs_s": round(njobs / (single_ms * 1e-3), 1),
            "speedup": round(single_ms / batch_ms, 3),
            "launches_per_run": {"batched": batch_launches, "one_call_per_job": single_launches},
            "work_items": info["tiles"], "passes": info["passes"], "grid": info["grid"],
            "inputs": "uniform 252-bit values (< r) from torch.randint on the device"}


def median_closed_run(run, njobs: int, reps: int = 3):
    """Run a closed loop `reps` times (`run(None)` -> (latencies, span_s));
    return the median run by span and every run's rate in jobs/s, fastest
    first."""
    runs = sorted((run(None) for _ in range(reps)), key=lambda r: r[1])
    return runs[len(runs) // 2], [round(njobs / r[1], 1) for r in runs]


def serving_trace(njobs: int, seed: int = 99):
    """(arrival at rate 1, kind, log_size) per job: Poisson arrivals
    (divide the times by the offered rate); 70% NTT / coset LDE (log2 size
    uniform 12..22, half each), 30% MSM (log2 points 14..20)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0, njobs))
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


def bench_serving(zk, torch, dev: int, njobs: int = 1000, rate: float = 2000.0, wave_jobs: int = 64,
                  hbm_budget: int = 150 * 10**9):
    """Serving loop (continuous batching) vs one call per job on the same GPU,
    same arrival trace.

    Inputs: every job reads its own seeded window of a pinned pool of 2^24
    uniform Fr elements (job i: a seeded offset), so no two jobs share an
    input.  Outputs of the timed runs go to per-size rings of pinned buffers;
    a separate verification pass runs every job of the trace through the
    server, in waves, into buffers of its own and compares it with the same
    job run alone (one call).  Rates: the configured Poisson 2000 jobs/s
    (open loop), a closed loop (all jobs at once: saturation throughput), and
    an open-loop sweep that finds the largest offered rate the serving loop
    sustains at a p99 no higher than the one-call arm's p99 at 80% of that
    arm's saturation throughput (equal p99)."""
    trace = serving_trace(njobs)
    rng = np.random.default_rng(1234)

    def pinned(rows, cols):
        t = torch.empty((rows, cols), dtype=torch.int64).pin_memory()
        return t, t.numpy().view(np.uint64)

    pool_log = 24
    pool_t, pool = pinned(1 << pool_log, 4)
    pool[:] = rand_fr(1 << pool_log, 2024)
    offs = [int(rng.integers(0, (1 << pool_log) - (1 << k) + 1)) for _, _, k in trace]
    inputs = [pool[o:o + (1 << k)] for o, (_, _, k) in zip(offs, trace)]

    consts = {}
    for k in range(12, 25):
        w = root_of_unity(k)
        consts[k] = dict(omega=mont(w), omega_inv=mont(pow(w, -1, R_MOD)), divisor=mont(pow(1 << k, -1, R_MOD)))
    g7 = mont(7)

    def out_rows(kind, k):
        return 1 if kind == "msm" else (1 << (k + 2) if kind == "lde" else 1 << k)

    def out_cols(kind):
        return 12 if kind == "msm" else 4

    ring = {}
    RING = 4
    ring_slot = []
    seen = {}
    for _, kind, k in trace:
        key = (kind, k)
        if key not in ring:
            ring[key] = [pinned(out_rows(kind, k), out_cols(kind)) for _ in range(RING)]
        i = seen.get(key, 0)
        seen[key] = i + 1
        ring_slot.append(ring[key][i % RING][1])
    nb = 1 << 20
    bases = gen_bases(zk, torch, nb, 4545, dev).cpu().numpy().view(np.uint64)

    def make_job(i, out):
        _, kind, k = trace[i]
        a = inputs[i]
        if kind == "ntt":
            return zk.ntt_job(a, out, k, consts[k]["omega"])
        if kind == "lde":
            return zk.lde_job(a, out, k, k + 2, consts[k]["omega_inv"], consts[k]["divisor"], g7,
                              consts[k + 2]["omega"])
        return zk.msm_job(a, out, 1 << k, bid)

    def pct(x, q):
        return float(np.percentile(np.asarray(x), q)) if len(x) else None

    srv = zk.Server(device=dev, hbm_budget=hbm_budget, max_wave_jobs=wave_jobs)
    bid = srv.add_bases(bases)

    def run_server(offered, jobs_idx=None, outs=None):
        """offered: jobs/s for an open loop, None for a closed loop"""
        idx = list(range(len(trace))) if jobs_idx is None else jobs_idx
        lats = [None] * len(idx)
        tickets = [None] * len(idx)
        done_evt = threading.Event()

        def waiter():
            for m in range(len(idx)):
                while tickets[m] is None:
                    time.sleep(0.0002)
                lats[m] = srv.wait(tickets[m]) / 1e3
            done_evt.set()

        thw = threading.Thread(target=waiter)
        thw.start()
        t0 = time.perf_counter()
        keep = []
        t_first = trace[idx[0]][0]
        for m, i in enumerate(idx):
            if offered:
                d = t0 + (trace[i][0] - t_first) / offered - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            j = make_job(i, ring_slot[i] if outs is None else outs[m])
            keep.append(j)
            tickets[m] = srv.submit(j)
        done_evt.wait()
        thw.join()
        return lats, time.perf_counter() - t0

    stream = torch.cuda.Stream(device=dev)
    d_bases = torch.from_numpy(bases.view(np.int64)).to(f"cuda:{dev}")
    d_out = torch.zeros(12, dtype=torch.int64, device=f"cuda:{dev}")

    def one_call(i, out, normalised=False):
        _, kind, k = trace[i]
        if normalised and kind == "msm":
            # the serving loop returns normalised points (Z = one): compare
            # with the host-buffer call, which normalises too
            out[:] = zk.msm(inputs[i], bases[: 1 << k], device=dev).reshape(out.shape)
            return
        a = torch.from_numpy(inputs[i].view(np.int64))
        o = torch.from_numpy(out.view(np.int64))
        with torch.cuda.stream(stream):
            d = a.to(f"cuda:{dev}", non_blocking=True)
            if kind == "ntt":
                zk.ntt_dev(d, k, consts[k]["omega"], stream=stream)
                o.copy_(d, non_blocking=True)
            elif kind == "lde":
                e = torch.empty((1 << (k + 2), 4), dtype=torch.int64, device=f"cuda:{dev}")
                zk.lagrange_to_extended_dev(d, e, k, k + 2, consts[k]["omega_inv"], consts[k]["divisor"], g7,
                                            consts[k + 2]["omega"], stream=stream)
                o.copy_(e, non_blocking=True)
            else:
                zk.msm_dev(d, d_bases[: 1 << k], d_out, stream=stream)
                o.copy_(d_out.view(1, 12), non_blocking=True)
        stream.synchronize()

    def run_plain(offered):
        lats = []
        t0 = time.perf_counter()
        for i, (at, kind, k) in enumerate(trace):
            arrive = t0
            if offered:
                arrive = t0 + (at - trace[0][0]) / offered
                d = arrive - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            one_call(i, ring_slot[i])
            lats.append(time.perf_counter() - arrive)
        return lats, time.perf_counter() - t0

    n = len(trace)
    # ---- warm-up: tables, pools, allocator ----
    run_server(None)
    for key, slots in ring.items():
        i = next(m for m, (_, kd, k) in enumerate(trace) if (kd, k) == key)
        one_call(i, slots[0][1])
    # ---- configured load: Poisson 2000 jobs/s, and saturation ----
    # closed loops: three runs per arm, the median run (by span) reported and
    # every run's rate listed, so that one run caught by a host-side stall
    # does not set the saturation figures or the one-call capacity
    lat_s, span_s = run_server(rate)
    (lat_sc, span_sc), sc_runs = median_closed_run(run_server, n)
    lat_p, span_p = run_plain(rate)
    (lat_pc, span_pc), pc_runs = median_closed_run(run_plain, n)
    st = srv.stats()
    one_cap = n / span_pc
    # ---- equal p99: each arm's p99 latency over a sweep of offered rates on
    # the same Poisson trace; for every p99 the one-call arm reaches, the
    # largest rate the serving loop sustains within that p99 ----
    one_curve = []
    for frac in (0.5, 0.7, 0.8, 0.9, 0.95):
        lat_x, span_x = run_plain(frac * one_cap)
        one_curve.append({"offered_jobs_s": round(frac * one_cap, 1), "achieved_jobs_s": round(n / span_x, 1),
                          "p50_ms": round(pct(lat_x, 50) * 1e3, 2), "p99_ms": round(pct(lat_x, 99) * 1e3, 2)})
    sweep = []
    for mult in (0.5, 1.0, 1.5, 2.0, 2.5, 3.0, 3.5, 4.0):
        lam = one_cap * mult
        lat_b, span_b = run_server(lam)
        sweep.append({"offered_jobs_s": round(lam, 1), "achieved_jobs_s": round(n / span_b, 1),
                      "p50_ms": round(pct(lat_b, 50) * 1e3, 2), "p99_ms": round(pct(lat_b, 99) * 1e3, 2)})
        if pct(lat_b, 99) > 4 * max(r["p99_ms"] for r in one_curve) / 1e3:
            break
    # for each target p99: the largest measured rate within it, refined by
    # bisection toward the smallest higher measured rate that exceeds it
    # (three runs per target, every run recorded in the sweep)
    at_p99 = []
    for r in one_curve:
        target = r["p99_ms"]
        ok = [b["offered_jobs_s"] for b in sweep if b["p99_ms"] <= target]
        best = max(ok) if ok else None
        if best is not None:
            over = [b["offered_jobs_s"] for b in sweep if b["offered_jobs_s"] > best and b["p99_ms"] > target]
            hi = min(over) if over else None
            for _ in range(3 if hi is not None else 0):
                mid = 0.5 * (best + hi)
                lat_m, span_m = run_server(mid)
                p99 = pct(lat_m, 99) * 1e3
                sweep.append({"offered_jobs_s": round(mid, 1), "achieved_jobs_s": round(n / span_m, 1),
                              "p50_ms": round(pct(lat_m, 50) * 1e3, 2), "p99_ms": round(p99, 2),
                              "bisection_for_p99_ms": target})
                if p99 <= target:
                    best = mid
                else:
                    hi = mid
        at_p99.append({"p99_ms": target, "one_call_jobs_s": r["offered_jobs_s"],
                       "batched_jobs_s": round(best, 1) if best is not None else None,
                       "ratio": round(best / r["offered_jobs_s"], 3) if best is not None else None})
    # ---- verification: every job, batched (in waves, own buffers) vs alone ----
    verified, checked, chunk = 0, 0, []
    arena_bytes = 4 << 30
    arena_t, arena = pinned(arena_bytes // 32, 4)
    scratch_t, scratch = pinned(1 << 24, 4)
    arena_flat = arena.reshape(-1)
    scratch_flat = scratch.reshape(-1)

    def flush(chunk):
        nonlocal verified, checked
        if not chunk:
            return
        outs, pos = [], 0
        for i in chunk:
            _, kind, k = trace[i]
            words = out_rows(kind, k) * out_cols(kind)
            outs.append(arena_flat[pos:pos + words].reshape(out_rows(kind, k), out_cols(kind)))
            pos += (words + 7) // 8 * 8
        run_server(None, chunk, outs)
        for i, o in zip(chunk, outs):
            ref = scratch_flat[: o.size].reshape(o.shape)
            one_call(i, ref, normalised=True)
            checked += 1
            verified += int(np.array_equal(o, ref))

    used = 0
    for i, (_, kind, k) in enumerate(trace):
        words = out_rows(kind, k) * out_cols(kind)
        need = (words + 7) // 8 * 8 * 8
        if chunk and (used + need > arena_bytes or len(chunk) >= wave_jobs):
            flush(chunk)
            chunk, used = [], 0
        chunk.append(i)
        used += need
    flush(chunk)
    st_after = srv.stats()
    srv.close()
    del arena_t, arena, scratch_t, scratch
    if verified != n:
        raise RuntimeError(f"serving: {n - verified} of {n} jobs differ from the same job run alone")

    # device time of each job alone (inputs resident, no copies; best of 3),
    # summed over the trace: the compute floor of any schedule on one GPU
    dev_ms = {}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for key in ring:
        kind, k = key
        i = next(m for m, (_, kd, kk) in enumerate(trace) if (kd, kk) == key)
        d = torch.from_numpy(inputs[i].view(np.int64)).to(f"cuda:{dev}")
        e = torch.empty((1 << (k + 2), 4), dtype=torch.int64, device=f"cuda:{dev}") if kind == "lde" else None
        best_ms = 1e30
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
            best_ms = min(best_ms, ev0.elapsed_time(ev1))
        dev_ms[key] = best_ms
        del d, e
    trace_dev_s = sum(dev_ms[(kind, k)] for _, kind, k in trace) / 1e3
    by_kind = {kd: round(sum(dev_ms[(kind, k)] for _, kind, k in trace if kind == kd) / 1e3, 3)
               for kd in ("ntt", "lde", "msm")}
    h2d = sum((1 << k) * 32 for _, kind, k in trace)
    d2h = sum(96 if kind == "msm" else (1 << (k + 2 if kind == "lde" else k)) * 32 for _, kind, k in trace)
    pcie = pcie_bandwidth(torch, dev)
    pcie.update({"trace_h2d_gb": round(h2d / 1e9, 2), "trace_d2h_gb": round(d2h / 1e9, 2),
                 "batched_closed_loop_d2h_gbs": round(d2h / span_sc / 1e9, 2),
                 "batched_closed_loop_h2d_gbs": round(h2d / span_sc / 1e9, 2),
                 "one_call_closed_loop_d2h_gbs": round(d2h / span_pc / 1e9, 2)})
    eq = {"rule": "same Poisson trace at each offered rate; for each p99 the one-call arm reaches (at 50-95% of "
                  "its saturation throughput), the largest offered rate at which the serving loop's p99 is no "
                  "higher: the largest such rate of a sweep in steps of 0.5x the one-call capacity, then three "
                  "bisection runs toward the next swept rate; ratio of offered rates",
          "at_p99": at_p99, "one_call_curve": one_curve}
    return {
        "jobs": n, "offered_rate_jobs_s": rate,
        "mix": "35% NTT 2^12-2^22, 35% coset LDE x4 2^12-2^22, 30% MSM 2^14-2^20 (resident 2^20 bases)",
        "inputs": "per job: its own seeded window of a pinned pool of 2^24 uniform Fr",
        "verified": f"{verified}/{checked} equal to the same job run alone",
        "open_loop_2000": {
            "batched": {"jobs_s": round(n / span_s, 1), "p50_ms": round(pct(lat_s, 50) * 1e3, 3),
                        "p99_ms": round(pct(lat_s, 99) * 1e3, 3)},
            "one_call_per_job": {"jobs_s": round(n / span_p, 1), "p50_ms": round(pct(lat_p, 50) * 1e3, 3),
                                 "p99_ms": round(pct(lat_p, 99) * 1e3, 3)}},
        "closed_loop_saturation": {
            "batched_jobs_s": round(n / span_sc, 1), "one_call_per_job_jobs_s": round(one_cap, 1),
            "speedup": round(span_pc / span_sc, 3),
            "batched_p99_ms": round(pct(lat_sc, 99) * 1e3, 3), "one_call_p99_ms": round(pct(lat_pc, 99) * 1e3, 3),
            "runs": "median of 3 closed-loop runs per arm",
            "batched_runs_jobs_s": sc_runs, "one_call_runs_jobs_s": pc_runs},
        "equal_p99": eq, "batched_rate_sweep": sweep, "eager_waves": os.environ.get("ZKGPU_SERVER_EAGER_WAVES", "8 (library default)"),
        "server": {"waves": st["waves"], "batch_launches": st["batch_launches"], "hbm_peak_gb":
                   round(st["hbm_peak"] / 1e9, 2), "rejected": st["rejected"], "failed": st_after["failed"],
                   "msm_merged_passes": st_after["msm_merged_passes"],
                   "msm_merged_jobs": st_after["msm_merged_jobs"]},
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
    out["pipes"] = PIPE_FRACS["msm_apply"]
    return out


HBM_GBS = 6543.1
# DRAM bytes (read + write) per launch over algorithmic bytes, from one ncu
# capture of the same kernel on a smaller case (traffic grows with the
# elements processed): ntt_pass_kernel<6> on a 2^24 transform, plan 6+6+6+6,
# launches 1.588 / 1.611 GB and 1.051 / 1.082 GB.
TRAFFIC_RATIO = {"ntt_pass_b6": 0.97}
TRAFFIC_SOURCE = {"ntt_pass_b6": "ncu dram__bytes_read.sum + dram__bytes_write.sum of ntt_pass_kernel<6> on a "
                                 "2^24 transform (plan 6+6+6+6), scaled by algorithmic bytes"}
# Pipe utilisation of the dominant kernels from one ncu --set full capture
# each (ntt_pass_kernel<6> on a 2^24 transform, ba_apply_kernel<1> in the
# 2^22 MSM): the IMAD-convention frac counts products per second, these say
# how busy the pipes the FP64-limb product actually uses are.
PIPE_FRACS = {
    "ntt_pass_b6": {"fp64": 0.398, "alu": 0.525, "fma_imad": 0.097, "issue_active": 0.579, "warps_active": 0.245,
                    "source": "ncu sm__inst_executed_pipe_{fp64,alu,fma}, smsp__issue_active, sm__warps_active of "
                              "ntt_pass_kernel<6> on a 2^24 transform (second pass)"},
    "msm_apply": {"kernel": "ba_apply_kernel<1> (round 0, 55 % of the MSM with the other rounds)",
                  "fp64": 0.350, "alu": 0.504, "fma_imad": 0.105, "issue_active": None, "warps_active": 0.238,
                  "source": "ncu sections SpeedOfLight, WarpStateStats, ComputeWorkloadAnalysis and LaunchStats "
                            "of ba_apply_kernel<1> in the 2^22 MSM (issue active not in those sections)"},
}


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
    `lde20` = LDE 2^20 -> 2^22, `msm20` / `msm22` = MSM of 2^20 / 2^22 points
    (10% of the scalars < 2^16)."""
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
    elif args.case in ("msm20", "msm22"):
        n = 1 << (20 if args.case == "msm20" else 22)
        sc = rand_fr(n, 8)
        sc[: n // 10] = small_fr(n // 10, 9)  # 10% of the scalars < 2^16, as in the benchmark
        s = torch.from_numpy(sc.view(np.int64)).cuda()
        b = gen_bases(zk, torch, n, 4141, 0)
        out = torch.zeros(12, dtype=torch.int64, device="cuda")

        def step():
            zk.msm_dev(s, b, out, stream=stream)
    torch.cuda.synchronize()  # inputs were made on torch's stream
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
    ap.add_argument("--case", choices=["ntt22", "ntt24", "lde20", "msm20", "msm22"], default=None,
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
