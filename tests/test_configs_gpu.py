"""GPU: the batched and serving workloads at their stated sizes, every job
bit-exact against the oracle.

* 512 independent NTT jobs, log2 size uniform in 10..20, each forward or
  inverse and with or without a coset shift, seeded inputs, run by one
  persistent launch replayed from a CUDA graph under the plans the autotuner
  installs for batched transforms; two runs (the second on refilled inputs).
* The serving mix: NTT and coset-LDE (x4) jobs of 2^12..2^22, MSM jobs of
  2^14..2^20 points against 2^20 resident bases, submitted together into a
  server with 64-job waves, so that MSMs of unequal sizes share one multi-MSM
  pass.  Each result is checked against the oracle (MSMs through the bases'
  known discrete logs) and against the same job run alone.

These replace the one-call-per-job flow of src/gpulock.rs:133-226 with
cuda/fft.cu:275-405 / :450-551 per job.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def _batch_jobs(oracle, torch, sizes, flags, seed):
    jobs, refs = [], []
    for i, (k, (inverse, coset)) in enumerate(zip(sizes, flags)):
        n = 1 << k
        a = oracle.rand_fr(n, seed + i)
        w = oracle.omega(k)
        job = {"tensor": torch.from_numpy(a.view(np.int64)).cuda(), "log_n": k}
        x = a
        if coset:
            c = oracle.mul(oracle.to_mont(7), oracle.omega(k + 2))
            job["coset"] = c
            x = oracle.distribute_powers(x, c)
        if inverse:
            w = oracle.inv(w)
            job["scale"] = oracle.inv(oracle.to_mont(n))
            refs.append(oracle.ifft(x, w, k, job["scale"]))
        else:
            refs.append(oracle.best_fft(x, w, k))
        job["omega"] = w
        jobs.append(job)
    return jobs, refs


def test_batched_512_jobs_tuned_two_runs(zk, oracle):
    torch = pytest.importorskip("torch")
    zk.autotune(zk.TUNE_NTT_BATCHED, 10, 20)
    rng = np.random.default_rng(77)
    sizes = [int(k) for k in rng.integers(10, 21, 512)]
    flags = [(bool(rng.integers(0, 2)), bool(rng.integers(0, 2))) for _ in sizes]
    assert len(set(sizes)) == 11 and any(f[0] and f[1] for f in flags)
    jobs, refs = _batch_jobs(oracle, torch, sizes, flags, 10_000)
    batch = zk.NttBatch(jobs)
    batch.run()
    torch.cuda.synchronize()
    batch.check()
    bad = [i for i, (j, r) in enumerate(zip(jobs, refs)) if not np.array_equal(_host(j["tensor"]), r)]
    assert not bad, f"run 1: jobs {bad[:8]} differ"
    # refill the same buffers with new seeded inputs and replay the graph
    jobs2, refs2 = _batch_jobs(oracle, torch, sizes, flags, 20_000)
    for j, j2 in zip(jobs, jobs2):
        j["tensor"].copy_(j2["tensor"])
    del jobs2
    batch.run()
    torch.cuda.synchronize()
    batch.check()
    bad = [i for i, (j, r) in enumerate(zip(jobs, refs2)) if not np.array_equal(_host(j["tensor"]), r)]
    assert not bad, f"run 2: jobs {bad[:8]} differ"
    batch.close()
    for k in range(10, 21):  # back to the built-in plans for the tests that follow
        zk.set_ntt_plan(k, [])


def _serving_trace(njobs, seed):
    """kind and log2 size per job: 35% NTT 2^12..2^22, 35% coset LDE x4 of
    2^12..2^22, 30% MSM of 2^14..2^20 points"""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(njobs):
        u = rng.random()
        if u < 0.35:
            out.append(("ntt", int(rng.integers(12, 23))))
        elif u < 0.70:
            out.append(("lde", int(rng.integers(12, 23))))
        else:
            out.append(("msm", int(rng.integers(14, 21))))
    return out


def test_serving_mix_at_stated_sizes(zk, oracle):
    torch = pytest.importorskip("torch")
    trace = _serving_trace(96, 99)
    kinds = [k for k, _ in trace]
    assert {"ntt", "lde", "msm"} <= set(kinds)
    nb = 1 << 20
    kb = oracle.rand_fr(nb, 4545)
    d_bases = torch.empty((nb, 8), dtype=torch.int64, device="cuda")
    zk.g1_mul_fixed_dev(torch.from_numpy(kb.view(np.int64)).cuda(), d_bases)
    torch.cuda.synchronize()
    bases = _host(d_bases).copy()
    srv = zk.Server(device=0, hbm_budget=150 * 10**9, max_wave_jobs=64)
    bid = srv.add_bases(bases)
    g7 = oracle.to_mont(7)
    jobs = []
    for i, (kind, k) in enumerate(trace):
        if kind == "msm":
            n = 1 << k
            s = oracle.rand_fr(n, 7000 + i)
            out = np.zeros(12, np.uint64)
            jobs.append((kind, k, zk.msm_job(s, out, n, bid), s, out))
        elif kind == "ntt":
            a = oracle.rand_fr(1 << k, 7000 + i)
            out = np.zeros_like(a)
            jobs.append((kind, k, zk.ntt_job(a, out, k, oracle.omega(k)), a, out))
        else:
            a = oracle.rand_fr(1 << k, 7000 + i)
            out = np.zeros((1 << (k + 2), 4), np.uint64)
            wi, d = oracle.inv(oracle.omega(k)), oracle.inv(oracle.to_mont(1 << k))
            jobs.append((kind, k, zk.lde_job(a, out, k, k + 2, wi, d, g7, oracle.omega(k + 2)), a, out))
    tickets = [srv.submit(j[2]) for j in jobs]
    for t in tickets:
        srv.wait(t, timeout_ms=600_000)
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert st["msm_merged_passes"] >= 1, "no wave ran its MSMs as one multi-MSM pass"
    srv.close()
    for i, (kind, k, jb, inp, out) in enumerate(jobs):
        if kind == "msm":
            aff = out[:8] if out[8:].any() else np.zeros(8, np.uint64)
            assert np.array_equal(aff, oracle.msm_by_dlog(inp, kb[: 1 << k])), f"job {i} msm 2^{k}"
        elif kind == "ntt":
            assert np.array_equal(out, oracle.best_fft(inp, oracle.omega(k), k)), f"job {i} ntt 2^{k}"
        else:
            wi, d = oracle.inv(oracle.omega(k)), oracle.inv(oracle.to_mont(1 << k))
            ref = oracle.coeff_to_extended(oracle.ifft(inp, wi, k, d), k, k + 2, g7, oracle.omega(k + 2))
            assert np.array_equal(out, ref), f"job {i} lde 2^{k}"
