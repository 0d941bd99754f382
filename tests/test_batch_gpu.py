"""GPU: batched NTTs of uneven sizes in one persistent launch (graph replay),
each result bit-exact against the oracle, on two consecutive runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_jobs(oracle, torch, rng, sizes, seed):
    jobs, refs = [], []
    for i, k in enumerate(sizes):
        n = 1 << k
        a = oracle.rand_fr(n, seed + i)
        inverse = bool(rng.integers(0, 2))
        coset = bool(rng.integers(0, 2))
        w = oracle.omega(k)
        job = {"tensor": torch.from_numpy(a.view(np.int64)).cuda(), "log_n": k}
        x = a
        if coset:
            c = oracle.mul(oracle.to_mont(7), oracle.omega(k + 1))
            job["coset"] = c
            x = oracle.distribute_powers(x, c)
        if inverse:
            w = oracle.inv(w)
            job["scale"] = oracle.inv(oracle.to_mont(n))
            ref = oracle.ifft(x, w, k, job["scale"])
        else:
            ref = oracle.best_fft(x, w, k)
        job["omega"] = w
        jobs.append(job)
        refs.append(ref)
    return jobs, refs


def test_batch_uneven_sizes_two_runs(zk, oracle):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    sizes = [int(k) for k in rng.integers(3, 18, 48)] + [20, 12, 11, 3]
    jobs, refs = make_jobs(oracle, torch, rng, sizes, 100)
    batch = zk.NttBatch(jobs)
    info = batch.info()
    assert info["passes"] >= len(sizes) and info["grid"] > 0
    batch.run()
    torch.cuda.synchronize()
    batch.check()
    for j, ref in zip(jobs, refs):
        assert np.array_equal(j["tensor"].cpu().numpy().view(np.uint64), ref), j["log_n"]
    # second run: refill the same buffers with new inputs; the graph is replayed
    rng2 = np.random.default_rng(5)  # replay the same draws: sizes, then per-job flags
    rng2.integers(3, 18, 48)
    jobs2, refs2 = make_jobs(oracle, torch, rng2, sizes, 900)
    for j, j2 in zip(jobs, jobs2):
        assert ("coset" in j) == ("coset" in j2) and ("scale" in j) == ("scale" in j2)
    for j, j2 in zip(jobs, jobs2):
        j["tensor"].copy_(j2["tensor"])
    batch.run()
    torch.cuda.synchronize()
    batch.check()
    for j, ref in zip(jobs, refs2):
        assert np.array_equal(j["tensor"].cpu().numpy().view(np.uint64), ref), j["log_n"]
    batch.close()


def test_batch_matches_single_calls(zk, oracle):
    """same job alone (zkgpu_ntt_dev) and inside a batch mix: identical output"""
    torch = pytest.importorskip("torch")
    k = 16
    a = oracle.rand_fr(1 << k, 77)
    w = oracle.omega(k)
    alone = torch.from_numpy(a.view(np.int64)).cuda()
    zk.ntt_dev(alone, k, w)
    mixed = torch.from_numpy(a.view(np.int64)).cuda()
    others = [{"tensor": torch.from_numpy(oracle.rand_fr(1 << s, s).view(np.int64)).cuda(), "log_n": s,
               "omega": oracle.omega(s)} for s in (10, 14, 19, 8)]
    batch = zk.NttBatch(others[:2] + [{"tensor": mixed, "log_n": k, "omega": w}] + others[2:])
    batch.run()
    torch.cuda.synchronize()
    batch.check()
    assert torch.equal(alone, mixed)
    batch.close()


def test_release_cached_keeps_live_batches_correct(zk, oracle):
    """zkgpu_release_cached drops the device's cached tables and pooled
    memory; a batch built before it still holds its own tables, and the next
    plain call rebuilds what it needs — all results stay bit-exact."""
    torch = pytest.importorskip("torch")
    k = 14
    a = oracle.rand_fr(1 << k, 91)
    w = oracle.omega(k)
    t = torch.from_numpy(a.view(np.int64)).cuda()
    batch = zk.NttBatch([{"tensor": t, "log_n": k, "omega": w}])
    zk.release_cached(0)
    batch.run()
    torch.cuda.synchronize()
    batch.check()
    assert np.array_equal(t.cpu().numpy().view(np.uint64), oracle.best_fft(a, w, k))
    batch.close()
    zk.release_cached(0)
    t2 = torch.from_numpy(a.view(np.int64)).cuda()
    zk.ntt_dev(t2, k, w)
    torch.cuda.synchronize()
    assert np.array_equal(t2.cpu().numpy().view(np.uint64), oracle.best_fft(a, w, k))
