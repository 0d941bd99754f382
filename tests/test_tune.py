"""Autotuner: plan validation and installation (CPU), and on the GPU that
every plan shape the tuner may pick is bit-exact against the oracle, that
tuning installs valid choices, and that saved choices load back."""
import numpy as np
import pytest


def test_plan_validation_cpu(zk):
    # unsupported plans are refused without touching a device
    invalid = [(12, [12]),              # one pass is at most 11 bits
               (12, [2, 10]),           # passes are at least 3 bits
               (12, [6, 5]),            # widths must sum to log_n
               (20, [12, 8]),           # at most 11 bits per pass
               (29, [10, 10, 9]),       # beyond the field's two-adicity
               (25, [5, 5, 5, 5, 5])]   # at most 4 passes
    for log_n, bits in invalid:
        with pytest.raises(zk.ZkGpuError):
            zk.set_ntt_plan(log_n, bits, device=5)
    zk.set_ntt_plan(20, [10, 10], device=5)
    assert zk.get_ntt_plan(20, device=5) == [10, 10]
    zk.set_ntt_plan(20, [], device=5)          # back to the built-in plan
    assert zk.get_ntt_plan(20, device=5) == [7, 7, 6]
    zk.set_ntt_plan(9, [9], device=5)
    zk.set_ntt_plan(9, [3, 3, 3], device=5)
    assert zk.get_ntt_plan(9, device=5) == [3, 3, 3]
    zk.set_ntt_plan(9, [], device=5)
    assert zk.get_ntt_plan(24, device=5) == [8, 8, 8]
    assert zk.get_ntt_plan(2, device=5) == []
    with pytest.raises(zk.ZkGpuError):
        zk.set_msm_window(22, 3, device=5)
    zk.set_msm_window(22, 13, device=5)
    assert zk.get_msm_window(22, device=5) == 13
    zk.set_msm_window(22, 0, device=5)
    assert zk.get_msm_window(22, device=5) == 16


PLANS = [(6, [3, 3]), (9, [3, 3, 3]), (11, [11]), (11, [5, 6]), (12, [3, 9]), (12, [9, 3]), (12, [3, 3, 3, 3]),
         (14, [11, 3]), (16, [4, 4, 4, 4]), (17, [6, 11]), (20, [10, 10]), (20, [11, 9]), (22, [11, 11]),
         (22, [6, 5, 6, 5])]


@pytest.mark.gpu
@pytest.mark.parametrize("log_n,bits", PLANS)
def test_every_plan_shape_bit_exact(zk, oracle, log_n, bits):
    """forward, inverse-with-scale and coset transforms under an installed plan
    equal the oracle (and the LDE path, which reads the source out of place)"""
    zk.set_ntt_plan(log_n, bits)
    try:
        assert zk.get_ntt_plan(log_n) == bits
        a = oracle.rand_fr(1 << log_n, 900 + log_n)
        w = oracle.omega(log_n)
        assert np.array_equal(zk.fft(a, w, log_n), oracle.best_fft(a, w, log_n))
        c = oracle.to_mont(5)
        assert np.array_equal(zk.coset_fft(a, w, log_n, c), oracle.best_fft(oracle.distribute_powers(a, c), w, log_n))
        wi, d = oracle.inv(w), oracle.inv(oracle.to_mont(1 << log_n))
        assert np.array_equal(zk.ifft(a, wi, log_n, d), oracle.ifft(a, wi, log_n, d))
        if log_n <= 20:
            k = log_n - 2
            vals = oracle.rand_fr(1 << k, 77)
            wk = oracle.omega(k)
            wik, dk = oracle.inv(wk), oracle.inv(oracle.to_mont(1 << k))
            g = oracle.to_mont(7)
            ref = oracle.coeff_to_extended(oracle.ifft(vals, wik, k, dk), k, log_n, g, w)
            assert np.array_equal(zk.lagrange_to_extended(vals, k, log_n, wik, dk, g, w), ref)
    finally:
        zk.set_ntt_plan(log_n, [])


@pytest.mark.gpu
def test_batch_under_installed_plans(zk, oracle):
    torch = pytest.importorskip("torch")
    zk.set_ntt_plan(12, [3, 9])
    zk.set_ntt_plan(14, [4, 5, 5])
    try:
        jobs, refs = [], []
        for i, k in enumerate([12, 14, 12, 14, 10]):
            a = oracle.rand_fr(1 << k, 300 + i)
            w = oracle.omega(k)
            t = torch.from_numpy(a.view(np.int64)).cuda()
            jobs.append({"tensor": t, "log_n": k, "omega": w})
            refs.append(oracle.best_fft(a, w, k))
        b = zk.NttBatch(jobs)
        b.run()
        torch.cuda.synchronize()
        for j, r in zip(jobs, refs):
            assert np.array_equal(j["tensor"].cpu().numpy().view(np.uint64), r)
    finally:
        zk.set_ntt_plan(12, [])
        zk.set_ntt_plan(14, [])


@pytest.mark.gpu
def test_autotune_installs_valid_choices_and_roundtrips(zk, oracle, tmp_path):
    ms = zk.autotune(zk.TUNE_NTT_BATCHED, 10, 13)
    assert ms > 0
    ms += zk.autotune(zk.TUNE_NTT | zk.TUNE_MSM, 14, 15, reps=2)
    plans = {k: zk.get_ntt_plan(k) for k in range(10, 16)}
    for k, p in plans.items():
        assert sum(p) == k
    windows = {k: zk.get_msm_window(k) for k in (14, 15)}
    path = str(tmp_path / "tune.txt")
    zk.tune_save(path)
    for k in plans:
        zk.set_ntt_plan(k, [])
    for k in windows:
        zk.set_msm_window(k, 0)
    assert zk.tune_load(path) == len(plans) + len(windows)
    assert {k: zk.get_ntt_plan(k) for k in plans} == plans
    assert {k: zk.get_msm_window(k) for k in windows} == windows
    # results under the tuned choices stay bit-exact
    a = oracle.rand_fr(1 << 15, 15)
    w = oracle.omega(15)
    assert np.array_equal(zk.fft(a, w, 15), oracle.best_fft(a, w, 15))
    s = oracle.rand_fr(1 << 14, 3)
    pts = oracle.rand_bases(1 << 14, 4)
    out = zk.msm(s, pts)
    assert np.array_equal(out[:8], oracle.multiexp(s, pts))
    for k in plans:
        zk.set_ntt_plan(k, [])
    for k in windows:
        zk.set_msm_window(k, 0)
