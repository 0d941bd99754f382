"""CPU: the serving loop's host logic — job footprints and the HBM-budget
admission policy (strict arrival order, oversize rejected, budget never
exceeded).  These entry points touch no device."""
import numpy as np


def test_footprints(zk):
    a = np.zeros((1, 4), np.uint64)
    ntt = zk.ntt_job(a, a, 20, np.zeros(4, np.uint64))
    assert zk.job_footprint(ntt) >= 2 * (1 << 20) * 32
    lde = zk.lde_job(a, a, 20, 22, *([np.zeros(4, np.uint64)] * 4))
    assert zk.job_footprint(lde) >= 2 * (1 << 22) * 32
    small, big = zk.msm_job(a, a, 1 << 14, 0), zk.msm_job(a, a, 1 << 20, 0)
    assert zk.job_footprint(big) > zk.job_footprint(small) >= (1 << 14) * 32


def test_admission_fifo_and_budget():
    import zk_gpu_b200 as zk
    rng = np.random.default_rng(3)
    fp = rng.integers(1, 100, 200).astype(np.uint64)
    budget = 250
    peak, rounds = zk.admission_simulate(budget, fp)
    assert peak <= budget
    assert (rounds >= 0).all()
    # strict arrival order: admission rounds never decrease
    assert (np.diff(rounds) >= 0).all()
    # every round is filled greedily: the next job did not fit
    for r in range(rounds.max()):
        used = fp[rounds == r].sum()
        nxt = fp[np.argmax(rounds == r + 1)]
        assert used <= budget and used + nxt > budget


def test_admission_rejects_oversize():
    import zk_gpu_b200 as zk
    fp = np.array([10, 500, 20, 30], np.uint64)
    peak, rounds = zk.admission_simulate(100, fp)
    assert rounds[1] == -1
    assert list(rounds[[0, 2, 3]]) == [0, 0, 0]
    assert peak == 60
