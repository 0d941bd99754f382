"""GPU parity: the sm_100a Pippenger MSM through the C ABI against the CPU
oracle (halo2 best_multiexp restated), bit-exact after affine normalisation."""
import ctypes

import numpy as np
import pytest

from oracle import bigref as B

pytestmark = pytest.mark.gpu


def affine_of(out12):
    """normalised Jacobian (x, y, one) or all-zero identity -> 8 words (x, y)"""
    out12 = np.asarray(out12, np.uint64)
    if not out12[8:12].any():
        assert not out12.any()
        return np.zeros(8, np.uint64)
    return out12[:8].copy()


@pytest.mark.parametrize("n", [0, 1, 2, 3, 7, 31, 255, 256, 257, 1000, 4096, 65536])
def test_msm_sizes(zk, oracle, n):
    s = oracle.rand_fr(n, 100 + n)
    pts = oracle.rand_bases(n, 200 + n)
    got = affine_of(zk.msm(s, pts))
    assert np.array_equal(got, oracle.multiexp(s, pts))


def test_msm_reference_api(zk, oracle):
    """parallel_msm_api(device, data, GpuAffine*, len, GpuProjective*) (src/api.rs:12)"""
    n = 1024
    s = oracle.rand_fr(n, 5)
    pts = oracle.rand_bases(n, 6)
    acc = zk.GpuProjective()
    assert zk.parallel_msm_api(0, s, pts, n, acc) == 0
    out = np.concatenate([np.array(acc.x, np.uint64), np.array(acc.y, np.uint64), np.array(acc.z, np.uint64)])
    assert np.array_equal(affine_of(out), oracle.multiexp(s, pts))
    assert np.array_equal(np.array(acc.z, np.uint64), oracle.to_mont(1, oracle.FQ))


def test_msm_edge_cases(zk, oracle):
    n = 2048
    pts, k = oracle.rand_bases(n, 9, with_dlog=True)
    # all-zero scalars -> identity
    assert not zk.msm(np.zeros((n, 4), np.uint64), pts).any()
    s = oracle.rand_fr(n, 10)
    # identity bases (0, 0) are skipped
    pts2 = pts.copy()
    pts2[::7] = 0
    assert np.array_equal(affine_of(zk.msm(s, pts2)), oracle.multiexp(s, pts2))
    # P + (-P) cancels: scalar 1 and r - 1 on the same base, everything else zero
    s3 = np.zeros((n, 4), np.uint64)
    pts3 = pts.copy()
    pts3[1] = pts3[0]
    s3[0] = oracle.to_mont(1)
    s3[1] = oracle.to_mont(B.R_MOD - 1)
    assert not zk.msm(s3, pts3).any()
    # the same point many times in one bucket (doubling inside bucket sums)
    pts4 = np.tile(pts[0], (n, 1))
    s4 = np.tile(oracle.to_mont(3), (n, 1))
    assert np.array_equal(affine_of(zk.msm(s4, pts4)), oracle.multiexp(s4, pts4))
    # extreme scalars: r - 1, 2^253, 2^k - 1 patterns hitting window boundaries
    vals = [B.R_MOD - 1, 1 << 253, (1 << 254) - 1 - (1 << 200), (1 << 16) - 1, 1 << 15, (1 << 15) + 1, 2**128 - 1]
    s5 = oracle.rand_fr(n, 11)
    for i, v in enumerate(vals):
        s5[i] = oracle.to_mont(v % B.R_MOD)
    assert np.array_equal(affine_of(zk.msm(s5, pts)), oracle.multiexp(s5, pts))


@pytest.mark.parametrize("value", [1, 2**15, 2**16 + 1, 7])
def test_msm_skewed_buckets(zk, oracle, value):
    """every scalar equal: each window's points all land in one bucket, which
    the sub-bucket split and the block-wide reduction must handle"""
    n = 1 << 16
    s = np.tile(oracle.to_mont(value), (n, 1))
    pts, k = oracle.rand_bases(n, 40 + value % 97, with_dlog=True)
    assert np.array_equal(affine_of(zk.msm(s, pts)), oracle.msm_by_dlog(s, k))


def test_msm_small_scalar_mix(zk, oracle):
    n = 1 << 16
    s = oracle.rand_fr(n, 12)
    small = oracle.rand_fr_small(n // 10, 13, bits=16)
    s[: n // 10] = small
    pts, k = oracle.rand_bases(n, 14, with_dlog=True)
    assert np.array_equal(affine_of(zk.msm(s, pts)), oracle.msm_by_dlog(s, k))


def test_msm_full_size_2p22(zk, oracle):
    """benchmark size: 2^22 bases, 10% scalars < 2^16, checked through the
    bases' discrete logs: sum s_i [k_i] G = [sum s_i k_i] G"""
    n = 1 << 22
    s = oracle.rand_fr(n, 22)
    s[: n // 10] = oracle.rand_fr_small(n // 10, 23, bits=16)
    pts, k = oracle.rand_bases(n, 24, with_dlog=True)
    assert np.array_equal(affine_of(zk.msm(s, pts)), oracle.msm_by_dlog(s, k))


def test_msm_device_api(zk, oracle):
    torch = pytest.importorskip("torch")
    n = 5000
    s = oracle.rand_fr(n, 31)
    pts = oracle.rand_bases(n, 32)
    ts = torch.from_numpy(s.view(np.int64)).cuda()
    tb = torch.from_numpy(pts.view(np.int64)).cuda()
    out = torch.zeros(12, dtype=torch.int64, device="cuda")
    zk.msm_dev(ts, tb, out)
    torch.cuda.synchronize()
    jac = out.cpu().numpy().view(np.uint64)
    assert np.array_equal(oracle.g1_normalize(jac), oracle.multiexp(s, pts))


def test_g1_mul_fixed_matches_oracle_bases(zk, oracle):
    """k_i * (1, 2) on the device (the MSM-bases generator) equals the
    oracle's fixed-base multiples for the same seeded k_i, bit-exact, with
    the edge scalars 0 (identity (0, 0)), 1 (the generator) and r - 1 (-G)."""
    import torch
    n = 5000
    pts, k = oracle.rand_bases(n, 31, with_dlog=True)
    r = B.R_MOD
    k[0] = oracle.to_mont(0)
    k[1] = oracle.to_mont(1)
    k[2] = oracle.to_mont(r - 1)
    d_k = torch.from_numpy(k.view(np.int64)).cuda()
    d_out = torch.empty((n, 8), dtype=torch.int64, device="cuda")
    zk.g1_mul_fixed_dev(d_k, d_out)
    got = d_out.cpu().numpy().view(np.uint64)
    q = zk.FQ_MODULUS
    assert not got[0].any()
    assert np.array_equal(got[1], zk.G1_GENERATOR)
    assert np.array_equal(got[2][:4], zk.G1_GENERATOR[:4])
    assert np.array_equal(got[2][4:], oracle.to_mont(q - 2, oracle.FQ))
    assert np.array_equal(got[3:], pts[3:])


@pytest.mark.parametrize("n", [1, 300, 1 << 14, 1 << 17])
def test_msm_host_and_device_horner_agree(zk, oracle, n):
    """the host-buffer call finishes the windows' Horner step on the host, the
    device call on the GPU: both must give the same (normalised) point"""
    import torch
    s = oracle.rand_fr(n, 700 + n)
    pts = oracle.rand_bases(n, 701 + n)
    host = zk.msm(s, pts)
    d_s = torch.from_numpy(s.view(np.int64)).cuda()
    d_b = torch.from_numpy(pts.view(np.int64)).cuda()
    d_o = torch.zeros(12, dtype=torch.int64, device="cuda")
    zk.msm_dev(d_s, d_b, d_o)
    torch.cuda.synchronize()
    jac = d_o.cpu().numpy().view(np.uint64)
    assert np.array_equal(affine_of(host), oracle.g1_normalize(jac))
    if n <= 1 << 14:
        assert np.array_equal(affine_of(host), oracle.multiexp(s, pts))


@pytest.mark.parametrize("n_pos,n_neg", [(2048, 2048), (3000, 1096), (1, 1), (517, 0)])
def test_msm_in_bucket_doubling_and_cancellation(zk, oracle, n_pos, n_neg):
    """All scalars equal, so each window has a single bucket holding copies
    of P and -P in the order the sort left them: the pairwise (affine) bucket
    sums meet P + P (doubling), P + (-P) (identity) and identity operands."""
    pts, k = oracle.rand_bases(1, 77, with_dlog=True)
    q = zk.FQ_MODULUS
    p = pts[0]
    neg = p.copy()
    neg[4:] = oracle.to_mont((q - oracle.from_mont(p[4:], oracle.FQ)) % q, oracle.FQ)
    n = n_pos + n_neg
    rng = np.random.default_rng(n_pos * 7 + n_neg)
    order = rng.permutation(n)
    bases = np.empty((n, 8), np.uint64)
    bases[order[:n_pos]] = p
    bases[order[n_pos:]] = neg
    s = np.tile(oracle.to_mont(0xBEEF), (n, 1))
    # expected: 0xBEEF * (n_pos - n_neg) * k * G
    kk = oracle.mul(oracle.to_mont((n_pos - n_neg) % B.R_MOD), k[0])
    want = oracle.msm_by_dlog(s[:1], kk.reshape(1, 4))
    assert np.array_equal(affine_of(zk.msm(s, bases)), want)
