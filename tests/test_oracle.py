"""CPU: the oracle against an independent bigint reference and known answers.

Pins the C restatement of halo2 best_fft / ifft / distribute_powers /
best_multiexp (oracle/zkoracle.c) before anything is compared against it.
"""
import numpy as np
import pytest

from oracle import bigref as B


def test_field_constants(oracle):
    # cuda/bn256.h:37-56 values, re-derived
    R = 1 << 256
    for fid, p in ((oracle.FR, B.R_MOD), (oracle.FQ, B.Q_MOD)):
        one = oracle.to_mont(1, fid)
        assert oracle.to_int(one) == R % p
        assert oracle.from_mont(one, fid) == 1
    assert B.R_MOD.bit_length() == 254 and B.Q_MOD.bit_length() == 254


@pytest.mark.parametrize("fid,p", [(0, B.R_MOD), (1, B.Q_MOD)])
def test_field_ops_vs_bigint(oracle, fid, p):
    rng = np.random.default_rng(1)
    vals = [int(x) for x in rng.integers(0, 2**63, 16)] + [0, 1, p - 1, p - 2, (p - 1) // 2]
    vals = [v % p for v in vals] + [int.from_bytes(rng.bytes(32), "little") % p for _ in range(16)]
    for i, x in enumerate(vals):
        y = vals[(i * 7 + 3) % len(vals)]
        a, b = oracle.to_mont(x, fid), oracle.to_mont(y, fid)
        assert oracle.from_mont(oracle.mul(a, b, fid), fid) == x * y % p
        assert oracle.from_mont(oracle.add(a, b, fid), fid) == (x + y) % p
        assert oracle.from_mont(oracle.sub(a, b, fid), fid) == (x - y) % p
        if x:
            assert oracle.from_mont(oracle.inv(a, fid), fid) == pow(x, -1, p)


def test_root_of_unity(oracle):
    # Fr::ROOT_OF_UNITY = 7^((r-1)/2^28) (bn256.h:57, commented) and its squares
    for k in range(0, 29):
        w = oracle.omega(k)
        assert B.mont_to_int(w) == B.root_of_unity(k)
    w28 = B.root_of_unity(28)
    assert pow(w28, 1 << 28, B.R_MOD) == 1 and pow(w28, 1 << 27, B.R_MOD) == B.R_MOD - 1
    assert hex(w28) == "0x3ddb9f5166d18b798865ea93dd31f743215cf6dd39329c8d34f1ed960c37c9c"


@pytest.mark.parametrize("log_n", [0, 1, 2, 3, 4, 6, 9])
def test_best_fft_vs_dft(oracle, log_n):
    n = 1 << log_n
    a = oracle.rand_fr(n, 100 + log_n)
    out = oracle.best_fft(a, oracle.omega(log_n), log_n)
    ref = B.dft([B.mont_to_int(v) for v in a], B.root_of_unity(log_n))
    assert [B.mont_to_int(v) for v in out] == ref


def test_best_fft_naive_dft_larger(oracle):
    log_n = 11
    a = oracle.rand_fr(1 << log_n, 5)
    w = oracle.omega(log_n)
    assert np.array_equal(oracle.best_fft(a, w, log_n), oracle.naive_dft(a, w))


def test_fft_kats(oracle):
    log_n = 10
    n = 1 << log_n
    w = oracle.omega(log_n)
    one = oracle.to_mont(1)
    delta = np.zeros((n, 4), np.uint64)
    delta[0] = one
    assert np.all(oracle.best_fft(delta, w, log_n) == one)          # NTT(delta_0) = all ones
    ones = np.tile(one, (n, 1))
    out = oracle.best_fft(ones, w, log_n)                            # NTT(1) = n * delta_0
    assert oracle.from_mont(out[0]) == n and not out[1:].any()


def test_ifft_roundtrip(oracle):
    log_n = 12
    n = 1 << log_n
    a = oracle.rand_fr(n, 9)
    w = oracle.omega(log_n)
    w_inv = oracle.inv(w)
    d = oracle.inv(oracle.to_mont(n))
    assert np.array_equal(oracle.ifft(oracle.best_fft(a, w, log_n), w_inv, log_n, d), a)


def test_distribute_powers(oracle):
    a = oracle.rand_fr(37, 3)
    c = oracle.to_mont(7)
    out = oracle.distribute_powers(a, c)
    for i in range(37):
        assert B.mont_to_int(out[i]) == B.mont_to_int(a[i]) * pow(7, i, B.R_MOD) % B.R_MOD


def test_coeff_to_extended_matches_parts(oracle):
    """zero-padded 2^(k+2) coset NTT == 4 coset parts c_j = g w_ext^j, interleaved
    (the reference's parallel_coeff_to_extended_part_api formulation, fft.cu:572-576)."""
    k, e = 6, 2
    n, N = 1 << k, 1 << (k + e)
    a = oracle.rand_fr(n, 11)
    g = oracle.to_mont(7)
    w_ext = oracle.omega(k + e)
    ext = oracle.coeff_to_extended(a, k, k + e, g, w_ext)
    w = oracle.omega(k)
    for j in range(1 << e):
        c = oracle.mul(g, oracle.pow_(w_ext, j))
        part = oracle.best_fft(oracle.distribute_powers(a, c), w, k)
        assert np.array_equal(part, ext[j::1 << e])
    assert ext.shape == (N, 4)


def test_extended_to_coeff_inverts_coeff_to_extended(oracle):
    """extended_to_coeff(coeff_to_extended(a)) == a zero-padded, and the
    truncation keeps the first m coefficients"""
    k, e = 7, 2
    n, N = 1 << k, 1 << (k + e)
    a = oracle.rand_fr(n, 12)
    g = oracle.to_mont(7)
    w_ext = oracle.omega(k + e)
    ext = oracle.coeff_to_extended(a, k, k + e, g, w_ext)
    d = oracle.inv(oracle.to_mont(N))
    back = oracle.extended_to_coeff(ext, k + e, N, oracle.inv(w_ext), d, oracle.inv(g))
    assert np.array_equal(back[:n], a)
    assert not back[n:].any()
    part = oracle.extended_to_coeff(ext, k + e, n + 3, oracle.inv(w_ext), d, oracle.inv(g))
    assert np.array_equal(part, back[: n + 3])


def test_twiddle_lut(oracle):
    # halo2 generate_twiddle_lookup_table(w, k, 10, true): w^i (i<1024) ++ w^(1024 h)
    k = 14
    w = oracle.omega(k)
    lut = oracle.twiddle_lut(w, k, 10, True)
    assert lut.shape[0] == 1024 + (1 << (k - 10))
    wi = B.mont_to_int(w)
    for i in (0, 1, 5, 1023):
        assert B.mont_to_int(lut[i]) == pow(wi, i, B.R_MOD)
    for h in (0, 1, 15):
        assert B.mont_to_int(lut[1024 + h]) == pow(wi, 1024 * h, B.R_MOD)
    assert oracle.twiddle_lut(oracle.omega(8), 8).shape[0] == 256   # dense table when k <= 10


def test_generator_and_order(oracle):
    G = oracle.g1_generator()
    assert oracle.g1_on_curve(G)
    r_minus_1 = oracle.to_mont(B.R_MOD - 1)
    neg = oracle.g1_scalar_mul(G, r_minus_1)                        # [r-1]G = -G
    assert not oracle.g1_add(neg, G).any()                           # [r]G = O (identity (0,0))


def test_bases_and_msm_vs_bigint(oracle):
    n = 24
    s = oracle.rand_fr(n, 3)
    pts, k = oracle.rand_bases(n, 5, with_dlog=True)
    for i in range(n):
        assert oracle.g1_on_curve(pts[i])
    for i in range(3):
        assert B.limbs_to_point(pts[i]) == B.g1_mul((1, 2), B.mont_to_int(k[i]))
    ref = B.msm([B.mont_to_int(v) for v in s], [B.limbs_to_point(p) for p in pts])
    assert B.limbs_to_point(oracle.multiexp(s, pts)) == ref
    assert B.limbs_to_point(oracle.naive_msm(s, pts)) == ref
    assert B.limbs_to_point(oracle.msm_by_dlog(s, k)) == ref


@pytest.mark.parametrize("n", [0, 1, 3, 31, 33, 257, 1000])
def test_multiexp_edge_sizes(oracle, n):
    s = oracle.rand_fr(n, 7)
    pts, k = oracle.rand_bases(n, 8, with_dlog=True)
    assert np.array_equal(oracle.multiexp(s, pts), oracle.msm_by_dlog(s, k))


def test_multiexp_identity_and_cancellation(oracle):
    pts, k = oracle.rand_bases(8, 2, with_dlog=True)
    zero = np.zeros((8, 4), np.uint64)
    assert not oracle.multiexp(zero, pts).any()
    # P + (-P) = O : scalars 1 and r-1 on the same base
    s = np.stack([oracle.to_mont(1), oracle.to_mont(B.R_MOD - 1)])
    two = np.stack([pts[0], pts[0]])
    assert not oracle.multiexp(s, two).any()
    # identity base (0, 0) contributes nothing
    pts2 = pts.copy()
    pts2[3] = 0
    s = oracle.rand_fr(8, 4)
    k2 = k.copy()
    k2[3] = 0
    assert np.array_equal(oracle.multiexp(s, pts2), oracle.msm_by_dlog(s, k2))


def test_small_scalars(oracle):
    n = 500
    s = oracle.rand_fr_small(n, 1, bits=16)
    for v in s[:10]:
        assert oracle.from_mont(v) < 2**16
    pts, k = oracle.rand_bases(n, 2, with_dlog=True)
    assert np.array_equal(oracle.multiexp(s, pts), oracle.msm_by_dlog(s, k))


def test_elementwise_vector_ops_vs_bigint(oracle):
    n = 64
    a, b = oracle.rand_fr(n, 21), oracle.rand_fr(n, 22)
    c = oracle.to_mont(99991)
    R = B.R_MOD

    def val(x):
        return oracle.from_mont(x)

    s, d, m, ax = oracle.add_vec(a, b), oracle.sub_vec(a, b), oracle.mul_vec(a, b), oracle.axpy_vec(a, c, b)
    for i in range(n):
        x, y = val(a[i]), val(b[i])
        assert val(s[i]) == (x + y) % R
        assert val(d[i]) == (x - y) % R
        assert val(m[i]) == x * y % R
        assert val(ax[i]) == (x * 99991 + y) % R


@pytest.mark.parametrize("k,e", [(2, 1), (4, 2), (5, 3)])
def test_divide_by_vanishing_vs_direct_evaluation(oracle, k, e):
    """ext[i] / ((g w^i)^n - 1), with the denominator evaluated directly in bigint"""
    R = B.R_MOD
    N = 1 << (k + e)
    ext = oracle.rand_fr(N, 31 + k)
    g = 7
    w = oracle.from_mont(oracle.omega(k + e))
    out = oracle.divide_by_vanishing(ext, k, k + e, oracle.to_mont(g), oracle.omega(k + e))
    for i in range(N):
        t = (pow(g * pow(w, i, R) % R, 1 << k, R) - 1) % R
        assert oracle.from_mont(out[i]) == oracle.from_mont(ext[i]) * pow(t, -1, R) % R
    with pytest.raises(ValueError):
        oracle.divide_by_vanishing(ext, k, k + e, oracle.to_mont(1), oracle.omega(k + e))
