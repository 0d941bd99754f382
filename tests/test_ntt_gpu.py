"""GPU parity: the sm_100a NTT through the C ABI against the CPU oracle
(bit-exact), at every plan shape (1..4 passes), plus size-independent
properties at the full benchmark sizes."""
import numpy as np
import pytest

from oracle import bigref as B

pytestmark = pytest.mark.gpu


def inv_n(oracle, log_n):
    return oracle.inv(oracle.to_mont(1 << log_n))


def test_self_test(zk):
    assert zk.do_fft_ffi(0) == 0


@pytest.mark.parametrize("field", ["fr", "fq"])
def test_field_ops(zk, oracle, field):
    fid = oracle.FR if field == "fr" else oracle.FQ
    p = B.R_MOD if field == "fr" else B.Q_MOD
    n = 4096
    a = oracle.rand_fr(n, 1)   # < r < q: valid in both fields
    b = oracle.rand_fr(n, 2)
    edge = [0, 1, 2, p - 1, p - 2, (p - 1) // 2, (p + 1) // 2, 2**255 % p, 2**128 + 1]
    for i, v in enumerate(edge):
        a[i] = oracle.from_int(v)
        b[len(edge) - 1 - i] = oracle.from_int(v)
        a[len(edge) + i] = oracle.from_int(v)
        b[len(edge) + i] = oracle.from_int(v)
    for op, fn in (("mul", oracle.mul), ("add", oracle.add), ("sub", oracle.sub)):
        got = zk.field_op(op, a, b, field)
        ref = np.stack([fn(a[i], b[i], fid) for i in range(n)])
        assert np.array_equal(got, ref), op


@pytest.mark.parametrize("log_n", list(range(0, 21)))
def test_fft_all_plans(zk, oracle, log_n):
    n = 1 << log_n
    a = oracle.rand_fr(n, 1000 + log_n)
    w = oracle.omega(log_n)
    got = zk.fft(a, w, log_n)
    assert np.array_equal(got, oracle.best_fft(a, w, log_n))


@pytest.mark.parametrize("log_n", [10, 16, 22])
def test_reference_api_fft(zk, oracle, log_n):
    """parallel_fft_api with the halo2 twiddle table, as the reference caller passes it."""
    n = 1 << log_n
    a = oracle.rand_fr(n, 7 + log_n)
    w = oracle.omega(log_n)
    tw = oracle.twiddle_lut(w, log_n, 10, True)
    ref = oracle.best_fft(a, w, log_n)
    assert zk.parallel_fft_api(0, a, w, tw, n, log_n, tw.shape[0]) == 0
    assert np.array_equal(a, ref)


@pytest.mark.parametrize("log_n", [3, 12, 13, 19])
def test_reference_api_ifft(zk, oracle, log_n):
    n = 1 << log_n
    a = oracle.rand_fr(n, 70 + log_n)
    w_inv = oracle.inv(oracle.omega(log_n))
    d = inv_n(oracle, log_n)
    tw = oracle.twiddle_lut(w_inv, log_n, 10, True)
    ref = oracle.ifft(a, w_inv, log_n, d)
    assert zk.parallel_ifft_api(0, a, w_inv, tw, n, log_n, tw.shape[0], d) == 0
    assert np.array_equal(a, ref)


@pytest.mark.parametrize("log_n", [2, 5, 12, 14, 20])
def test_reference_api_coset_part(zk, oracle, log_n):
    """parallel_coeff_to_extended_part_api: a[i] *= c^i then fft (fft.cu:223-232)."""
    n = 1 << log_n
    a = oracle.rand_fr(n, 30 + log_n)
    w = oracle.omega(log_n)
    c = oracle.mul(oracle.to_mont(7), oracle.omega(log_n + 2))
    ref = oracle.best_fft(oracle.distribute_powers(a, c), w, log_n)
    assert zk.parallel_coeff_to_extended_part_api(0, a, w, None, n, log_n, 0, c) == 0
    assert np.array_equal(a, ref)


@pytest.mark.parametrize("k,e", [(3, 1), (8, 2), (12, 2), (16, 2)])
def test_lagrange_to_extended(zk, oracle, k, e):
    n = 1 << k
    vals = oracle.rand_fr(n, 50 + k)
    w_inv, d = oracle.inv(oracle.omega(k)), inv_n(oracle, k)
    g, w_ext = oracle.to_mont(7), oracle.omega(k + e)
    coeffs = oracle.ifft(vals, w_inv, k, d)
    ref = oracle.coeff_to_extended(coeffs, k, k + e, g, w_ext)
    got = zk.lagrange_to_extended(vals, k, k + e, w_inv, d, g, w_ext)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("log_ext,m", [(0, 1), (1, 2), (2, 3), (3, 8), (10, 700), (14, 12345), (18, 1 << 18)])
def test_extended_to_coeff(zk, oracle, log_ext, m):
    """inverse LDE (ifft on the extended domain, times 7^-i, truncate) vs the oracle"""
    N = 1 << log_ext
    ext = oracle.rand_fr(N, 60 + log_ext)
    w_inv, d = oracle.inv(oracle.omega(log_ext)), inv_n(oracle, log_ext)
    g_inv = oracle.inv(oracle.to_mont(7))
    ref = oracle.extended_to_coeff(ext, log_ext, m, w_inv, d, g_inv)
    got = zk.extended_to_coeff(ext, log_ext, m, w_inv, d, g_inv)
    assert np.array_equal(got, ref)


def test_extended_to_coeff_invalid(zk, oracle):
    ext = oracle.rand_fr(1 << 10, 1)
    w_inv, d, g_inv = oracle.inv(oracle.omega(10)), inv_n(oracle, 10), oracle.inv(oracle.to_mont(7))
    with pytest.raises(zk.ZkGpuError):
        zk.extended_to_coeff(ext, 10, (1 << 10) + 1, w_inv, d, g_inv)   # m beyond the domain
    with pytest.raises(zk.ZkGpuError):
        zk.extended_to_coeff(ext, 10, 16, oracle.inv(oracle.omega(9)), d, g_inv)   # wrong root order


def test_lde_inverse_roundtrip_2p24(zk, oracle):
    """size-independent property at the benchmark size: lagrange 2^24 -> coset
    extended 2^26 -> coefficients (truncated to 2^24) -> fft gives the values
    back, and the truncated-away coefficients are all zero"""
    torch = pytest.importorskip("torch")
    k, e = 24, 2
    vals = oracle.rand_fr(1 << k, 424)
    w, w_ext = oracle.omega(k), oracle.omega(k + e)
    c = dict(omega_inv=oracle.inv(w), divisor=inv_n(oracle, k), g=oracle.to_mont(7), omega_ext=w_ext)
    d_vals = torch.from_numpy(vals.view(np.int64)).cuda()
    d_ext = torch.empty(((1 << (k + e)), 4), dtype=torch.int64, device="cuda")
    zk.lagrange_to_extended_dev(d_vals, d_ext, k, k + e, c["omega_inv"], c["divisor"], c["g"], c["omega_ext"])
    d_co = torch.empty(((1 << (k + e)), 4), dtype=torch.int64, device="cuda")
    zk.extended_to_coeff_dev(d_ext, d_co, k + e, oracle.inv(w_ext), inv_n(oracle, k + e),
                             oracle.inv(oracle.to_mont(7)))
    del d_ext
    assert not d_co[1 << k:].any().item()
    zk.ntt_dev(d_co[: 1 << k], k, w)
    torch.cuda.synchronize()
    assert torch.equal(d_co[: 1 << k], d_vals)


def test_edge_inputs(zk, oracle):
    log_n = 14
    n = 1 << log_n
    w = oracle.omega(log_n)
    zero = np.zeros((n, 4), np.uint64)
    assert not zk.fft(zero, w, log_n).any()
    one = oracle.to_mont(1)
    delta = zero.copy()
    delta[0] = one
    assert np.array_equal(zk.fft(delta, w, log_n), np.tile(one, (n, 1)))
    top = np.tile(oracle.from_int(B.R_MOD - 1), (n, 1))          # every element p - 1
    assert np.array_equal(zk.fft(top, w, log_n), oracle.best_fft(top, w, log_n))


def test_invalid_omega_rejected(zk, oracle):
    a = oracle.rand_fr(1 << 10, 1)
    before = a.copy()
    w_bad = oracle.omega(11)   # order 2^11, not 2^10
    assert zk.parallel_fft_api(0, a, w_bad, None, 1 << 10, 10, 0) == zk.EINVAL
    assert np.array_equal(a, before)


def test_full_size_fft_2p24(zk, oracle):
    """the 2^24 transform, bit-exact against the oracle"""
    log_n = 24
    a = oracle.rand_fr(1 << log_n, 24)
    w = oracle.omega(log_n)
    assert np.array_equal(zk.fft(a, w, log_n), oracle.best_fft(a, w, log_n))


def test_full_size_lde_2p24_to_2p26(zk, oracle):
    """the benchmark workload (lagrange 2^24 -> coset extended 2^26), bit-exact"""
    k, e = 24, 2
    vals = oracle.rand_fr(1 << k, 2024)
    w_inv, d = oracle.inv(oracle.omega(k)), inv_n(oracle, k)
    g, w_ext = oracle.to_mont(7), oracle.omega(k + e)
    got = zk.lagrange_to_extended(vals, k, k + e, w_inv, d, g, w_ext)
    ref = oracle.coeff_to_extended(oracle.ifft(vals, w_inv, k, d), k, k + e, g, w_ext)
    assert np.array_equal(got, ref)


def test_roundtrip_2p26(zk, oracle):
    """size-independent property at 2^26: ifft(fft(a)) == a"""
    log_n = 26
    a = oracle.rand_fr(1 << log_n, 26)
    w = oracle.omega(log_n)
    f = zk.fft(a, w, log_n)
    back = zk.ifft(f, oracle.inv(w), log_n, inv_n(oracle, log_n))
    assert np.array_equal(back, a)


def test_device_api_matches_host_api(zk, oracle):
    torch = pytest.importorskip("torch")
    log_n = 18
    a = oracle.rand_fr(1 << log_n, 18)
    w = oracle.omega(log_n)
    t = torch.from_numpy(a.view(np.int64)).cuda()
    zk.ntt_dev(t, log_n, w, coset=oracle.to_mont(5), post_scale=oracle.to_mont(3))
    torch.cuda.synchronize()
    got = t.cpu().numpy().view(np.uint64)
    ref = oracle.best_fft(oracle.distribute_powers(a, oracle.to_mont(5)), w, log_n)
    ref = oracle.mul_vec(ref, np.tile(oracle.to_mont(3), (1 << log_n, 1)))
    assert np.array_equal(got, ref)
