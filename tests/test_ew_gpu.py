"""GPU: element-wise extended-domain ops and the division by the vanishing
polynomial (zkgpu_ew_dev, zkgpu_divide_by_vanishing_dev) through the C ABI,
bit-exact against the oracle (halo2's Polynomial Mul/Add/Sub/scalar Mul and
EvaluationDomain::divide_by_vanishing_poly), 2^0 .. 2^20 and one 2^26 case."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def _inputs(oracle, n, seed):
    a = oracle.rand_fr(n, seed)
    b = oracle.rand_fr(n, seed + 1)
    # edge values at the front: 0, 1, p - 1, (p - 1) / 2 in Montgomery form
    edges = [oracle.to_mont(v) for v in (0, 1, R_MOD - 1, (R_MOD - 1) // 2)]
    for i, e in enumerate(edges[: min(n, 4)]):
        a[i] = e
        b[(i + 1) % n] = e
    return a, b


@pytest.mark.parametrize("n", [0, 1, 5, 1000, 1 << 10, 1 << 14, (1 << 20) + 3])
def test_ew_ops_match_oracle(zk, oracle, n):
    torch = pytest.importorskip("torch")
    if n == 0:
        t = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
        rc = zk.lib().zkgpu_ew_dev(0, zk.EW_ADD, t.data_ptr(), t.data_ptr(), t.data_ptr(), None, 0, None)
        assert rc == 0
        return
    a, b = _inputs(oracle, n, 40 + n % 97)
    c = oracle.to_mont(123456789123456789)
    da, db = _dev(torch, a), _dev(torch, b)
    want = {
        zk.EW_MUL: oracle.mul_vec(a, b),
        zk.EW_ADD: oracle.add_vec(a, b),
        zk.EW_SUB: oracle.sub_vec(a, b),
        zk.EW_SCALE: oracle.axpy_vec(a, c),
        zk.EW_AXPY: oracle.axpy_vec(a, c, b),
    }
    for op, ref in want.items():
        out = torch.empty_like(da)
        zk.ew_dev(op, out, da, db if op != zk.EW_SCALE else None, c if op in (zk.EW_SCALE, zk.EW_AXPY) else None)
        torch.cuda.synchronize()
        assert np.array_equal(_host(out), ref), f"op {op}, n {n}"
    # in place (out aliases a), as halo2's h = h * y + e accumulation uses it
    acc = da.clone()
    zk.ew_dev(zk.EW_AXPY, acc, acc, db, c)
    torch.cuda.synchronize()
    assert np.array_equal(_host(acc), want[zk.EW_AXPY])


def test_ew_rejects_bad_arguments(zk, oracle):
    torch = pytest.importorskip("torch")
    t = torch.zeros((8, 4), dtype=torch.int64, device="cuda")
    bad_c = np.array([2**64 - 1] * 4, dtype=np.uint64)  # not canonical
    L = zk.lib()
    assert L.zkgpu_ew_dev(0, 9, t.data_ptr(), t.data_ptr(), t.data_ptr(), None, 8, None) == zk.EINVAL
    assert L.zkgpu_ew_dev(0, zk.EW_MUL, t.data_ptr(), t.data_ptr(), None, None, 8, None) == zk.EINVAL
    assert L.zkgpu_ew_dev(0, zk.EW_SCALE, t.data_ptr(), t.data_ptr(), None, None, 8, None) == zk.EINVAL
    assert L.zkgpu_ew_dev(0, zk.EW_SCALE, t.data_ptr(), t.data_ptr(), None, bad_c.ctypes.data, 8, None) == zk.EINVAL


@pytest.mark.parametrize("k,e", [(3, 1), (10, 2), (12, 3), (16, 2), (18, 6)])
def test_divide_by_vanishing_matches_oracle(zk, oracle, k, e):
    torch = pytest.importorskip("torch")
    N = 1 << (k + e)
    ext = oracle.rand_fr(N, 500 + k + e)
    g, w_ext = oracle.to_mont(7), oracle.omega(k + e)
    d = _dev(torch, ext)
    zk.divide_by_vanishing_dev(d, k, k + e, g, w_ext)
    torch.cuda.synchronize()
    assert np.array_equal(_host(d), oracle.divide_by_vanishing(ext, k, k + e, g, w_ext))


def test_divide_by_vanishing_rejects_vanishing_coset(zk, oracle):
    torch = pytest.importorskip("torch")
    k, e = 8, 2
    d = _dev(torch, oracle.rand_fr(1 << (k + e), 3))
    before = d.clone()
    L = zk.lib()
    one, w = oracle.to_mont(1), oracle.omega(k + e)
    # g = 1: X^n - 1 is zero at X = 1, the coset is the subgroup itself
    assert L.zkgpu_divide_by_vanishing_dev(0, d.data_ptr(), k, k + e, one.ctypes.data, w.ctypes.data, None) == zk.EINVAL
    # extension factor above 64
    assert L.zkgpu_divide_by_vanishing_dev(0, d.data_ptr(), 3, 10, oracle.to_mont(7).ctypes.data,
                                           oracle.omega(10).ctypes.data, None) == zk.EINVAL
    torch.cuda.synchronize()
    assert torch.equal(d, before)


def test_quotient_step_composition(zk, oracle):
    """A small halo2 quotient step on the device: LDE two polynomials to the
    extended coset, combine h = a * b * y + a, divide by X^n - 1 there and
    return to coefficients; against the same composition on the oracle."""
    torch = pytest.importorskip("torch")
    k, e = 12, 2
    n, N = 1 << k, 1 << (k + e)
    w, we = oracle.omega(k), oracle.omega(k + e)
    wi, wei = oracle.inv(w), oracle.inv(we)
    dk, dN = oracle.inv(oracle.to_mont(n)), oracle.inv(oracle.to_mont(N))
    g = oracle.to_mont(7)
    gi = oracle.inv(g)
    y = oracle.to_mont(987654321)
    va, vb = oracle.rand_fr(n, 11), oracle.rand_fr(n, 12)
    ea = oracle.coeff_to_extended(oracle.ifft(va, wi, k, dk), k, k + e, g, we)
    eb = oracle.coeff_to_extended(oracle.ifft(vb, wi, k, dk), k, k + e, g, we)
    h = oracle.axpy_vec(oracle.mul_vec(ea, eb), y, ea)
    h = oracle.divide_by_vanishing(h, k, k + e, g, we)
    want = oracle.extended_to_coeff(h, k + e, N, wei, dN, gi)

    dva, dvb = _dev(torch, va), _dev(torch, vb)
    da = torch.empty((N, 4), dtype=torch.int64, device="cuda")
    db = torch.empty_like(da)
    zk.lagrange_to_extended_dev(dva, da, k, k + e, wi, dk, g, we)
    zk.lagrange_to_extended_dev(dvb, db, k, k + e, wi, dk, g, we)
    dh = torch.empty_like(da)
    zk.ew_dev(zk.EW_MUL, dh, da, db)
    zk.ew_dev(zk.EW_AXPY, dh, dh, da, y)
    zk.divide_by_vanishing_dev(dh, k, k + e, g, we)
    out = torch.empty_like(da)
    zk.extended_to_coeff_dev(dh, out, k + e, wei, dN, gi)
    torch.cuda.synchronize()
    assert np.array_equal(_host(out), want)


def test_full_size_2p26_axpy_and_vanishing(zk, oracle):
    """One extended-domain vector of 2^26 (the LDE output size of 2^24 -> 2^26):
    h = a * y + b, then / (X^(2^24) - 1) on the coset 7<w_ext>, bit-exact."""
    torch = pytest.importorskip("torch")
    k, e = 24, 2
    N = 1 << (k + e)
    a = oracle.rand_fr(N, 2601)
    b = oracle.rand_fr(N, 2602)
    y = oracle.to_mont(31337)
    g, we = oracle.to_mont(7), oracle.omega(k + e)
    want = oracle.divide_by_vanishing(oracle.axpy_vec(a, y, b), k, k + e, g, we)
    da, db = _dev(torch, a), _dev(torch, b)
    del a, b
    zk.ew_dev(zk.EW_AXPY, da, da, db, y)
    del db
    zk.divide_by_vanishing_dev(da, k, k + e, g, we)
    torch.cuda.synchronize()
    assert np.array_equal(_host(da), want)
