"""ctypes wrapper over the CPU oracle (oracle/libzkoracle.so).

TEST INFRASTRUCTURE ONLY: the checker for tests, ``__graft_entry__.smoke()``
and the benchmark's CPU-baseline leg.  The product library never imports it.

Arrays are numpy ``uint64`` with a trailing dimension of 4 (one Fr/Fq element,
4 x u64 little-endian Montgomery limbs) or 8 (one affine G1 point x, y).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libzkoracle.so")
_lib = None

FR, FQ = 0, 1
R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
Q_MOD = 21888242871839275222246405745257275088696311157297823662689037894645226208583


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    src = os.path.join(_HERE, "zkoracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        u32, u64, i32, sz = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_size_t
        sig = {
            "zko_field_mul": (None, [i32, P, P, P]),
            "zko_field_add": (None, [i32, P, P, P]),
            "zko_field_sub": (None, [i32, P, P, P]),
            "zko_field_pow": (None, [i32, P, P, P]),
            "zko_field_inv": (None, [i32, P, P]),
            "zko_to_mont": (None, [i32, P, P]),
            "zko_from_mont": (None, [i32, P, P]),
            "zko_field_mul_vec": (None, [i32, P, P, P, sz, i32]),
            "zko_field_dot": (None, [i32, P, P, P, sz, i32]),
            "zko_field_add_vec": (None, [i32, P, P, P, sz, i32]),
            "zko_field_sub_vec": (None, [i32, P, P, P, sz, i32]),
            "zko_field_axpy_vec": (None, [i32, P, P, P, P, sz, i32]),
            "zko_divide_by_vanishing": (i32, [P, u32, u32, P, P, i32]),
            "zko_rand_fr": (None, [P, sz, u64, sz, i32]),
            "zko_rand_fr_small": (None, [P, sz, u64, sz, i32, i32]),
            "zko_rand_bases": (None, [P, P, sz, u64, sz, i32]),
            "zko_best_fft": (i32, [P, P, u32, i32]),
            "zko_ifft": (i32, [P, P, u32, P, i32]),
            "zko_distribute_powers": (i32, [P, sz, P, i32]),
            "zko_coeff_to_extended": (i32, [P, u32, P, u32, P, P, i32]),
            "zko_twiddle_lut": (sz, [P, P, u32, u32, i32]),
            "zko_omega": (i32, [P, u32]),
            "zko_naive_dft": (i32, [P, P, sz, P]),
            "zko_g1_normalize": (None, [P, P]),
            "zko_g1_scalar_mul": (None, [P, P, P]),
            "zko_g1_add_affine": (None, [P, P, P]),
            "zko_g1_on_curve": (i32, [P]),
            "zko_multiexp": (i32, [P, P, P, sz, i32]),
            "zko_naive_msm": (i32, [P, P, P, sz]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], "need C-contiguous uint64"
    return a.ctypes.data


def _e(x) -> np.ndarray:
    """A single element as a (4,) uint64 array (from an int = raw limbs, or array)."""
    if isinstance(x, (int, np.integer)):
        x = int(x)
        return np.array([(x >> (64 * i)) & (2**64 - 1) for i in range(4)], dtype=np.uint64)
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint64).reshape(4))


def to_int(limbs) -> int:
    limbs = np.asarray(limbs, dtype=np.uint64).reshape(-1)
    return sum(int(v) << (64 * i) for i, v in enumerate(limbs))


def from_int(x: int, words: int = 4) -> np.ndarray:
    return np.array([(x >> (64 * i)) & (2**64 - 1) for i in range(words)], dtype=np.uint64)


# ---- field ----------------------------------------------------------------
def mul(a, b, fid=FR):
    out = np.zeros(4, np.uint64)
    a, b = _e(a), _e(b)
    lib().zko_field_mul(fid, _p(out), _p(a), _p(b))
    return out


def add(a, b, fid=FR):
    out = np.zeros(4, np.uint64)
    a, b = _e(a), _e(b)
    lib().zko_field_add(fid, _p(out), _p(a), _p(b))
    return out


def sub(a, b, fid=FR):
    out = np.zeros(4, np.uint64)
    a, b = _e(a), _e(b)
    lib().zko_field_sub(fid, _p(out), _p(a), _p(b))
    return out


def pow_(a, e: int, fid=FR):
    out = np.zeros(4, np.uint64)
    a, ee = _e(a), from_int(e)
    lib().zko_field_pow(fid, _p(out), _p(a), _p(ee))
    return out


def inv(a, fid=FR):
    out = np.zeros(4, np.uint64)
    a = _e(a)
    lib().zko_field_inv(fid, _p(out), _p(a))
    return out


def to_mont(c: int, fid=FR) -> np.ndarray:
    out = np.zeros(4, np.uint64)
    cc = from_int(c % (R_MOD if fid == FR else Q_MOD))
    lib().zko_to_mont(fid, _p(out), _p(cc))
    return out


def from_mont(m, fid=FR) -> int:
    out = np.zeros(4, np.uint64)
    m = _e(m)
    lib().zko_from_mont(fid, _p(out), _p(m))
    return to_int(out)


def mul_vec(a: np.ndarray, b: np.ndarray, fid=FR, threads=0) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.empty_like(a)
    lib().zko_field_mul_vec(fid, _p(out), _p(a), _p(b), a.shape[0], threads)
    return out


def add_vec(a: np.ndarray, b: np.ndarray, fid=FR, threads=0) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.empty_like(a)
    lib().zko_field_add_vec(fid, _p(out), _p(a), _p(b), a.shape[0], threads)
    return out


def sub_vec(a: np.ndarray, b: np.ndarray, fid=FR, threads=0) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.empty_like(a)
    lib().zko_field_sub_vec(fid, _p(out), _p(a), _p(b), a.shape[0], threads)
    return out


def axpy_vec(a: np.ndarray, c, b=None, fid=FR, threads=0) -> np.ndarray:
    """a * c (+ b): c one element, a and b vectors"""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    cc = _e(c)
    out = np.empty_like(a)
    bp = None
    if b is not None:
        b = np.ascontiguousarray(b, dtype=np.uint64)
        bp = _p(b)
    lib().zko_field_axpy_vec(fid, _p(out), _p(a), _p(cc), bp, a.shape[0], threads)
    return out


def divide_by_vanishing(ext: np.ndarray, log_n: int, log_ext: int, g, w_ext, threads: int = 0) -> np.ndarray:
    """halo2 EvaluationDomain::divide_by_vanishing_poly over the coset g<w_ext>
    (returns a new array; raises if X^n - 1 vanishes somewhere on the coset)"""
    out = np.array(ext, dtype=np.uint64, copy=True, order="C")
    gg, w = _e(g), _e(w_ext)
    if lib().zko_divide_by_vanishing(_p(out), log_n, log_ext, _p(gg), _p(w), threads) != 0:
        raise ValueError("X^n - 1 vanishes on this coset")
    return out


# ---- inputs ---------------------------------------------------------------
def rand_fr(n: int, seed: int, start: int = 0, threads: int = 0) -> np.ndarray:
    out = np.empty((n, 4), np.uint64)
    lib().zko_rand_fr(_p(out), n, seed, start, threads)
    return out


def rand_fr_small(n: int, seed: int, bits: int = 16, start: int = 0, threads: int = 0) -> np.ndarray:
    out = np.empty((n, 4), np.uint64)
    lib().zko_rand_fr_small(_p(out), n, seed, start, bits, threads)
    return out


def rand_bases(n: int, seed: int, start: int = 0, threads: int = 0, with_dlog: bool = False):
    out = np.empty((n, 8), np.uint64)
    k = np.empty((n, 4), np.uint64) if with_dlog else None
    lib().zko_rand_bases(_p(out), _p(k) if with_dlog else None, n, seed, start, threads)
    return (out, k) if with_dlog else out


# ---- NTT ------------------------------------------------------------------
def omega(log_n: int) -> np.ndarray:
    out = np.zeros(4, np.uint64)
    assert lib().zko_omega(_p(out), log_n) == 0
    return out


def best_fft(a: np.ndarray, w, log_n: int, threads: int = 0) -> np.ndarray:
    a = np.array(a, dtype=np.uint64, copy=True, order="C")
    assert a.shape == (1 << log_n, 4)
    w = _e(w)
    assert lib().zko_best_fft(_p(a), _p(w), log_n, threads) == 0
    return a


def ifft(a: np.ndarray, w_inv, log_n: int, divisor, threads: int = 0) -> np.ndarray:
    a = np.array(a, dtype=np.uint64, copy=True, order="C")
    w, d = _e(w_inv), _e(divisor)
    assert lib().zko_ifft(_p(a), _p(w), log_n, _p(d), threads) == 0
    return a


def distribute_powers(a: np.ndarray, c, threads: int = 0) -> np.ndarray:
    a = np.array(a, dtype=np.uint64, copy=True, order="C")
    c = _e(c)
    assert lib().zko_distribute_powers(_p(a), a.shape[0], _p(c), threads) == 0
    return a


def coeff_to_extended(a: np.ndarray, log_n: int, log_ext: int, g, w_ext, threads: int = 0) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    ext = np.empty((1 << log_ext, 4), np.uint64)
    g, w = _e(g), _e(w_ext)
    assert lib().zko_coeff_to_extended(_p(a), log_n, _p(ext), log_ext, _p(g), _p(w), threads) == 0
    return ext


def extended_to_coeff(ext: np.ndarray, log_ext: int, m: int, w_ext_inv, ext_divisor, g_inv,
                      threads: int = 0) -> np.ndarray:
    """halo2 EvaluationDomain::extended_to_coeff (halo2_proofs/src/poly/domain.rs,
    the external halo2 fork the reference's callers use): ifft over the
    extended domain, distribute powers of g^-1 (undo the coset), truncate to m."""
    a = ifft(ext, w_ext_inv, log_ext, ext_divisor, threads)
    a = distribute_powers(a, g_inv, threads)
    return np.ascontiguousarray(a[:m])


def twiddle_lut(w, log_n: int, sparse_degree: int = 10, with_last_level: bool = True) -> np.ndarray:
    w = _e(w)
    n = lib().zko_twiddle_lut(None, _p(w), log_n, sparse_degree, int(with_last_level))
    out = np.empty((n, 4), np.uint64)
    lib().zko_twiddle_lut(_p(out), _p(w), log_n, sparse_degree, int(with_last_level))
    return out


def naive_dft(a: np.ndarray, w) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    out = np.empty_like(a)
    w = _e(w)
    lib().zko_naive_dft(_p(out), _p(a), a.shape[0], _p(w))
    return out


# ---- G1 -------------------------------------------------------------------
def g1_normalize(jac) -> np.ndarray:
    jac = np.ascontiguousarray(np.asarray(jac, dtype=np.uint64).reshape(12))
    out = np.zeros(8, np.uint64)
    lib().zko_g1_normalize(_p(out), _p(jac))
    return out


def g1_scalar_mul(base_xy, k_mont) -> np.ndarray:
    b = np.ascontiguousarray(np.asarray(base_xy, dtype=np.uint64).reshape(8))
    k = _e(k_mont)
    out = np.zeros(8, np.uint64)
    lib().zko_g1_scalar_mul(_p(out), _p(b), _p(k))
    return out


def g1_add(a_xy, b_xy) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a_xy, dtype=np.uint64).reshape(8))
    b = np.ascontiguousarray(np.asarray(b_xy, dtype=np.uint64).reshape(8))
    out = np.zeros(8, np.uint64)
    lib().zko_g1_add_affine(_p(out), _p(a), _p(b))
    return out


def g1_on_curve(xy) -> bool:
    a = np.ascontiguousarray(np.asarray(xy, dtype=np.uint64).reshape(8))
    return bool(lib().zko_g1_on_curve(_p(a)))


def g1_generator() -> np.ndarray:
    return np.concatenate([to_mont(1, FQ), to_mont(2, FQ)])


def multiexp(scalars: np.ndarray, bases: np.ndarray, threads: int = 0) -> np.ndarray:
    s = np.ascontiguousarray(scalars, dtype=np.uint64)
    b = np.ascontiguousarray(bases, dtype=np.uint64)
    assert s.shape[0] == b.shape[0]
    out = np.zeros(8, np.uint64)
    lib().zko_multiexp(_p(out), _p(s), _p(b), s.shape[0], threads)
    return out


def naive_msm(scalars: np.ndarray, bases: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(scalars, dtype=np.uint64)
    b = np.ascontiguousarray(bases, dtype=np.uint64)
    out = np.zeros(8, np.uint64)
    lib().zko_naive_msm(_p(out), _p(s), _p(b), s.shape[0])
    return out


def field_dot(a: np.ndarray, b: np.ndarray, fid=FR, threads=0) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.zeros(4, np.uint64)
    lib().zko_field_dot(fid, _p(out), _p(a), _p(b), a.shape[0], threads)
    return out


def msm_by_dlog(scalars: np.ndarray, k_mont: np.ndarray, threads: int = 0) -> np.ndarray:
    """sum s_i [k_i] G = [sum s_i k_i] G — a size-independent MSM check when
    the bases' discrete logs k_i are known (bases from rand_bases(with_dlog))."""
    return g1_scalar_mul(g1_generator(), field_dot(scalars, k_mont, FR, threads))
