"""zk_gpu_b200 — B200 (sm_100a) halo2/BN256 NTT + MSM behind a C ABI.

The product is ``libzkgpu.so`` (CUDA kernels + C-ABI, ``include/zkgpu.h``).
This module is the Python host mirror of the reference's FFI surface
(src/api.rs:3-14): the same entry-point names, argument meaning and status
codes, over ``ctypes``.  Arrays are numpy ``uint64`` with a trailing
dimension of 4 (one Fr/Fq element, 4 x u64 little-endian Montgomery limbs)
or 8 (one affine G1 point x, y).  Device-resident variants take torch CUDA
tensors (``torch.uint64`` / ``int64`` storage) and a CUDA stream.

There is no CPU fallback: if the library is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzkgpu.so")

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, EADMIT, ENODEV, EBUSY = range(8)
# BN254 base field modulus and the G1 generator (1, 2) in Montgomery form
FQ_MODULUS = 21888242871839275222246405745257275088696311157297823662689037894645226208583


def _fq_mont_words(x: int) -> list:
    m = (x << 256) % FQ_MODULUS
    return [(m >> (64 * j)) & (2**64 - 1) for j in range(4)]


G1_GENERATOR = np.array(_fq_mont_words(1) + _fq_mont_words(2), dtype=np.uint64)

_STATUS = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "ETIMEOUT", 5: "EADMIT", 6: "ENODEV", 7: "EBUSY"}

_lib = None


class ZkGpuError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        msg = _STATUS.get(int(code), str(code))
        detail = ""
        try:
            detail = lib().zkgpu_last_error().decode()
        except Exception:  # pragma: no cover
            pass
        super().__init__(f"{where}: {msg} {detail}".strip())
        self.code = int(code)


class GpuAffine(ctypes.Structure):
    """src/lib.rs:22-28"""
    _fields_ = [("x", ctypes.c_uint64 * 4), ("y", ctypes.c_uint64 * 4)]


class GpuProjective(ctypes.Structure):
    """src/lib.rs:30-35"""
    _fields_ = [("x", ctypes.c_uint64 * 4), ("y", ctypes.c_uint64 * 4), ("z", ctypes.c_uint64 * 4)]


# name -> (restype, argtypes); exactly the functions include/zkgpu.h declares
P = ctypes.c_void_p
_u64, _u32, _i32, _sz = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_size_t
EXPORTS = {
    "do_fft_ffi": (_u64, [_sz]),
    "parallel_fft_api": (_u64, [_sz, P, P, P, _u64, _u64, _u64]),
    "parallel_ifft_api": (_u64, [_sz, P, P, P, _u64, _u64, _u64, P]),
    "parallel_coeff_to_extended_part_api": (_u64, [_sz, P, P, P, _u64, _u64, _u64, P]),
    "parallel_msm_api": (_u64, [_sz, P, P, _u64, P]),
    "zkgpu_fft": (_i32, [_i32, P, _u32, P]),
    "zkgpu_ifft": (_i32, [_i32, P, _u32, P, P]),
    "zkgpu_coset_fft": (_i32, [_i32, P, _u32, P, P]),
    "zkgpu_msm": (_i32, [_i32, P, P, _u64, P]),
    "zkgpu_lagrange_to_extended": (_i32, [_i32, P, _u32, P, _u32, P, P, P, P]),
    "zkgpu_ntt_dev": (_i32, [_i32, P, _u32, P, P, P, P]),
    "zkgpu_lagrange_to_extended_dev": (_i32, [_i32, P, _u32, P, _u32, P, P, P, P, P]),
    "zkgpu_msm_dev": (_i32, [_i32, P, P, _u64, P, P]),
    "zkgpu_ntt_dev_static": (_i32, [_i32, P, _u32, P, P]),
    "zkgpu_g1_mul_fixed_dev": (_i32, [_i32, P, P, _u64, P, P]),
    "zkgpu_extended_to_coeff": (_i32, [_i32, P, _u32, P, _u64, P, P, P]),
    "zkgpu_autotune": (_i32, [_i32, _u32, _u32, _u32, _u32, P]),
    "zkgpu_tune_set_ntt_plan": (_i32, [_i32, _u32, _u32, P]),
    "zkgpu_tune_get_ntt_plan": (_i32, [_i32, _u32, P, P]),
    "zkgpu_tune_set_msm_window": (_i32, [_i32, _u32, _u32]),
    "zkgpu_tune_get_msm_window": (_i32, [_i32, _u32, P]),
    "zkgpu_tune_save": (_i32, [_i32, ctypes.c_char_p]),
    "zkgpu_tune_load": (_i32, [_i32, ctypes.c_char_p, P]),
    "zkgpu_extended_to_coeff_dev": (_i32, [_i32, P, _u32, P, _u64, P, P, P, P]),
    "zkgpu_ew_dev": (_i32, [_i32, _u32, P, P, P, P, _u64, P]),
    "zkgpu_divide_by_vanishing_dev": (_i32, [_i32, P, _u32, _u32, P, P, P]),
    "zkgpu_ntt_batch_create": (_i32, [_i32, P, _u32, P]),
    "zkgpu_ntt_batch_run": (_i32, [P, P]),
    "zkgpu_ntt_batch_check": (_i32, [P]),
    "zkgpu_ntt_batch_info": (None, [P, P, P, P]),
    "zkgpu_ntt_batch_destroy": (None, [P]),
    "zkgpu_selftest_wait_timeout": (_i32, [_i32, P, _u32]),
    "zkgpu_job_footprint": (_u64, [P]),
    "zkgpu_admission_simulate": (_u64, [_u64, P, _u32, P]),
    "zkgpu_server_create": (_i32, [_i32, _u64, _u32, P]),
    "zkgpu_server_add_bases": (_i32, [P, P, _u64, P]),
    "zkgpu_server_submit": (_i32, [P, P, P]),
    "zkgpu_server_wait": (_i32, [P, _u64, _u32, P]),
    "zkgpu_server_stats_get": (_i32, [P, P]),
    "zkgpu_server_destroy": (None, [P]),
    "zkgpu_field_op": (_i32, [_i32, _i32, _i32, P, P, P, _u64]),
    "zkgpu_release_cached": (_i32, [_i32]),
    "zkgpu_last_error": (ctypes.c_char_p, []),
    "zkgpu_launch_count": (_u64, [_i32]),
    "zkgpu_version": (ctypes.c_char_p, []),
    "zkgpu_int_peak": (_i32, [_i32, _u32, P, P]),
    "zkgpu_prof_enable": (None, [_i32]),
    "zkgpu_prof_reset": (None, []),
    "zkgpu_prof_read": (_i32, [ctypes.c_char_p, _u64]),
}


def lib():
    """Load libzkgpu.so (built in-tree by zk_gpu_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m zk_gpu_b200.build` (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _arr(a, words=4) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    assert a.ndim >= 1 and a.shape[-1] == words, f"expected trailing dimension {words}"
    return a


def _el(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint64).reshape(4))


def _check(code: int, where: str):
    if int(code) != 0:
        raise ZkGpuError(int(code), where)


# ---------------------------------------------------------------------------
# reference-compatible entry points (src/api.rs:3-14), raw status returned
# ---------------------------------------------------------------------------
def do_fft_ffi(device_id: int = 0) -> int:
    return int(lib().do_fft_ffi(device_id))


def parallel_fft_api(device_id: int, req: np.ndarray, omega, twiddle, n: int, log_n: int, twiddle_size: int) -> int:
    """In place on ``req`` ((n, 4) uint64, C-contiguous)."""
    tw = None if twiddle is None else _arr(twiddle).ctypes.data
    return int(lib().parallel_fft_api(device_id, req.ctypes.data, _el(omega).ctypes.data, tw, n, log_n, twiddle_size))


def parallel_ifft_api(device_id: int, req: np.ndarray, omega, twiddle, n: int, log_n: int, twiddle_size: int,
                      divisor) -> int:
    tw = None if twiddle is None else _arr(twiddle).ctypes.data
    return int(lib().parallel_ifft_api(device_id, req.ctypes.data, _el(omega).ctypes.data, tw, n, log_n,
                                       twiddle_size, _el(divisor).ctypes.data))


def parallel_coeff_to_extended_part_api(device_id: int, req: np.ndarray, omega, twiddle, n: int, log_n: int,
                                        twiddle_size: int, c) -> int:
    tw = None if twiddle is None else _arr(twiddle).ctypes.data
    return int(lib().parallel_coeff_to_extended_part_api(device_id, req.ctypes.data, _el(omega).ctypes.data, tw, n,
                                                         log_n, twiddle_size, _el(c).ctypes.data))


def parallel_msm_api(device_id: int, data: np.ndarray, bases: np.ndarray, length: int, acc: GpuProjective) -> int:
    return int(lib().parallel_msm_api(device_id, _arr(data).ctypes.data, _arr(bases, 8).ctypes.data, length,
                                      ctypes.addressof(acc)))


# ---------------------------------------------------------------------------
# short names: fft / ifft / coset_fft / msm (return new arrays, raise)
# ---------------------------------------------------------------------------
def fft(a: np.ndarray, omega, log_n: int, device: int = 0) -> np.ndarray:
    out = np.array(_arr(a), copy=True)
    _check(lib().zkgpu_fft(device, out.ctypes.data, log_n, _el(omega).ctypes.data), "fft")
    return out


def ifft(a: np.ndarray, omega_inv, log_n: int, divisor, device: int = 0) -> np.ndarray:
    out = np.array(_arr(a), copy=True)
    _check(lib().zkgpu_ifft(device, out.ctypes.data, log_n, _el(omega_inv).ctypes.data, _el(divisor).ctypes.data),
           "ifft")
    return out


def coset_fft(a: np.ndarray, omega, log_n: int, c, device: int = 0) -> np.ndarray:
    out = np.array(_arr(a), copy=True)
    _check(lib().zkgpu_coset_fft(device, out.ctypes.data, log_n, _el(omega).ctypes.data, _el(c).ctypes.data),
           "coset_fft")
    return out


def lagrange_to_extended(values: np.ndarray, log_n: int, log_ext: int, omega_inv, divisor, g, omega_ext,
                         device: int = 0) -> np.ndarray:
    v = _arr(values)
    ext = np.empty((1 << log_ext, 4), np.uint64)
    _check(lib().zkgpu_lagrange_to_extended(device, v.ctypes.data, log_n, ext.ctypes.data, log_ext,
                                            _el(omega_inv).ctypes.data, _el(divisor).ctypes.data,
                                            _el(g).ctypes.data, _el(omega_ext).ctypes.data), "lagrange_to_extended")
    return ext


def extended_to_coeff(ext: np.ndarray, log_ext: int, m: int, omega_ext_inv, ext_divisor, g_inv,
                      device: int = 0) -> np.ndarray:
    """halo2 extended -> coefficients: ifft over 2^log_ext, times g_inv^i,
    first m coefficients."""
    e = _arr(ext)
    out = np.empty((m, 4), np.uint64)
    _check(lib().zkgpu_extended_to_coeff(device, e.ctypes.data, log_ext, out.ctypes.data, m,
                                         _el(omega_ext_inv).ctypes.data, _el(ext_divisor).ctypes.data,
                                         _el(g_inv).ctypes.data), "extended_to_coeff")
    return out


def msm(scalars: np.ndarray, bases: np.ndarray, device: int = 0) -> np.ndarray:
    """Returns the Jacobian sum (12 u64: X, Y, Z), normalised (Z = one) or all-zero."""
    s, b = _arr(scalars), _arr(bases, 8)
    assert s.shape[0] == b.shape[0]
    out = np.zeros(12, np.uint64)
    _check(lib().zkgpu_msm(device, s.ctypes.data, b.ctypes.data, s.shape[0], out.ctypes.data), "msm")
    return out


def field_op(op: str, a: np.ndarray, b: np.ndarray, field: str = "fr", device: int = 0) -> np.ndarray:
    a, b = _arr(a), _arr(b)
    out = np.empty_like(a)
    _check(lib().zkgpu_field_op(device, {"mul": 0, "add": 1, "sub": 2, "inv": 3}[op], {"fr": 0, "fq": 1}[field],
                                a.ctypes.data, b.ctypes.data, out.ctypes.data, a.shape[0]), "field_op")
    return out


def release_cached(device: int = 0):
    """Free the library's cached tables and pooled memory on `device`."""
    _check(lib().zkgpu_release_cached(device), "release_cached")


def launch_count(reset: bool = False) -> int:
    return int(lib().zkgpu_launch_count(1 if reset else 0))


def int_peak(device: int = 0, iters: int = 4096):
    """(IMAD/s, Fr Montgomery products/s) measured on `device`."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(lib().zkgpu_int_peak(device, iters, ctypes.byref(a), ctypes.byref(b)), "int_peak")
    return a.value, b.value


def prof_enable(on: bool = True):
    lib().zkgpu_prof_enable(1 if on else 0)


def prof_reset():
    lib().zkgpu_prof_reset()


def prof_read() -> dict:
    """{kernel: {"launches", "ms", "work", "bytes"}} for launches timed since the last reset."""
    buf = ctypes.create_string_buffer(1 << 16)
    lib().zkgpu_prof_read(buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms, work, by = line.split()
        out[name] = {"launches": int(cnt), "ms": float(ms), "work": float(work), "bytes": float(by)}
    return out


# ---------------------------------------------------------------------------
# device-resident API over torch tensors (plumbing only)
# ---------------------------------------------------------------------------
def _ptr(t) -> int:
    return int(t.data_ptr())


def _stream_ptr(stream) -> int | None:
    if stream is None:
        import torch
        return int(torch.cuda.current_stream().cuda_stream)
    return int(getattr(stream, "cuda_stream", stream))


def ntt_dev(t, log_n: int, omega, coset=None, post_scale=None, stream=None, device: int | None = None):
    """In-place NTT of a CUDA tensor of shape (2^log_n, 4), dtype int64/uint64."""
    dev = t.device.index if device is None else device
    c = _el(coset).ctypes.data if coset is not None else None
    cc = _el(coset) if coset is not None else None
    ps = _el(post_scale) if post_scale is not None else None
    om = _el(omega)
    _check(lib().zkgpu_ntt_dev(dev, _ptr(t), log_n, om.ctypes.data, cc.ctypes.data if cc is not None else None,
                               ps.ctypes.data if ps is not None else None, _stream_ptr(stream)), "ntt_dev")
    del c


def lagrange_to_extended_dev(values, ext, log_n: int, log_ext: int, omega_inv, divisor, g, omega_ext, stream=None):
    dev = values.device.index
    wi, d, gg, we = _el(omega_inv), _el(divisor), _el(g), _el(omega_ext)
    _check(lib().zkgpu_lagrange_to_extended_dev(dev, _ptr(values), log_n, _ptr(ext), log_ext, wi.ctypes.data,
                                                d.ctypes.data, gg.ctypes.data, we.ctypes.data, _stream_ptr(stream)),
           "lagrange_to_extended_dev")


def extended_to_coeff_dev(ext, out, log_ext: int, omega_ext_inv, ext_divisor, g_inv, stream=None):
    """out (m, 4) <- the first m coefficients of ext (2^log_ext, 4) moved off
    the coset g (g_inv = g^-1); device tensors."""
    dev = ext.device.index
    wi, d, gi = _el(omega_ext_inv), _el(ext_divisor), _el(g_inv)
    _check(lib().zkgpu_extended_to_coeff_dev(dev, _ptr(ext), log_ext, _ptr(out), out.shape[0], wi.ctypes.data,
                                             d.ctypes.data, gi.ctypes.data, _stream_ptr(stream)),
           "extended_to_coeff_dev")


EW_MUL, EW_ADD, EW_SUB, EW_SCALE, EW_AXPY = range(5)


def ew_dev(op: int, out, a, b=None, c=None, stream=None):
    """Element-wise op on CUDA tensors of shape (n, 4): out = a*b, a+b, a-b,
    a*c or a*c + b (c one element); out may be a or b."""
    dev = a.device.index
    cc = _el(c) if c is not None else None
    _check(lib().zkgpu_ew_dev(dev, op, _ptr(out), _ptr(a), _ptr(b) if b is not None else None,
                              cc.ctypes.data if cc is not None else None, a.shape[0], _stream_ptr(stream)),
           "ew_dev")


def divide_by_vanishing_dev(ext, log_n: int, log_ext: int, g, omega_ext, stream=None):
    """In place: ext[k] /= (g * omega_ext^k)^(2^log_n) - 1 (halo2 divide_by_vanishing_poly)."""
    gg, we = _el(g), _el(omega_ext)
    _check(lib().zkgpu_divide_by_vanishing_dev(ext.device.index, _ptr(ext), log_n, log_ext, gg.ctypes.data,
                                               we.ctypes.data, _stream_ptr(stream)), "divide_by_vanishing_dev")


JOB_COSET, JOB_SCALE = 1, 2


class NttJob(ctypes.Structure):
    """zkgpu_ntt_job (include/zkgpu.h)"""
    _fields_ = [("data", ctypes.c_void_p), ("log_n", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("omega", ctypes.c_uint64 * 4), ("coset", ctypes.c_uint64 * 4), ("scale", ctypes.c_uint64 * 4)]


class NttBatch:
    """Many in-place NTTs of uneven sizes run by one persistent launch from a
    captured CUDA graph.  jobs: dicts with keys tensor (CUDA, (2^log_n, 4)),
    log_n, omega, and optional coset, scale."""

    def __init__(self, jobs: list, device: int = 0):
        arr = (NttJob * len(jobs))()
        for i, j in enumerate(jobs):
            arr[i].data = _ptr(j["tensor"])
            arr[i].log_n = j["log_n"]
            flags = 0
            arr[i].omega[:] = [int(v) for v in _el(j["omega"])]
            if j.get("coset") is not None:
                flags |= JOB_COSET
                arr[i].coset[:] = [int(v) for v in _el(j["coset"])]
            if j.get("scale") is not None:
                flags |= JOB_SCALE
                arr[i].scale[:] = [int(v) for v in _el(j["scale"])]
            arr[i].flags = flags
        self._jobs = arr
        self.handle = ctypes.c_void_p()
        _check(lib().zkgpu_ntt_batch_create(device, arr, len(jobs), ctypes.byref(self.handle)), "ntt_batch_create")

    def run(self, stream=None):
        _check(lib().zkgpu_ntt_batch_run(self.handle, _stream_ptr(stream)), "ntt_batch_run")

    def check(self):
        _check(lib().zkgpu_ntt_batch_check(self.handle), "ntt_batch_check")

    def info(self) -> dict:
        p, t, g = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int()
        lib().zkgpu_ntt_batch_info(self.handle, ctypes.byref(p), ctypes.byref(t), ctypes.byref(g))
        return {"passes": p.value, "tiles": t.value, "grid": g.value}

    def close(self):
        if self.handle:
            lib().zkgpu_ntt_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


KIND_NTT, KIND_LDE, KIND_MSM = 0, 1, 2


class Job(ctypes.Structure):
    """zkgpu_job (include/zkgpu.h)"""
    _fields_ = [("kind", ctypes.c_uint32), ("log_n", ctypes.c_uint32), ("log_ext", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("n", ctypes.c_uint64), ("bases_id", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("input", ctypes.c_void_p), ("output", ctypes.c_void_p),
                ("omega", ctypes.c_uint64 * 4), ("coset", ctypes.c_uint64 * 4), ("scale", ctypes.c_uint64 * 4),
                ("omega_ext", ctypes.c_uint64 * 4)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("submitted", "rejected", "completed", "failed", "waves",
                                               "batch_launches", "hbm_budget", "hbm_used", "hbm_peak", "pending",
                                               "inflight", "msm_merged_passes", "msm_merged_jobs", "table_builds",
                                               "cache_clears", "memory_waits", "max_launch_us")]


def _set4(dst, v):
    dst[:] = [int(x) for x in _el(v)]


def ntt_job(inp: np.ndarray, out: np.ndarray, log_n: int, omega, coset=None, scale=None) -> Job:
    j = Job()
    j.kind, j.log_n = KIND_NTT, log_n
    j.input, j.output = inp.ctypes.data, out.ctypes.data
    _set4(j.omega, omega)
    if coset is not None:
        j.flags |= JOB_COSET
        _set4(j.coset, coset)
    if scale is not None:
        j.flags |= JOB_SCALE
        _set4(j.scale, scale)
    return j


def lde_job(inp: np.ndarray, out: np.ndarray, log_n: int, log_ext: int, omega_inv, divisor, g, omega_ext) -> Job:
    j = Job()
    j.kind, j.log_n, j.log_ext = KIND_LDE, log_n, log_ext
    j.input, j.output = inp.ctypes.data, out.ctypes.data
    _set4(j.omega, omega_inv)
    _set4(j.scale, divisor)
    _set4(j.coset, g)
    _set4(j.omega_ext, omega_ext)
    return j


def msm_job(scalars: np.ndarray, out: np.ndarray, n: int, bases_id: int) -> Job:
    j = Job()
    j.kind, j.n, j.bases_id = KIND_MSM, n, bases_id
    j.input, j.output = scalars.ctypes.data, out.ctypes.data
    return j


class Server:
    """Serving loop (continuous batching, HBM-budget admission) over the C ABI.
    Host buffers passed to submit() must stay alive until wait() returns."""

    def __init__(self, device: int = 0, hbm_budget: int = 150 * 10**9, max_wave_jobs: int = 256):
        self.handle = ctypes.c_void_p()
        _check(lib().zkgpu_server_create(device, hbm_budget, max_wave_jobs, ctypes.byref(self.handle)),
               "server_create")
        self._keep = {}

    def add_bases(self, bases: np.ndarray) -> int:
        b = _arr(bases, 8)
        bid = ctypes.c_uint32()
        _check(lib().zkgpu_server_add_bases(self.handle, b.ctypes.data, b.shape[0], ctypes.byref(bid)), "add_bases")
        return bid.value

    def submit(self, job: Job, keep=None) -> int:
        t = ctypes.c_uint64()
        _check(lib().zkgpu_server_submit(self.handle, ctypes.byref(job), ctypes.byref(t)), "server_submit")
        self._keep[t.value] = (job, keep)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 0) -> float:
        lat = ctypes.c_double()
        rc = lib().zkgpu_server_wait(self.handle, ticket, timeout_ms, ctypes.byref(lat))
        self._keep.pop(ticket, None)
        _check(rc, "server_wait")
        return lat.value

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib().zkgpu_server_stats_get(self.handle, ctypes.byref(s)), "server_stats")
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self.handle:
            lib().zkgpu_server_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def job_footprint(job: Job) -> int:
    return int(lib().zkgpu_job_footprint(ctypes.byref(job)))


def admission_simulate(budget: int, footprints) -> tuple:
    fp = np.ascontiguousarray(footprints, dtype=np.uint64)
    rounds = np.zeros(fp.shape[0], np.int32)
    peak = lib().zkgpu_admission_simulate(budget, fp.ctypes.data, fp.shape[0], rounds.ctypes.data)
    return int(peak), rounds


def msm_dev(scalars, bases, out, stream=None):
    dev = scalars.device.index
    _check(lib().zkgpu_msm_dev(dev, _ptr(scalars), _ptr(bases), scalars.shape[0], _ptr(out), _stream_ptr(stream)),
           "msm_dev")


def g1_mul_fixed_dev(scalars, out, base=None, stream=None):
    """out[i] = scalars[i] * base on the device (affine, Fq Montgomery; base
    defaults to the generator (1, 2)).  scalars: (n, 4) int64 Fr Montgomery,
    out: (n, 8) int64."""
    if base is None:
        base = G1_GENERATOR
    b = _arr(base, 8).reshape(-1)
    dev = scalars.device.index
    _check(lib().zkgpu_g1_mul_fixed_dev(dev, b.ctypes.data, _ptr(scalars), scalars.shape[0], _ptr(out),
                                        _stream_ptr(stream)), "g1_mul_fixed_dev")


TUNE_NTT, TUNE_MSM, TUNE_NTT_BATCHED = 1, 2, 4


def autotune(what: int, log_min: int, log_max: int, device: int = 0, reps: int = 3) -> float:
    """Time candidate NTT plans / MSM windows for sizes 2^log_min..2^log_max
    on `device` and install the fastest; returns the device ms spent."""
    ms = ctypes.c_double()
    _check(lib().zkgpu_autotune(device, what, log_min, log_max, reps, ctypes.byref(ms)), "autotune")
    return ms.value


def set_ntt_plan(log_n: int, bits, device: int = 0):
    """Install pass widths for 2^log_n (empty / None: the built-in plan)."""
    bits = list(bits or [])
    arr = (ctypes.c_uint32 * max(4, len(bits)))(*(bits + [0] * (4 - len(bits))))
    _check(lib().zkgpu_tune_set_ntt_plan(device, log_n, len(bits), arr), "tune_set_ntt_plan")


def get_ntt_plan(log_n: int, device: int = 0) -> list:
    npass = ctypes.c_uint32()
    arr = (ctypes.c_uint32 * 4)()
    _check(lib().zkgpu_tune_get_ntt_plan(device, log_n, ctypes.byref(npass), arr), "tune_get_ntt_plan")
    return [int(arr[k]) for k in range(npass.value)]


def set_msm_window(log_n: int, c: int, device: int = 0):
    _check(lib().zkgpu_tune_set_msm_window(device, log_n, c), "tune_set_msm_window")


def get_msm_window(log_n: int, device: int = 0) -> int:
    c = ctypes.c_uint32()
    _check(lib().zkgpu_tune_get_msm_window(device, log_n, ctypes.byref(c)), "tune_get_msm_window")
    return c.value


def tune_save(path: str, device: int = 0):
    _check(lib().zkgpu_tune_save(device, path.encode()), "tune_save")


def tune_load(path: str, device: int = 0) -> int:
    n = ctypes.c_uint32()
    _check(lib().zkgpu_tune_load(device, path.encode(), ctypes.byref(n)), "tune_load")
    return n.value
