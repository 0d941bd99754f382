"""Time the reference's own CUDA path (cuda/fft.cu compiled for sm_100a into
oracle/_ref/libref_fft.so by `make -C oracle ref`) on the benchmark configs,
through its own C exports, as context rows beside this library's numbers.

Configs, all within the reference's documented limits (NTT n >= 2^10; MSM
length a power of two above 256, cuda/fft.cu:330-340, 460-479):
  * forward NTT 2^16 (parallel_fft_api);
  * the 2^24 -> 2^26 coset LDE as the reference's callers run it: one
    parallel_ifft_api of 2^24, then four parallel_coeff_to_extended_part_api
    calls of 2^24 with c_j = 7 * w_ext^j (the extended evaluations
    interleaved, k = 4 i + j);
  * MSM of 2^22 points, 10 % of the scalars below 2^16 (parallel_msm_api).
Each reference call is synchronous and copies its inputs and outputs
(cuda/fft.cu:282-285, 388, 455-489, 541), so the wall time of a call is its
end-to-end time, comparable with this library's host-buffer calls.  Inputs
come from the oracle's seeded generators.  Usage (needs a CUDA device):

    python oracle/ref_gpu_timing.py > ref_gpu.json
"""
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import pyoracle as O  # noqa: E402


def load_ref():
    lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_fft.so"))
    P = ctypes.c_void_p
    # the C definitions, cuda/fft.cu:560-582
    lib.parallel_fft_api.argtypes = [ctypes.c_int, P, P, P, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
    lib.parallel_ifft_api.argtypes = [ctypes.c_int, P, P, P, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, P]
    lib.parallel_coeff_to_extended_part_api.argtypes = [ctypes.c_int, P, P, P, ctypes.c_uint64, ctypes.c_int,
                                                        ctypes.c_int, P]
    lib.parallel_msm_api.argtypes = [ctypes.c_int, P, P, ctypes.c_uint64, P, ctypes.c_uint64]
    for f in ("parallel_fft_api", "parallel_ifft_api", "parallel_coeff_to_extended_part_api", "parallel_msm_api"):
        getattr(lib, f).restype = ctypes.c_int
    return lib


def timed(fn, reps=1):
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return best


def main():
    ref = load_ref()
    out = {"library": "reference cuda/fft.cu rebuilt for sm_100a (oracle/_ref/libref_fft.so)"}

    # forward NTT 2^16, best of 5 (the first call pays the context start-up)
    k = 16
    n = 1 << k
    w = O.omega(k)
    tw = O.twiddle_lut(w, k, 10, True)
    a = O.rand_fr(n, 16)
    buf = a.copy()
    assert ref.parallel_fft_api(0, buf.ctypes.data, w.ctypes.data, tw.ctypes.data, n, k, tw.shape[0]) == 0
    ok = np.array_equal(buf, O.best_fft(a, w, k))

    def fft16():
        b = a.copy()
        assert ref.parallel_fft_api(0, b.ctypes.data, w.ctypes.data, tw.ctypes.data, n, k, tw.shape[0]) == 0
    t = timed(fft16, 5)
    out["ntt_2p16"] = {"ms": round(t * 1e3, 3), "melem_s": round(n / t / 1e6, 2), "matches_oracle": bool(ok)}

    # LDE 2^24 -> 2^26: ifft, then four coset parts
    k, e = 24, 2
    n = 1 << k
    w = O.omega(k)
    wi = O.inv(w)
    d = O.inv(O.to_mont(n))
    twi = O.twiddle_lut(wi, k, 10, True)
    tw = O.twiddle_lut(w, k, 10, True)
    vals = O.rand_fr(n, 24)
    we = O.omega(k + e)
    g = O.to_mont(7)
    cs = [O.mul(g, O.pow_(we, j)) for j in range(1 << e)]
    parts = [None] * (1 << e)

    def lde():
        coeffs = vals.copy()
        assert ref.parallel_ifft_api(0, coeffs.ctypes.data, wi.ctypes.data, twi.ctypes.data, n, k, twi.shape[0],
                                     d.ctypes.data) == 0
        for j, c in enumerate(cs):
            p = coeffs.copy()
            assert ref.parallel_coeff_to_extended_part_api(0, p.ctypes.data, w.ctypes.data, tw.ctypes.data, n, k,
                                                           tw.shape[0], c.ctypes.data) == 0
            parts[j] = p
    t = timed(lde, 1)
    out["lde_2p24_2p26"] = {"ms": round(t * 1e3, 1), "melem_s": round(n / t / 1e6, 3),
                            "calls": "1 ifft + 4 coset parts of 2^24, each with its own copies"}

    # MSM 2^22, 10 % small scalars
    n = 1 << 22
    s = O.rand_fr(n, 22)
    s[: n // 10] = O.rand_fr_small(n // 10, 23, bits=16)
    bases = O.rand_bases(n, 24)
    acc = np.zeros(12, np.uint64)

    def msm():
        assert ref.parallel_msm_api(0, s.ctypes.data, bases.ctypes.data, n, acc.ctypes.data, 0) == 0
    t = timed(msm, 1)
    out["msm_2p22"] = {"ms": round(t * 1e3, 1), "mpts_s": round(n / t / 1e6, 3)}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
