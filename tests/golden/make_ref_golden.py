"""Generate golden vectors from the reference's own CUDA path.

Runs the reference library (cuda/fft.cu compiled from its sources by
`make -C oracle ref` into oracle/_ref/libref_fft.so) through its C exports on
seeded inputs made by the oracle, and saves inputs + reference outputs as
.npz fixtures.  Needs a CUDA device; run it as

    python tests/golden/make_ref_golden.py --out <dir>

then copy the .npz files into tests/golden/.  The reference path's size limits
are respected (NTT n >= 2^10; MSM length a power of two > 256,
cuda/fft.cu:330-340, 460-479).  The reference is never imported by the tests;
only these files are.
"""
import argparse
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402


def load_ref():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_fft.so"))
    P = ctypes.c_void_p
    # C definitions, cuda/fft.cu:560-582
    lib.parallel_fft_api.argtypes = [ctypes.c_int, P, P, P, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
    lib.parallel_ifft_api.argtypes = [ctypes.c_int, P, P, P, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, P]
    lib.parallel_coeff_to_extended_part_api.argtypes = [ctypes.c_int, P, P, P, ctypes.c_uint64, ctypes.c_int,
                                                        ctypes.c_int, P]
    lib.parallel_msm_api.argtypes = [ctypes.c_int, P, P, ctypes.c_uint64, P, ctypes.c_uint64]
    for f in ("parallel_fft_api", "parallel_ifft_api", "parallel_coeff_to_extended_part_api", "parallel_msm_api"):
        getattr(lib, f).restype = ctypes.c_int
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    ref = load_ref()
    for k in (10, 12):
        n = 1 << k
        w = O.omega(k)
        tw = O.twiddle_lut(w, k, 10, True)
        a = O.rand_fr(n, 5000 + k)
        out = a.copy()
        assert ref.parallel_fft_api(0, out.ctypes.data, w.ctypes.data, tw.ctypes.data, n, k, tw.shape[0]) == 0
        np.savez(os.path.join(args.out, f"ref_fft_{k}.npz"), input=a, omega=w, output=out)

        wi = O.inv(w)
        twi = O.twiddle_lut(wi, k, 10, True)
        d = O.inv(O.to_mont(n))
        out = a.copy()
        assert ref.parallel_ifft_api(0, out.ctypes.data, wi.ctypes.data, twi.ctypes.data, n, k, twi.shape[0],
                                     d.ctypes.data) == 0
        np.savez(os.path.join(args.out, f"ref_ifft_{k}.npz"), input=a, omega=wi, divisor=d, output=out)

        # one part of the x4 extended domain: c = g * w_ext^1
        c = O.mul(O.to_mont(7), O.omega(k + 2))
        out = a.copy()
        assert ref.parallel_coeff_to_extended_part_api(0, out.ctypes.data, w.ctypes.data, tw.ctypes.data, n, k,
                                                       tw.shape[0], c.ctypes.data) == 0
        np.savez(os.path.join(args.out, f"ref_coset_{k}.npz"), input=a, omega=w, c=c, output=out)

    for lg, small in ((10, False), (12, True)):
        n = 1 << lg
        s = O.rand_fr(n, 6000 + lg)
        if small:
            s[: n // 10] = O.rand_fr_small(n // 10, 6100 + lg, bits=16)
        bases = O.rand_bases(n, 6200 + lg)
        acc = np.zeros(12, np.uint64)
        assert ref.parallel_msm_api(0, s.ctypes.data, bases.ctypes.data, n, acc.ctypes.data, 0) == 0
        np.savez(os.path.join(args.out, f"ref_msm_{lg}.npz"), scalars=s, bases=bases, output=acc)
    print("golden vectors written to", args.out)


if __name__ == "__main__":
    main()
