"""CPU: libzkgpu.so loads (without a GPU) and exports exactly what
include/zkgpu.h declares; argument validation needs no device."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "zkgpu.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", src, re.M)
    return sorted(set(n for n in names if n not in ("if", "while")))


def test_header_declares_reference_symbols():
    names = declared_symbols()
    # src/api.rs:3-14
    for ref in ("do_fft_ffi", "parallel_fft_api", "parallel_ifft_api", "parallel_coeff_to_extended_part_api",
                "parallel_msm_api"):
        assert ref in names


def test_library_exports_every_declared_symbol(zk):
    out = subprocess.run(["nm", "-D", "--defined-only", zk.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (\S+)$", out, re.M))
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, missing
    # the ctypes mirror binds the same set
    assert set(zk.EXPORTS) == set(declared_symbols())


def test_struct_layouts(zk):
    import ctypes
    assert ctypes.sizeof(zk.GpuAffine) == 64 and ctypes.sizeof(zk.GpuProjective) == 96


def test_argument_validation_without_device(zk, oracle):
    a = np.zeros((8, 4), np.uint64)
    w = oracle.omega(3)
    # n != 2^log_n
    assert zk.parallel_fft_api(0, a, w, None, 7, 3, 0) == zk.EINVAL
    # omega of the wrong order
    assert zk.parallel_fft_api(0, a, oracle.omega(4), None, 8, 3, 0) == zk.EINVAL
    # non-canonical omega
    bad = np.array([2**64 - 1] * 4, np.uint64)
    assert zk.parallel_fft_api(0, a, bad, None, 8, 3, 0) == zk.EINVAL
    # log_n beyond the two-adicity
    assert zk.lib().zkgpu_fft(0, a.ctypes.data, 29, w.ctypes.data) == zk.EINVAL
    assert zk.lib().zkgpu_version().startswith(b"zkgpu")
