"""CPU: the MSM's branch-free divstep Fq inversion (fq_inv.cuh, compiled for
the host from the same source the kernels use) against Python bigints, on
random values, the edges 1, 2, (q-1)/2, q-1, and long runs of equal bits."""
import os
import random
import shutil
import subprocess

import pytest

Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_divstep_inversion_matches_bigint(tmp_path):
    exe = tmp_path / "fq_inv_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), os.path.join(HERE, "fq_inv_check.cpp")], check=True)
    rng = random.Random(2024)
    vals = [1, 2, 3, (Q - 1) // 2, Q - 2, Q - 1, 1 << 253, (1 << 254) % Q] + [rng.randrange(1, Q) for _ in range(3000)]
    # powers of two, all-ones patterns and q - 2^k: long runs of equal bits
    vals += [1 << k for k in range(254)] + [(1 << k) - 1 for k in range(2, 254)] + [Q - (1 << k) for k in range(253)]
    inp = "".join(f"{v:064x}\n" for v in vals)
    out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True).stdout.split()
    assert len(out) == len(vals)
    for v, r in zip(vals, out):
        assert int(r, 16) == pow(v, -1, Q), hex(v)


@pytest.mark.gpu
def test_device_divstep_inversion_matches_bigint(zk):
    """The same inversion on the GPU (zkgpu_field_op op 3, the function the
    MSM rounds call): edges, long runs of equal bits and random values."""
    import numpy as np
    rng = random.Random(4049)
    vals = [0, 1, 2, 3, (Q - 1) // 2, Q - 2, Q - 1] + [1 << k for k in range(254)] + \
        [(1 << k) - 1 for k in range(2, 254)] + [Q - (1 << k) for k in range(253)] + \
        [rng.randrange(1, Q) for _ in range(8000)]
    a = np.array([[(v >> (64 * i)) & ((1 << 64) - 1) for i in range(4)] for v in vals], dtype=np.uint64)
    out = zk.field_op("inv", a, a, "fq")
    for v, row in zip(vals, out):
        got = sum(int(w) << (64 * i) for i, w in enumerate(row))
        assert got == (pow(v, -1, Q) if v else 0), hex(v)
