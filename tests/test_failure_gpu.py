"""GPU failure detection without a fault: a bounded device wait that nothing
satisfies must expire, be reported as ZKGPU_ETIMEOUT, and leave the CUDA
context usable for the next call."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(zk, oracle):
    w12 = oracle.omega(12)
    rc = zk.lib().zkgpu_selftest_wait_timeout(0, w12.ctypes.data, 200000)   # ~0.2 s budget
    assert rc == zk.ETIMEOUT
    # the device still works
    a = oracle.rand_fr(1 << 14, 3)
    assert np.array_equal(zk.fft(a, oracle.omega(14), 14), oracle.best_fft(a, oracle.omega(14), 14))


def test_selftest_rejects_bad_arguments(zk, oracle):
    assert zk.lib().zkgpu_selftest_wait_timeout(0, oracle.omega(13).ctypes.data, 1000) == zk.EINVAL
    assert zk.lib().zkgpu_selftest_wait_timeout(0, oracle.omega(12).ctypes.data, 0) == zk.EINVAL
