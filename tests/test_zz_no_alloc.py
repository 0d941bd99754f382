"""GPU: the allocation-free NTT entry point (zkgpu_ntt_dev_static).

It exists for callers that cannot allocate device memory — code running under
CUDA stream capture, or inside a runtime that owns every device allocation —
and keeps its scratch in a static device array inside libzkgpu.so.  Its
output must equal the ordinary device entry point's (zkgpu_ntt_dev), bit for
bit, on consecutive calls that reuse the shared array, and the CPU oracle's
halo2 best_fft on the same input (so a fault shared by both device entry
points cannot pass).  This file is collected last on purpose, and also passes
when run alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_LOG = 18  # ZKGPU_STATIC_NTT_MAX_LOG in include/zkgpu.h


def _run_static(zk, t, log_n, omega, stream):
    rc = zk.lib().zkgpu_ntt_dev_static(t.device.index, t.data_ptr(), log_n, omega.ctypes.data,
                                        stream.cuda_stream)
    assert rc == 0, zk.lib().zkgpu_last_error()


@pytest.mark.parametrize("sizes", [(MAX_LOG, MAX_LOG), (16, 11)])
def test_static_matches_default_entry_on_consecutive_calls(zk, oracle, sizes):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.Stream()
    for call, log_n in enumerate(sizes):
        a = oracle.rand_fr(1 << log_n, 900 + 10 * call + log_n)
        w = oracle.omega(log_n)
        t_static = torch.from_numpy(a.view(np.int64)).cuda()
        t_default = t_static.clone()
        torch.cuda.synchronize()
        _run_static(zk, t_static, log_n, w, stream)
        zk.ntt_dev(t_default, log_n, w, stream=stream)
        stream.synchronize()
        assert torch.equal(t_static, t_default), f"call {call}: log_n={log_n}"
        want = oracle.best_fft(a, w, log_n)
        assert np.array_equal(t_static.cpu().numpy().view(np.uint64), want), f"call {call}: oracle, log_n={log_n}"


def test_static_rejects_oversize(zk, oracle):
    torch = pytest.importorskip("torch")
    log_n = MAX_LOG + 1
    t = torch.zeros((1 << log_n, 4), dtype=torch.int64, device="cuda")
    w = oracle.omega(log_n)
    rc = zk.lib().zkgpu_ntt_dev_static(t.device.index, t.data_ptr(), log_n, w.ctypes.data, None)
    assert rc == zk.EINVAL
    assert b"ZKGPU_STATIC_NTT_MAX_LOG" in zk.lib().zkgpu_last_error()
    assert not t.any()
