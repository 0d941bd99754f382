"""CPU: host-side helpers of bench.py's serving measurement (no GPU)."""
import bench


def test_median_closed_run_ignores_one_stalled_run():
    spans = iter([1.58, 0.95, 1.00])
    calls = []

    def run(offered):
        calls.append(offered)
        sp = next(spans)
        return [sp / 2] * 10, sp

    (lat, span), rates = bench.median_closed_run(run, 1000)
    assert calls == [None, None, None]  # closed loops only
    assert span == 1.00 and lat == [0.5] * 10
    assert rates == [1052.6, 1000.0, 632.9]


def test_median_closed_run_single():
    (lat, span), rates = bench.median_closed_run(lambda o: ([1.0], 2.0), 100, reps=1)
    assert span == 2.0 and rates == [50.0]


def test_serving_trace_is_seeded_and_mixed():
    t1, t2 = bench.serving_trace(1000), bench.serving_trace(1000)
    assert t1 == t2
    kinds = {k for _, k, _ in t1}
    assert kinds == {"ntt", "lde", "msm"}
    assert all(12 <= lg <= 22 for _, k, lg in t1 if k != "msm")
    assert all(14 <= lg <= 20 for _, k, lg in t1 if k == "msm")
    assert all(a <= b for (a, _, _), (b, _, _) in zip(t1, t1[1:]))  # arrival times ascend
