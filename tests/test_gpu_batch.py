"""Cases in the mix: each result is the same, bit for bit, alone and beside others on the GPU."""
import pytest

from pysurf_b200 import batch

pytestmark = pytest.mark.gpu


def test_each_case_is_the_same_alone_and_in_the_mix():
    specs = [batch.CaseSpec(k, slope, height, ppd) for k, (slope, height, ppd) in
             enumerate([(1 / 15, 0.45, 16), (1 / 10, 0.3, 12), (1 / 25, 0.5, 14), (1 / 8, 0.25, 12),
                        (1 / 20, 0.6, 16), (1 / 30, 0.35, 12)])]
    alone = [batch.solveCase(spec) for spec in specs]
    mixed = batch.BatchRunner(slots=4).run(specs)
    for a, m in zip(alone, mixed):
        assert a.error is None and m.error is None
        assert a.index == m.index
        assert a.key() == m.key()
    assert any(r.breakingTime == r.breakingTime for r in alone)      # some broke (not NaN)


def test_a_served_stream_returns_every_request_with_its_latency():
    specs = [batch.CaseSpec(k, 1 / 15, 0.4, 12, endTime=0.5, toBreaking=False) for k in range(6)]
    arrivals = batch.poissonArrivals(len(specs), 20.0, seed=3)
    out = batch.serve([batch.Request(float(t), s) for t, s in zip(arrivals, specs)], slots=3)
    results = out['results']
    assert [r.index for r in results] == list(range(6))
    assert all(r.error is None and r.simulatedTime >= 0.5 for r in results)
    alone = batch.solveCase(specs[0])
    assert alone.key() == results[0].key()
    assert 0.0 < out['latency_p50_s'] <= out['latency_p99_s']
