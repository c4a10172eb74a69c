"""Solve server: request stream, admission and result invariance.

CPU tests check the synthetic stream and the latency summary.  GPU tests
check that a case's result is the same served alone, in a mix of
concurrently running cases, with and without CUDA graphs, and through the
plain one-at-a-time algorithm API.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from gridfoam_b200.serving import SIZES, CavityRequest, poisson_stream, summarize  # noqa: E402
from gridfoam_b200.serving.engine import ServeResult  # noqa: E402


def test_poisson_stream_statistics():
    reqs = poisson_stream(4000, rate=50.0, seed=0)
    arr = np.array([r.arrival for r in reqs])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert abs(np.mean(np.diff(arr)) - 1 / 50.0) < 0.1 / 50.0
    assert {r.n for r in reqs} == set(SIZES)
    re = np.array([r.re for r in reqs])
    assert re.min() >= 10.0 and re.max() <= 1000.0
    # log-uniform: the median sits near the geometric mean of the range
    assert abs(np.log(np.median(re)) - 0.5 * (np.log(10) + np.log(1000))) < 0.1
    lid = np.array([r.lid for r in reqs])
    assert lid.min() >= 0.5 and lid.max() <= 2.0
    assert np.allclose([r.nu for r in reqs], lid / re)
    again = poisson_stream(4000, rate=50.0, seed=0)
    assert again == reqs


def test_summarize_percentiles():
    res = [ServeResult(i, 16, arrival=float(i), admitted=float(i), finished=float(i) + 1.0 + (i % 10) * 0.1,
                       iterations=10, converged=True, residual=0.0) for i in range(100)]
    s = summarize(res)
    assert s["completed"] == 100
    assert s["p50_latency_s"] == pytest.approx(np.percentile([1.0 + (i % 10) * 0.1 for i in range(100)], 50))
    assert s["p99_latency_s"] <= 1.9 + 1e-12
    assert s["solves_per_s"] == pytest.approx(100 / (99 + 1.9))


def _mix():
    return [CavityRequest(0, 8, 100.0, 1.0, 0.0), CavityRequest(1, 12, 400.0, 1.5, 0.0),
            CavityRequest(2, 16, 30.0, 0.7, 0.0), CavityRequest(3, 12, 900.0, 2.0, 0.0)]


@pytest.mark.gpu
def test_result_same_alone_and_in_mix():
    from gridfoam_b200.serving import ServingEngine

    reqs = _mix()
    eng = ServingEngine(max_slots=4, max_outer=40, keep_fields=True)
    eng.prepare({r.n for r in reqs})
    mixed = {r.id: r for r in eng.run(reqs)}
    assert len(mixed) == len(reqs)
    for req in reqs:
        alone = eng.run([req])[0]
        m = mixed[req.id]
        assert alone.iterations == m.iterations
        # the same launches on the same data: bitwise equal
        np.testing.assert_array_equal(alone.U, m.U)
        np.testing.assert_array_equal(alone.p, m.p)


@pytest.mark.gpu
def test_graph_replay_matches_eager_and_plain_api():
    from gridfoam_b200.serving import ServingEngine, serve_sequential

    reqs = _mix()[:2]
    g = ServingEngine(max_slots=2, max_outer=30, keep_fields=True)
    g.prepare({r.n for r in reqs}, autotune=False)
    e = ServingEngine(max_slots=2, max_outer=30, keep_fields=True, use_graphs=False)
    e.prepare({r.n for r in reqs}, autotune=False)
    rg = {r.id: r for r in g.run(reqs)}
    re_ = {r.id: r for r in e.run(reqs)}
    rs = {r.id: r for r in serve_sequential(reqs, max_outer=30, keep_fields=True)}
    for req in reqs:
        np.testing.assert_array_equal(rg[req.id].U, re_[req.id].U)
        np.testing.assert_array_equal(rg[req.id].p, re_[req.id].p)
        assert rg[req.id].iterations == rs[req.id].iterations
        np.testing.assert_allclose(rg[req.id].U, rs[req.id].U, rtol=0, atol=1e-12)
        np.testing.assert_allclose(rg[req.id].p, rs[req.id].p, rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_small_cavity_converges_to_residual_control():
    from gridfoam_b200.serving import ServingEngine

    eng = ServingEngine(max_slots=2, max_outer=3000, p_solver_tol=1e-12)
    eng.prepare({8})
    (r,) = eng.run([CavityRequest(0, 8, 50.0, 1.0, 0.0)])
    assert r.converged and r.residual < 1e-6 and r.iterations < 3000
