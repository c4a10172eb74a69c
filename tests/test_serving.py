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


def test_batched_block_shares():
    from gridfoam_b200.serving import blocks_for

    assert blocks_for(16**3, False) == 4 and blocks_for(96**3, False) == 296
    assert blocks_for(48**3, False) == 108 and blocks_for(32**3, False) == 32
    assert blocks_for(16**3, True) == 1 and blocks_for(48**3, True) == 14 and blocks_for(96**3, True) == 74
    # the lane's sizes (up to 48^3) fit the batched CG's co-resident blocks
    # (4 a SM of 148) several at a time
    assert 5 * blocks_for(48**3, False) <= 4 * 148


def test_solo_threshold():
    from gridfoam_b200.serving.batched import BatchedEngine

    eng = BatchedEngine.__new__(BatchedEngine)
    eng.solo_cells = 200_000
    assert not eng.is_solo(48) and eng.is_solo(64) and eng.is_solo(96)
    eng.solo_cells = None
    assert not eng.is_solo(96)


def test_batched_stopping_rule_statuses():
    """The host side of the batched engine's stopping rule (no GPU): a
    residual below residualControl converges, a non-finite one ends the
    request, the endTime cap ends the rest."""
    from gridfoam_b200.serving.batched import BatchedEngine

    class _C:
        def __init__(self):
            self.iterations, self.residual, self.status = 0, float("inf"), "running"

    eng = BatchedEngine.__new__(BatchedEngine)
    eng.p_tol, eng.max_outer = 1e-6, 3
    eng._res_host = torch.tensor([5e-7, float("nan"), 1e-3], dtype=torch.float64)
    cases = [_C(), _C(), _C()]
    eng._finish(cases, 0.0)
    assert [c.status for c in cases] == ["converged", "nonfinite", "running"]
    cases[2].iterations = 2
    eng._res_host = torch.tensor([1e-3], dtype=torch.float64)
    eng._finish(cases[2:], 0.0)
    assert cases[2].status == "end_time"


def _converging_mix():
    return [CavityRequest(0, 8, 100.0, 1.0, 0.0), CavityRequest(1, 12, 400.0, 1.5, 0.0),
            CavityRequest(2, 16, 30.0, 0.7, 0.0), CavityRequest(3, 12, 900.0, 2.0, 0.0)]


@pytest.mark.gpu
def test_batched_engine_alone_equals_mix_and_converges():
    """Lockstep engine: every request converges to residualControl; each
    result is bitwise the same served alone (a batch of one) and in the mix
    (its solves run on the same blocks with the same kernels)."""
    from gridfoam_b200.serving import BatchedEngine

    reqs = _converging_mix()
    eng = BatchedEngine(max_slots=4, max_outer=3000, keep_fields=True)
    eng.prepare({r.n for r in reqs})
    mixed = {r.id: r for r in eng.run(reqs)}
    assert eng.captures >= 1 and eng.launches >= 2
    assert len(mixed) == len(reqs) and all(r.converged for r in mixed.values()), \
        [(r.id, r.status, r.residual, r.iterations) for r in mixed.values()]
    for req in reqs:
        (alone,) = eng.run([req])
        m = mixed[req.id]
        assert alone.iterations == m.iterations
        np.testing.assert_array_equal(alone.U, m.U)
        np.testing.assert_array_equal(alone.p, m.p)


@pytest.mark.gpu
def test_batched_engine_matches_plain_api_at_equal_residual():
    """The lockstep engine and the one-at-a-time plain API (other CG
    kernels, same algorithm) both run to residualControl: the converged
    velocities agree to the stopping tolerance."""
    from gridfoam_b200.serving import BatchedEngine, serve_sequential

    reqs = _converging_mix()[:2]
    eng = BatchedEngine(max_slots=2, max_outer=3000, keep_fields=True)
    eng.prepare({r.n for r in reqs})
    rb = {r.id: r for r in eng.run(reqs)}
    rs = {r.id: r for r in serve_sequential(reqs, max_outer=3000, p_solver_tol=1e-12, p_solver_rtol=0.01,
                                             keep_fields=True)}
    for req in reqs:
        assert rb[req.id].converged and rs[req.id].converged
        err = np.linalg.norm(rb[req.id].U - rs[req.id].U) / np.linalg.norm(rs[req.id].U)
        assert err < 1e-5, err


@pytest.mark.gpu
def test_batched_engine_fault_injection():
    """Host-side faults: a simulated out-of-memory at admission and a NaN
    input are each rejected or ended while the other requests converge."""
    from gridfoam_b200.serving import BatchedEngine

    reqs = _converging_mix()
    bad_nan = CavityRequest(10, 8, 100.0, 1.0, 0.0)
    oom = CavityRequest(11, 12, 100.0, 1.0, 0.0)
    eng = BatchedEngine(max_slots=6, max_outer=3000, keep_fields=False)
    eng.prepare({r.n for r in reqs})

    def hook(req):
        if req.id == oom.id:
            raise torch.cuda.OutOfMemoryError("simulated out-of-memory at admission")

    def poison(case):
        if case.req.id == bad_nan.id:
            case.algo.U.store[0, 5] = float("nan")  # NaN input field

    eng.admission_hook = hook
    eng.case_hook = poison
    res = {r.id: r for r in eng.run(reqs + [bad_nan, oom])}
    assert res[oom.id].status.startswith("rejected")
    assert res[bad_nan.id].status == "nonfinite"
    for r in reqs:
        assert res[r.id].converged, (r.id, res[r.id].status)
    # a request that can never fit the HBM budget is rejected, not queued
    small = BatchedEngine(hbm_budget=1 << 20, max_slots=2, max_outer=10)
    small.footprint = dict(eng.footprint)
    (rej,) = small.run([CavityRequest(20, 16, 100.0, 1.0, 0.0)])
    assert rej.status == "rejected_memory"


@pytest.mark.gpu
def test_batched_fp32_inner_matches_fp64_at_equal_residual():
    """FP32 inner CG iterations inside FP64 refinement, batched: every
    request converged to residualControl (p 1e-6) and its velocity within
    1e-5 relative L2 of the FP64 engine's converged velocity."""
    from gridfoam_b200.serving import BatchedEngine

    reqs = _converging_mix()
    out = {}
    for prec in ("float64", "float32"):
        eng = BatchedEngine(max_slots=4, max_outer=3000, keep_fields=True, inner_precision=prec)
        eng.prepare({r.n for r in reqs})
        out[prec] = {r.id: r for r in eng.run(reqs)}
    for req in reqs:
        a, b = out["float64"][req.id], out["float32"][req.id]
        assert a.converged and b.converged, (a.status, b.status)
        err = np.linalg.norm(b.U - a.U) / np.linalg.norm(a.U)
        assert err < 1e-5, (req.id, err)
