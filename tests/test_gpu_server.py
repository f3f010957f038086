"""Continuous-batching server (shape_server_*): every request's result in a
mixed Poisson trace equals a lone evaluation of its workload at its scale
factors, with and without HBM-budget evictions.

Tolerances: batched forms accumulate radar bins with float atomics whose
order varies between runs, so FP64 results agree to 1e-12 relative and FP32
ones to 1e-6 relative; the plain FP64 form is deterministic."""
import pytest

import cases
from shape_b200 import engine as eng

pytestmark = pytest.mark.gpu

TOL = {eng.FORM_PLAIN_FP64: 1e-12, eng.FORM_BATCHED_FP64: 1e-12, eng.FORM_BATCHED_FP32: 1e-6}


def _workloads():
    m1, p1, d1 = cases.c1()
    m2, p2, d2 = cases.c2(16)
    m3, p3, s3 = cases.c3(8, 1)
    return [
        (eng.make_engine(m1, p1, deldops=[d1]), eng.FORM_PLAIN_FP64),
        (eng.make_engine(m2, p2, deldops=[d2]), eng.FORM_BATCHED_FP32),
        (eng.make_engine(m2, p2, deldops=[d2]), eng.FORM_BATCHED_FP64),
        (eng.make_engine(m3, p3, lghtcrvs=s3), eng.FORM_BATCHED_FP32),
    ]


def _alone(engines, trace):
    out = []
    for w, _, sc in trace:
        e, form = engines[w]
        for j in range(3):
            e.set_scale(j, sc[j])
        s = e.evaluate(form)
        out.append((s["chi2"], s["objective"]))
    return out


def _check(engines, trace, res):
    alone = _alone(engines, trace)
    for (w, _, _), r, (c2, obj) in zip(trace, res, alone):
        tol = TOL[engines[w][1]]
        assert abs(r["chi2"] - c2) <= tol * abs(c2), (w, r["chi2"], c2)
        assert abs(r["objective"] - obj) <= tol * abs(obj), (w, r["objective"], obj)
        assert r["latency_s"] >= 0.0 and r["t_done"] >= r["t_start"]


def test_mixed_trace_matches_lone_evaluations(cuda_device):
    engines = _workloads()
    srv = eng.Server(device=0, hbm_budget_bytes=8 << 30, max_slots=6)
    for e, form in engines:
        srv.add_workload(e, form)
    trace = eng.poisson_trace(60, 2000.0, len(engines), seed=3)
    res, st = srv.run(trace)
    assert st["peak_concurrency"] >= 2           # requests overlapped
    assert st["instances_evicted"] == 0
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0.0
    _check(engines, trace, res)
    srv.close()


def test_budget_evictions_keep_results(cuda_device):
    engines = _workloads()
    srv = eng.Server(device=0, hbm_budget_bytes=8 << 30, max_slots=4)
    sizes = [srv.add_workload(e, form) for e, form in engines]
    assert sizes == list(range(len(engines)))
    need = [srv.workload_bytes(w) for w in range(len(engines))]
    srv.close()
    # room for the largest instance plus a little: workloads must take turns
    budget = max(need) + min(need) // 2
    srv = eng.Server(device=0, hbm_budget_bytes=budget, max_slots=4)
    for e, form in engines:
        srv.add_workload(e, form)
    trace = eng.poisson_trace(40, 1000.0, len(engines), seed=5)
    res, st = srv.run(trace)
    assert st["instances_evicted"] > 0
    assert st["peak_hbm_bytes"] <= budget
    _check(engines, trace, res)
    srv.close()
