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


def test_online_submit_poll(cuda_device):
    """Online use: requests submitted from two threads while others run,
    results collected by polling and waiting; each equals a lone evaluation.
    """
    import threading
    import time
    engines = _workloads()
    srv = eng.Server(device=0, hbm_budget_bytes=8 << 30, max_slots=4)
    for e, form in engines:
        srv.add_workload(e, form)
    srv.start()
    trace = eng.poisson_trace(48, 1500.0, len(engines), seed=9)
    tickets = [None] * len(trace)

    def submitter(lo, hi):
        for i in range(lo, hi):
            w, _, sc = trace[i]
            tickets[i] = srv.submit(w, sc)
            time.sleep(0.0005)
    th = [threading.Thread(target=submitter, args=(0, 24)), threading.Thread(target=submitter, args=(24, 48))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    res = []
    for i, tk in enumerate(tickets):
        r = srv.poll(tk) if i % 2 else None
        res.append(r if r is not None else srv.wait(tk, 60.0))
    st = srv.stats()
    srv.stop()
    assert st["requests_per_s"] > 0 and st["p99_latency_s"] >= st["p50_latency_s"] > 0.0
    _check(engines, trace, res)
    with pytest.raises(eng.EngineError):
        srv.submit(0)                      # stopped: no scheduler to serve it
    srv.close()


def test_no_head_of_line_blocking(cuda_device):
    """A request that cannot be admitted (its workload's instance is busy
    and the budget has no room for a second one) does not hold up a later
    request of a workload with an idle instance."""
    m2, p2, d2 = cases.c2(64)
    m1, p1, d1 = cases.c1()
    big = eng.make_engine(m2, p2, deldops=[d2])
    small = eng.make_engine(m1, p1, deldops=[d1])
    probe = eng.Server(device=0, hbm_budget_bytes=8 << 30, max_slots=4)
    wb = probe.add_workload(big, eng.FORM_BATCHED_FP64)
    ws = probe.add_workload(small, eng.FORM_PLAIN_FP64)
    need_big, need_small = probe.workload_bytes(wb), probe.workload_bytes(ws)
    probe.close()
    # one instance of each fits, a second instance of the big workload does not
    srv = eng.Server(device=0, hbm_budget_bytes=need_big + need_small + need_small // 2, max_slots=4)
    srv.add_workload(big, eng.FORM_BATCHED_FP64)
    srv.add_workload(small, eng.FORM_PLAIN_FP64)
    trace = [(0, 0.0, (1.0, 1.0, 1.0)), (0, 0.0, (1.01, 1.0, 1.0)), (1, 0.0, (1.0, 1.0, 1.0))]
    res, st = srv.run(trace)
    # the small request started before the second big one
    assert res[2]["t_start"] < res[1]["t_start"], [r["t_start"] for r in res]
    _check([(big, eng.FORM_BATCHED_FP64), (small, eng.FORM_PLAIN_FP64)], trace, res)
    srv.close()
