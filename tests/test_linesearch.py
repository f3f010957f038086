"""The engine's bracketing, Brent minimiser and bestfit iteration (host code
in libshape_b200.so, no GPU needed) against the reference's own mnbrak /
brent_abs and a reference-driven config-1 fit (tests/golden/).

With identical objective values the trial sequences must be identical, so
the comparisons are exact."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import golden_cases as gc
from oracle.bindings import Oracle
from shape_b200 import engine as eng
from shape_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_golden.json")))

OBJ = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)
POBJ = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int))


class FitParam(C.Structure):
    _fields_ = [("kind", C.c_int), ("index", C.c_int), ("step", C.c_double), ("tol", C.c_double),
                ("abstol", C.c_double)]


class FitOptions(C.Structure):
    _fields_ = [("form", C.c_int), ("term_prec", C.c_double), ("term_maxiter", C.c_int)]


class FitResult(C.Structure):
    _fields_ = [("initial_objective", C.c_double), ("final_objective", C.c_double),
                ("iterations", C.c_int), ("evaluations", C.c_int), ("trace_len", C.c_int)]


def lib():
    L = eng.load_library()
    L.shape_bracket_minimum.argtypes = [OBJ, C.c_void_p] + [C.POINTER(C.c_double)] * 6
    L.shape_brent_minimize.argtypes = [OBJ, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.shape_bestfit_host.argtypes = [POBJ, C.c_void_p, C.POINTER(C.c_double), C.POINTER(FitParam), C.c_int,
                                     C.POINTER(FitOptions), C.POINTER(FitResult), C.POINTER(C.c_double), C.c_int]
    return L


@pytest.mark.parametrize("case", gc.LINESEARCH_CASES, ids=[c[0] for c in gc.LINESEARCH_CASES])
def test_line_searches_match_reference(case):
    name, fn, ax, bx, tol, abstol = case
    g = GOLD["linesearch"][name]
    L = lib()
    trials = []

    def f(x, _u):
        trials.append(x)
        return fn(x)
    cb = OBJ(f)
    a, b, c = C.c_double(ax), C.c_double(bx), C.c_double(0)
    fa, fb, fc = C.c_double(0), C.c_double(0), C.c_double(0)
    assert L.shape_bracket_minimum(cb, None, C.byref(a), C.byref(b), C.byref(c),
                                   C.byref(fa), C.byref(fb), C.byref(fc)) == 0
    assert [a.value, b.value, c.value, fa.value, fb.value, fc.value] == g["bracket"]
    assert len(trials) == g["n_mnbrak"]
    xmin, fmin = C.c_double(0), C.c_double(0)
    it = L.shape_brent_minimize(cb, None, a.value, b.value, c.value, tol, abstol, C.byref(xmin), C.byref(fmin))
    assert it >= 1
    assert trials == g["trials"]
    assert xmin.value == g["xmin"] and fmin.value == g["fmin"]


def test_bestfit_iteration_matches_reference_fit():
    """The bestfit loop with the CPU oracle as objective reproduces the
    reference-driven config-1 fit trial for trial."""
    g = GOLD["bestfit_c1"]
    orc = Oracle()
    m = synth.ellipsoid_model()
    p = synth.eval_params()
    ds = synth.config1_dataset(lambda d, pp: orc.eval_deldop(m, d, pp)["fits"], p)
    dof = sum(fr.dof for fr in ds.frames)

    def objective(values, _u, posbnd, badradar):
        mm = m.copy()
        mm.scale = np.array([values[0], values[1], values[2]])
        o = orc.eval_deldop(mm, ds, p)
        fl = {"posbnd": 0, "posbnd_logfactor": 0.0, "badradar": 0, "badradar_logfactor": 0.0}
        for r, fr in zip(o["results"], ds.frames):
            if r["outbnd"]:
                fl["posbnd"] = 1
                fl["posbnd_logfactor"] += fr.dof * r["posbnd_logfactor"]
            if r["badradar"]:
                fl["badradar"] = 1
                fl["badradar_logfactor"] += fr.dof * r["badradar_logfactor"]
        fl["posbnd_logfactor"] /= dof
        fl["badradar_logfactor"] /= dof
        posbnd[0], badradar[0] = fl["posbnd"], fl["badradar"]
        return gc.objective_from(sum(r["chi2"] for r in o["results"]), dof, fl)
    cb = POBJ(objective)
    values = (C.c_double * 3)(*gc.FIT_START)
    params = (FitParam * 3)(*[FitParam(*t) for t in gc.FIT_PARAMS])
    opt = FitOptions(0, gc.FIT_TERM_PREC, gc.FIT_MAXITER)
    res = FitResult()
    trace = (C.c_double * 2000)()
    rc = lib().shape_bestfit_host(cb, None, values, params, 3, C.byref(opt), C.byref(res), trace, 1000)
    assert rc == 0
    got = [[int(trace[2 * i]), trace[2 * i + 1]] for i in range(res.trace_len)]
    assert got == g["trace"]
    assert list(values) == g["values"]
    assert res.initial_objective == g["initial"] and res.final_objective == g["final"]
    assert res.iterations == g["iterations"]
