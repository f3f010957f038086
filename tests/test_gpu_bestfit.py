"""bestfit on the device (each trial a device evaluation; a graph replay in
the batched forms) against the reference-driven config-1 fit in
tests/golden/: the FP64 objective agrees with the reference to ~1e-14, so
the line searches take the same decisions and visit the same trial values."""
import json
import os

import numpy as np
import pytest

import golden_cases as gc
from shape_b200 import engine as eng
from shape_b200 import synth

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_golden.json")))


@pytest.mark.parametrize("form", [eng.FORM_BATCHED_FP64, eng.FORM_PLAIN_FP64])
def test_device_bestfit_matches_reference_fit(cuda_device, form):
    import cases
    g = GOLD["bestfit_c1"]
    m, p, ds = cases.c1()
    e = eng.make_engine(m, p, deldops=[ds])
    for j, v in enumerate(gc.FIT_START):
        e.set_scale(j, v)
    res, trace = e.bestfit(gc.FIT_PARAMS, form=form, term_prec=gc.FIT_TERM_PREC,
                           term_maxiter=gc.FIT_MAXITER, trace_max=1000)
    assert len(trace) == len(g["trace"])
    for (k, x), (gk, gx) in zip(trace, g["trace"]):
        assert k == gk and abs(x - gx) <= 1e-9 * max(1.0, abs(gx))
    for j in range(3):
        assert abs(e.get_scale(j) - g["values"][j]) <= 1e-9
    assert abs(res["final_objective"] - g["final"]) <= 1e-10 * g["final"]
    assert res["iterations"] == g["iterations"]
    e.close()


def test_fp32_bestfit_converges_to_fp64_minimum(cuda_device):
    """The batched FP32 form drives the same fit to the same parameters
    within the FP32 objective's resolution."""
    import cases
    g = GOLD["bestfit_c1"]
    m, p, ds = cases.c1()
    e = eng.make_engine(m, p, deldops=[ds])
    for j, v in enumerate(gc.FIT_START):
        e.set_scale(j, v)
    res, _ = e.bestfit(gc.FIT_PARAMS, form=eng.FORM_BATCHED_FP32, term_prec=gc.FIT_TERM_PREC,
                       term_maxiter=gc.FIT_MAXITER)
    assert abs(res["final_objective"] - g["final"]) <= 1e-5 * g["final"]
    e.close()
