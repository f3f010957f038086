"""Doppler datasets on the GPU (pos2doppler / calc_doppler / chi2_doppler)
against the CPU oracle and the reference's golden vectors.

FP64 forms: facet maps bit-exact, fit spectra to 1e-12 of their peak, Doppler
limits exact (bins) / rtol 1e-12 (Hz), overflow terms (nonzero-bin count
exact, m2 rtol 1e-12), chi-square to 1e-10, flags exact. FP32 form:
chi-square to 1e-6."""
import json
import os

import numpy as np
import pytest

import cases
import golden_cases as gc
from shape_b200 import engine as eng
from shape_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_golden.json")))


def _dataset(name):
    model_fn, ds_fn, params = gc.DOPPLER_CASES[name]
    m = model_fn()
    ds = ds_fn(lambda d, p: cases.orc().eval_doppler(m, d, p)["fits"], params)
    return m, params, ds


@pytest.mark.parametrize("form", [eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64])
@pytest.mark.parametrize("name", sorted(gc.DOPPLER_CASES))
def test_doppler_fp64_matches_oracle_and_reference(cuda_device, name, form):
    m, p, ds = _dataset(name)
    o = cases.orc().eval_doppler(m, ds, p, keep_pos=True)
    g = GOLD["doppler"][name]
    e = eng.make_engine(m, p, dopplers=[ds])
    e.keep_pos(True)
    s = e.evaluate(form)
    res, ovf = e.results(), e.radar_overflow()
    for f, fr in enumerate(ds.frames):
        r, ro = res[f], o["results"][f]
        pg, po = e.pos(f), o["pos"][f]
        assert np.array_equal(pg["f"], po["f"]), (f, "facet map")
        fit, fo = e.fit(f), o["fits"][f]
        assert np.abs(fit - fo).max() <= 1e-12 * max(np.abs(fo).max(), 1e-300), (f, "fit")
        assert list(r["idoplim"]) == list(ro["idoplim"]), (f, r["idoplim"], ro["idoplim"])
        assert np.allclose(r["doplim"], ro["doplim"], rtol=1e-12, atol=0), f
        assert (r["badradar"], r["outbnd"]) == (ro["badradar"], ro["outbnd"]), f
        assert abs(r["badradar_logfactor"] - ro["badradar_logfactor"]) <= 1e-12 * max(1.0, abs(ro["badradar_logfactor"]))
        assert ovf[f][0] == g["frames"][f]["overflow_o2"], (f, ovf[f][0])
        assert abs(ovf[f][1] - g["frames"][f]["overflow_m2"]) <= 1e-12 * max(1e-300, abs(g["frames"][f]["overflow_m2"]))
        assert abs(r["chi2"] - ro["chi2"]) <= 1e-10 * abs(ro["chi2"]), (f, r["chi2"], ro["chi2"])
    chi2_o = sum(r["chi2"] for r in o["results"])
    assert abs(s["chi2"] - chi2_o) <= 1e-10 * chi2_o
    assert abs(s["chi2"] - g["chi2"]) <= 1e-10 * g["chi2"]
    assert s["badradar"] == g["flags"]["badradar"]
    assert abs(s["badradar_logfactor"] - g["flags"]["badradar_logfactor"]) <= 1e-12 * max(
        1.0, abs(g["flags"]["badradar_logfactor"]))
    e.close()


@pytest.mark.parametrize("name", ["dop_small", "dop_overflow"])
def test_doppler_fp32_tolerance(cuda_device, name):
    m, p, ds = _dataset(name)
    chi2_o = sum(r["chi2"] for r in cases.orc().eval_doppler(m, ds, p)["results"])
    e = eng.make_engine(m, p, dopplers=[ds])
    s = e.evaluate(eng.FORM_BATCHED_FP32)
    assert abs(s["chi2"] - chi2_o) <= 1e-6 * chi2_o, (s["chi2"], chi2_o)
    e.close()


def test_mixed_deldop_doppler_lightcurve(cuda_device):
    """All three dataset kinds in one engine: chi-square, dof-normalised flags
    and per-frame results in dataset order, every form."""
    m = gc.octa3_model()
    p = gc.P_DEFAULT
    dd = gc.DELDOP_CASES["small_long_orig"][1](cases.dd_synth(m), p)
    _, _, dp = _dataset("dop_overflow")
    lc = gc.LGHTCRV_CASES["kaasalainen"][1](cases.lc_synth(m), p)
    od = cases.orc().eval_deldop(m, dd, p)
    op = cases.orc().eval_doppler(m, dp, p)
    ol = cases.orc().eval_lghtcrv(m, lc, p)
    chi2_o = sum(r["chi2"] for r in od["results"]) + sum(r["chi2"] for r in op["results"]) + ol["chi2"]
    e = eng.make_engine(m, p, deldops=[dd], dopplers=[dp], lghtcrvs=[lc])
    for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
        s = e.evaluate(form)
        assert abs(s["chi2"] - chi2_o) <= 1e-10 * chi2_o, (form, s["chi2"], chi2_o)
        res = e.results()
        for k, r in enumerate(od["results"] + op["results"]):
            assert abs(res[k]["chi2"] - r["chi2"]) <= 1e-10 * abs(r["chi2"]), (form, k)
    s32 = e.evaluate(eng.FORM_BATCHED_FP32)
    assert abs(s32["chi2"] - chi2_o) <= 1e-6 * chi2_o
    e.close()
