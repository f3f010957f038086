"""Parity of the B200 engine (called through its C ABI) with the CPU oracle.

Bars (from the engine's contract):
  - FP64 forms: realized model, facet / z / cos(e) maps and POS limits
    bit-exact; fit images to rtol 1e-12 (only the order of the scatter-add
    differs); frame chi-square to relative 1e-10;
  - FP32 form: total delta-chi2/chi2 < 1e-6 against the FP64 oracle.
"""
import numpy as np
import pytest

import cases
from shape_b200 import engine as eng
from shape_b200 import synth

pytestmark = pytest.mark.gpu

CHI2_RTOL = 1e-10
FIT_RTOL = 1e-12
FP32_CHI2_RTOL = 1e-6


def _frame_checks(e, o, ds, exact_pos=True, frames=None):
    res = e.results()
    frames = range(ds.nframes) if frames is None else frames
    for f in frames:
        ro, rg = o["results"][f], res[f]
        for k in ("outbnd", "badradar", "xlim", "ylim", "idellim", "idoplim"):
            assert ro[k] == rg[k], (f, k, ro[k], rg[k])
        for k in ("dellim", "doplim"):
            np.testing.assert_allclose(rg[k], ro[k], rtol=1e-12, atol=1e-9, err_msg="frame %d %s" % (f, k))
        assert abs(rg["posbnd_logfactor"] - ro["posbnd_logfactor"]) <= 1e-12 * max(1.0, abs(ro["posbnd_logfactor"]))
        assert abs(rg["chi2"] - ro["chi2"]) <= CHI2_RTOL * abs(ro["chi2"]), (f, rg["chi2"], ro["chi2"])
        fit = e.fit(f)
        scale = max(np.abs(o["fits"][f]).max(), 1e-300)
        assert np.abs(fit - o["fits"][f]).max() <= FIT_RTOL * scale * 10, f
        if exact_pos:
            pg, po = e.pos(f), o["pos"][f]
            assert np.array_equal(pg["f"], po["f"]), "facet map differs in frame %d" % f
            assert np.array_equal(pg["z"], po["z"]), "z map differs in frame %d" % f
            assert np.array_equal(pg["cose"], po["cose"]), "cos(e) map differs in frame %d" % f


def test_realize_bit_exact(cuda_device):
    m, p, ds = cases.c1()
    o = cases.orc()
    e = eng.make_engine(m, p, deldops=[ds])
    e.evaluate(eng.FORM_PLAIN_FP64)
    rg, ro = e.realized(), o.realize(m)
    for k in ("x", "vn", "fn", "area"):
        assert np.array_equal(rg[k], ro[k]), k
    e.close()


@pytest.mark.parametrize("form", [eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64])
def test_config1_fp64_exact(cuda_device, form):
    m, p, ds = cases.c1()
    o = cases.orc().eval_deldop(m, ds, p, keep_pos=True)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    s = e.evaluate(form)
    _frame_checks(e, o, ds)
    chi2_o = sum(r["chi2"] for r in o["results"])
    assert abs(s["chi2"] - chi2_o) <= CHI2_RTOL * chi2_o
    assert np.array_equal(e.seen(), o["seen"])
    e.close()


def test_config2_subset_fp64_exact(cuda_device):
    m, p, ds = cases.c2(12)
    o = cases.orc().eval_deldop(m, ds, p, keep_pos=True)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    e.evaluate(eng.FORM_BATCHED_FP64)
    _frame_checks(e, o, ds)
    e.evaluate(eng.FORM_PLAIN_FP64)
    _frame_checks(e, o, ds)
    e.close()


def test_config2_fp32_tolerance(cuda_device):
    m, p, ds = cases.c2(64)
    o = cases.orc().eval_deldop(m, ds, p)
    chi2_o = sum(r["chi2"] for r in o["results"])
    e = eng.make_engine(m, p, deldops=[ds])
    s64 = e.evaluate(eng.FORM_BATCHED_FP64)
    assert abs(s64["chi2"] - chi2_o) <= CHI2_RTOL * chi2_o
    s32 = e.evaluate(eng.FORM_BATCHED_FP32)
    rel = abs(s32["chi2"] - chi2_o) / chi2_o
    per_frame = [abs(a["chi2"] - b["chi2"]) / b["chi2"] for a, b in zip(e.results(), o["results"])]
    print("FP32 total rel err %.3e, worst frame %.3e" % (rel, max(per_frame)))
    assert rel < FP32_CHI2_RTOL
    e.close()


@pytest.mark.parametrize("case", ["c1", "c2_12"])
def test_fp32_exact_option_radar_maps(cuda_device, case):
    """shape_engine_set_fp32_exact(1): radar views' facet and depth maps in
    the batched FP32 form equal the oracle's (pixels with a decision within
    FP32 error redone by the FP64 rules, FP64 depths), at jittered scale
    factors too; chi-square within the FP32 bar."""
    m, p, ds = cases.c1() if case == "c1" else cases.c2(12)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    e.set_fp32_exact(True)
    rng = np.random.default_rng(11)
    for trial in range(3):
        sc = [1.0, 1.0, 1.0] if trial == 0 else list(1.0 + 0.02 * rng.uniform(-1, 1, 3))
        for j in range(3):
            e.set_scale(j, sc[j])
        mm = cases.scaled_model(m, sc)
        o = cases.orc().eval_deldop(mm, ds, p, keep_pos=True)
        s = e.evaluate(eng.FORM_BATCHED_FP32)
        for f in range(ds.nframes):
            pg, po = e.pos(f), o["pos"][f]
            assert np.array_equal(pg["f"], po["f"]), (trial, f, "facet map")
            assert np.array_equal(pg["z"], po["z"]), (trial, f, "z map")
        chi2_o = sum(r["chi2"] for r in o["results"])
        assert abs(s["chi2"] - chi2_o) <= FP32_CHI2_RTOL * chi2_o, (trial, s["chi2"], chi2_o)
    e.close()


def test_lightcurve_fp64_exact(cuda_device):
    m, p, sets = cases.c3(12, 2)
    o = cases.orc()
    e = eng.make_engine(m, p, lghtcrvs=sets)
    e.keep_pos(True)
    s = e.evaluate(eng.FORM_PLAIN_FP64)
    tot = 0.0
    for k, ds in enumerate(sets):
        oo = o.eval_lghtcrv(m, ds, p, keep_pos=True)
        g = e.lghtcrv(k, ds)
        np.testing.assert_allclose(g["y"], oo["y"], rtol=1e-12)
        np.testing.assert_allclose(g["fit"], oo["fit"], rtol=1e-12)
        assert abs(g["chi2"] - oo["chi2"]) <= CHI2_RTOL * abs(oo["chi2"])
        tot += oo["chi2"]
        for i, pt in enumerate(ds.points):
            pg, po = e.lghtcrv_pos(k, i, pt), oo["pos"][i]
            for key in ("f", "z", "cose", "cosi", "zill", "fill"):
                assert np.array_equal(pg[key], po[key]), (k, i, key)
    assert abs(s["chi2"] - tot) <= CHI2_RTOL * tot
    s2 = e.evaluate(eng.FORM_BATCHED_FP64)
    assert abs(s2["chi2"] - tot) <= CHI2_RTOL * tot
    # FP32 form: the lightcurve views' facet assignment, depths and shadow
    # inputs follow the FP64 rules (decisions within FP32 error are redone
    # in FP64), so the facet maps equal the oracle's, and their cos(e) /
    # cos(i) are recomputed in FP64 from each pixel's good facet, so the
    # brightnesses and the chi-square (a small difference of large sums with
    # 1% noise, which magnifies any rounding of the cosines) are the FP64
    # forms': y to 1e-12, chi-square to 1e-10.
    s3 = e.evaluate(eng.FORM_BATCHED_FP32)
    worst = 0.0
    for k, ds in enumerate(sets):
        oo = o.eval_lghtcrv(m, ds, p, keep_pos=True)
        g = e.lghtcrv(k, ds)
        worst = max(worst, float(np.max(np.abs(g["y"] - oo["y"]) / np.abs(oo["y"]))))
        for i, pt in enumerate(ds.points):
            pg, po = e.lghtcrv_pos(k, i, pt), oo["pos"][i]
            assert np.array_equal(pg["f"], po["f"]), (k, i, "f")
            assert np.array_equal(pg["fill"], po["fill"]), (k, i, "fill")
            assert np.array_equal(pg["z"], po["z"]), (k, i, "z")
            assert np.array_equal(pg["cose"], po["cose"]), (k, i, "cose")
            assert np.array_equal(pg["cosi"], po["cosi"]), (k, i, "cosi")
    print("FP32 lightcurve worst per-point relative error %.3e, chi2 %.3e" % (worst, abs(s3["chi2"] - tot) / tot))
    assert worst < 1e-12
    assert abs(s3["chi2"] - tot) / tot < CHI2_RTOL
    e.close()


@pytest.mark.parametrize("codemethod,spb,stride,nsinc2", [
    (0, 1, 1, 1), (2, 2, 1, 2), (2, 3, 1, 3), (1, 2, 2, 1), (0, 4, 2, 2)])
def test_codemethods_fp64(cuda_device, codemethod, spb, stride, nsinc2):
    m = cases.c2_model()
    p = synth.eval_params(nsinc2=nsinc2, sinc2width=7)
    ds = cases.small_frames(m, p, 3, (61, 101), codemethod=codemethod, spb=spb, stride=stride)
    ds.set.dopfftlen = 64
    o = cases.orc().eval_deldop(m, ds, p, keep_pos=True)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    e.evaluate(eng.FORM_BATCHED_FP64)
    _frame_checks(e, o, ds)
    e.close()


@pytest.mark.parametrize("codemethod,spb,stride,nsinc2", [
    (0, 1, 1, 1), (2, 1, 1, 1), (2, 2, 1, 2), (2, 3, 1, 3), (1, 2, 2, 1), (0, 4, 2, 2)])
def test_codemethods_fp32(cuda_device, codemethod, spb, stride, nsinc2):
    """Batched FP32 over the code methods: the vector path (LONG_ORIG or
    spb = 1, nsinc2 = 1) and the general path (the others) within the FP32
    chi-square bar."""
    m = cases.c2_model()
    p = synth.eval_params(nsinc2=nsinc2, sinc2width=7)
    ds = cases.small_frames(m, p, 3, (61, 101), codemethod=codemethod, spb=spb, stride=stride)
    ds.set.dopfftlen = 64
    o = cases.orc().eval_deldop(m, ds, p)
    chi2_o = sum(r["chi2"] for r in o["results"])
    e = eng.make_engine(m, p, deldops=[ds])
    s = e.evaluate(eng.FORM_BATCHED_FP32)
    assert abs(s["chi2"] - chi2_o) <= FP32_CHI2_RTOL * chi2_o, (s["chi2"], chi2_o)
    e.close()


@pytest.mark.parametrize("law", [2, 3, 4, 5, 6, 7])
def test_radar_laws_fp64(cuda_device, law):
    m = cases.c2_model()
    p = synth.eval_params()
    ds = cases.small_frames(m, p, 2, (61, 81), law=cases.radar_law(law))
    o = cases.orc().eval_deldop(m, ds, p, keep_pos=True)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    e.evaluate(eng.FORM_PLAIN_FP64)
    _frame_checks(e, o, ds)
    e.close()


def test_outbnd_and_bin_overflow(cuda_device):
    """A POS window smaller than the model (posbnd path) and a single 9x9 tile
    holding more facets than a bin can (ordered full-scan path)."""
    m, _, _ = cases.c1()
    p = synth.eval_params()
    ds = synth.config1_dataset(cases.dd_synth(m), p)
    fr = ds.frames[0]
    fr.pos_n = 40           # window of 81 px: model (~130 px across) overflows
    ds2 = synth.config1_dataset(cases.dd_synth(m), p)
    ds2.frames[0].pos_n = 4
    ds2.frames[0].km_per_pixel = 0.3   # 9x9 px: ~1150 visible facets in one tile
    for d in (ds, ds2):
        o = cases.orc().eval_deldop(m, d, p, keep_pos=True)
        assert o["results"][0]["outbnd"] == (1 if d is ds else 0) or d is ds2
        for cap in (0, 64):            # autotuned bins, then bins that overflow
            e = eng.Engine()
            e.set_model(m)
            e.set_params(p)
            e.add_deldop(d)
            e.set_bin_capacity(cap)
            e.finalize()
            if cap:
                assert e.tuning()["max_bin"] > cap
            e.keep_pos(True)
            for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
                e.evaluate(form)
                _frame_checks(e, o, d)
            e.close()


def test_param_update_graph_replay(cuda_device):
    """Scale-factor trials through the captured graph match fresh evaluations."""
    m, p, ds = cases.c1()
    e = eng.make_engine(m, p, deldops=[ds])
    vals = []
    for sc in (1.0, 1.05, 0.97):
        e.set_scale(0, sc)
        e.set_scale(2, 2.0 - sc)
        a = e.evaluate(eng.FORM_BATCHED_FP64)["chi2"]
        b = e.evaluate(eng.FORM_PLAIN_FP64)["chi2"]
        mm = m.copy()
        mm.scale = np.array([sc, 1.0, 2.0 - sc])
        o = cases.orc().eval_deldop(mm, ds, p)
        c = o["results"][0]["chi2"]
        assert abs(a - c) <= CHI2_RTOL * c and abs(b - c) <= CHI2_RTOL * c
        vals.append(a)
    assert len(set(vals)) == 3
    e.close()


@pytest.mark.parametrize("form", [eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64, eng.FORM_BATCHED_FP32])
def test_lightcurve_off_knots(cuda_device, form):
    """Observation epochs strictly between the calculated ones (the golden
    case kaasalainen_off_knots, pinned bit-exact to the reference's
    calc_lghtcrv): every fit value is the natural spline off its knots.
    FP64 forms: y and fit to rtol 1e-12, chi-square 1e-10 against the oracle;
    FP32 form: per-point and chi-square error below 1e-6."""
    import golden_cases as gc
    model_fn, ds_fn, params = gc.LGHTCRV_CASES["kaasalainen_off_knots"]
    m = model_fn()
    o = cases.orc()
    ds = ds_fn(lambda d, p: o.eval_lghtcrv(m, d, p)["y"], params)
    assert ds.set.n == ds.set.ncalc - 1 and np.all((ds.t > ds.x[:-1]) & (ds.t < ds.x[1:]))
    oo = o.eval_lghtcrv(m, ds, params)
    e = eng.make_engine(m, params, lghtcrvs=[ds])
    s = e.evaluate(form)
    g = e.lghtcrv(0, ds)
    if form == eng.FORM_BATCHED_FP32:
        err = np.max(np.abs(g["fit"] - oo["fit"]) / np.abs(oo["fit"]))
        print("FP32 off-knot worst per-point relative error %.3e" % err)
        assert err < 1e-6
        assert abs(s["chi2"] - oo["chi2"]) <= FP32_CHI2_RTOL * abs(oo["chi2"])
    else:
        np.testing.assert_allclose(g["y"], oo["y"], rtol=1e-12)
        np.testing.assert_allclose(g["fit"], oo["fit"], rtol=1e-12)
        assert abs(s["chi2"] - oo["chi2"]) <= CHI2_RTOL * abs(oo["chi2"])
    e.close()
