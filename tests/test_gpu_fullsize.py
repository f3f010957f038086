"""Full-size parity of the engine (through its C ABI) with the CPU oracle.

FP64 forms: config 4 (16 frames of 511x511 POS and 256x256 delay-Doppler,
32768-facet model) and config 3 (4 lightcurves x 200 points, two views per
point with shadowing) at their full sizes: facet / z / cos(e) maps
bit-exact, fit images and lightcurve values to rtol 1e-12, chi-square to
1e-10.

Default batched FP32 form (no switches): delta-chi2/chi2 below 1e-6 against
the FP64 oracle, in total and in every frame, on config 1 under +-2% scale
jitter, config 3 and config 4 at full size and the serving mix's request
kinds (config-1 model with 1-4 frames, config-4 model with 1-2 frames,
config-2 model with 8 frames, jittered). Each case prints its worst
per-frame error.
"""
import numpy as np
import pytest

import cases
from shape_b200 import engine as eng
from shape_b200 import synth

pytestmark = pytest.mark.gpu

CHI2_RTOL = 1e-10
FIT_RTOL = 1e-12
FP32_RTOL = 1e-6


def _c4():
    m = synth.noisy_octa_model()
    p = synth.eval_params()
    return m, p, synth.config4_dataset(cases.dd_synth(m), p)


def _c3():
    m = cases.c2_model()
    p = synth.eval_params(mask_tol=0.0)
    return m, p, synth.config3_datasets(cases.lc_synth(m), p)


@pytest.fixture(scope="module")
def c4():
    return _c4()


@pytest.fixture(scope="module")
def c3():
    return _c3()


def _fp32_check(tag, e, o_results, s32):
    """Total and per-frame delta-chi2/chi2 of an FP32 evaluation against the
    oracle's per-frame results."""
    chi2_o = sum(r["chi2"] for r in o_results)
    tot = abs(s32["chi2"] - chi2_o) / chi2_o
    per = [abs(a["chi2"] - b["chi2"]) / b["chi2"] for a, b in zip(e.results(), o_results)]
    print("%s: FP32 delta-chi2/chi2 total %.3e, worst frame %.3e (frame %d of %d)"
          % (tag, tot, max(per), int(np.argmax(per)), len(per)))
    assert tot < FP32_RTOL, (tag, tot)
    assert max(per) < FP32_RTOL, (tag, per)


@pytest.mark.parametrize("form", [eng.FORM_BATCHED_FP64, eng.FORM_PLAIN_FP64])
def test_config4_full_fp64_exact(cuda_device, c4, form):
    m, p, ds = c4
    o = cases.orc().eval_deldop(m, ds, p, keep_pos=True)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    s = e.evaluate(form)
    res = e.results()
    for f in range(ds.nframes):
        ro, rg = o["results"][f], res[f]
        for k in ("outbnd", "badradar", "xlim", "ylim", "idellim", "idoplim"):
            assert ro[k] == rg[k], (f, k)
        assert abs(rg["chi2"] - ro["chi2"]) <= CHI2_RTOL * abs(ro["chi2"]), f
        fit = e.fit(f)
        assert np.abs(fit - o["fits"][f]).max() <= FIT_RTOL * 10 * np.abs(o["fits"][f]).max(), f
        pg, po = e.pos(f), o["pos"][f]
        assert np.array_equal(pg["f"], po["f"]), f
        assert np.array_equal(pg["z"], po["z"]), f
        assert np.array_equal(pg["cose"], po["cose"]), f
    chi2_o = sum(r["chi2"] for r in o["results"])
    assert abs(s["chi2"] - chi2_o) <= CHI2_RTOL * chi2_o
    assert np.array_equal(e.seen(), o["seen"])
    e.close()


@pytest.mark.parametrize("form", [eng.FORM_BATCHED_FP64, eng.FORM_PLAIN_FP64])
def test_config3_full_fp64(cuda_device, c3, form):
    """All 800 points' y and fit to 1e-12, each set's chi-square to 1e-10,
    and the observer / sun maps of every 40th point bit-exact."""
    m, p, sets = c3
    orc = cases.orc()
    e = eng.make_engine(m, p, lghtcrvs=sets)
    e.keep_pos(True)
    s = e.evaluate(form)
    tot = 0.0
    for k, ds in enumerate(sets):
        oo = orc.eval_lghtcrv(m, ds, p)
        g = e.lghtcrv(k, ds)
        np.testing.assert_allclose(g["y"], oo["y"], rtol=1e-12)
        np.testing.assert_allclose(g["fit"], oo["fit"], rtol=1e-12)
        assert abs(g["chi2"] - oo["chi2"]) <= CHI2_RTOL * abs(oo["chi2"])
        tot += oo["chi2"]
        # maps of every 40th point: the oracle on a set of just those points
        # (each point's maps depend on its own views only)
        sample = list(range(0, len(ds.points), 40))
        sset = type(ds.set).from_buffer_copy(ds.set)
        sset.ncalc = sset.n = len(sample)
        sub = synth.LightcurveDataset(sset, [ds.points[i] for i in sample], ds.x[sample].copy(),
                                      ds.x[sample].copy(), np.ones(len(sample)), np.ones(len(sample)))
        sub.bind()
        so = orc.eval_lghtcrv(m, sub, p, keep_pos=True)
        for j, i in enumerate(sample):
            pg, po = e.lghtcrv_pos(k, i, ds.points[i]), so["pos"][j]
            for key in ("f", "z", "cose", "cosi", "zill", "fill"):
                assert np.array_equal(pg[key], po[key]), (k, i, key)
    assert abs(s["chi2"] - tot) <= CHI2_RTOL * tot
    e.close()


def test_config4_full_fp32_default(cuda_device, c4):
    m, p, ds = c4
    e = eng.make_engine(m, p, deldops=[ds])
    rng = np.random.default_rng(44)
    for trial in range(3):
        sc = [1.0, 1.0, 1.0] if trial == 0 else list(1.0 + 0.02 * rng.uniform(-1, 1, 3))
        for j in range(3):
            e.set_scale(j, sc[j])
        o = cases.orc().eval_deldop(cases.scaled_model(m, sc), ds, p)
        _fp32_check("config 4 trial %d" % trial, e, o["results"], e.evaluate(eng.FORM_BATCHED_FP32))
    e.close()


def test_config3_full_fp32_default(cuda_device, c3):
    m, p, sets = c3
    orc = cases.orc()
    e = eng.make_engine(m, p, lghtcrvs=sets)
    s = e.evaluate(eng.FORM_BATCHED_FP32)
    tot, worst_pt, worst_set = 0.0, 0.0, 0.0
    for k, ds in enumerate(sets):
        oo = orc.eval_lghtcrv(m, ds, p)
        g = e.lghtcrv(k, ds)
        worst_pt = max(worst_pt, float(np.max(np.abs(g["y"] - oo["y"]) / np.abs(oo["y"]))))
        worst_set = max(worst_set, abs(g["chi2"] - oo["chi2"]) / abs(oo["chi2"]))
        tot += oo["chi2"]
    rel = abs(s["chi2"] - tot) / tot
    print("config 3: FP32 delta-chi2/chi2 total %.3e, worst set %.3e, worst point y %.3e"
          % (rel, worst_set, worst_pt))
    assert rel < FP32_RTOL and worst_set < FP32_RTOL and worst_pt < FP32_RTOL
    e.close()


def test_config1_fp32_default_jitter(cuda_device):
    """24 trials at scale factors 1 +- 2% (the serving mix's jitter and more
    than a fit's steps): every trial within the bar."""
    m, p, ds = cases.c1()
    e = eng.make_engine(m, p, deldops=[ds])
    rng = np.random.default_rng(2024)
    for trial in range(24):
        sc = list(1.0 + 0.02 * rng.uniform(-1, 1, 3))
        for j in range(3):
            e.set_scale(j, sc[j])
        o = cases.orc().eval_deldop(cases.scaled_model(m, sc), ds, p)
        _fp32_check("config 1 trial %d" % trial, e, o["results"], e.evaluate(eng.FORM_BATCHED_FP32))
    e.close()


@pytest.mark.parametrize("kind,nframes", [("c1", 1), ("c1", 2), ("c1", 4), ("c4", 1), ("c4", 2), ("c2", 8)])
def test_serving_kinds_fp32_default(cuda_device, c4, kind, nframes):
    """The serving mix's request kinds (a model with its first frames) at
    jittered scale factors, as the mix draws them."""
    p = synth.eval_params()
    if kind == "c1":
        m = synth.ellipsoid_model()
        full = synth.config1_frames(4, cases.dd_synth(m), p)
    elif kind == "c4":
        m, _, full = c4
    else:
        m, _, full = cases.c2(64)
    ds = synth.frame_prefix(full, nframes)
    e = eng.make_engine(m, p, deldops=[ds])
    rng = np.random.default_rng(7 + nframes)
    for trial in range(4):
        sc = list(1.0 + 0.02 * rng.uniform(-1, 1, 3))
        for j in range(3):
            e.set_scale(j, sc[j])
        o = cases.orc().eval_deldop(cases.scaled_model(m, sc), ds, p)
        _fp32_check("%s x%d trial %d" % (kind, nframes, trial), e, o["results"], e.evaluate(eng.FORM_BATCHED_FP32))
    e.close()
