"""Smeared delay-Doppler frames (several views per frame, the reference's
calc_deldop loop over views, src/shape/calc_fits.c:475-594).

CPU: the oracle's smeared frame against the reference compiled from its
sources (oracle/_ref), bit for bit: the fit is the mean over the views in
rendering order; posbnd, the limits, the POS maps and the seen marks are the
epoch view's; each view whose footprint is too wide adds dof * log-factor /
views to the badradar term.

GPU: the engine (shape_engine_add_deldop_set_views) against the same
reference: FP64 forms to the parity bars of the single-view frames (maps of
the epoch view bit-exact, fits to 1e-12 of the peak, chi-square to 1e-10),
the FP32 form to delta-chi2/chi2 < 1e-6.
"""
import math

import numpy as np
import pytest

import cases
from shape_b200 import synth


def _ref():
    from oracle.bindings import Reference
    try:
        return Reference()
    except RuntimeError:
        pytest.skip("reference CPU build (oracle/_ref) not present")


def _dataset(orc, m, p, nframes, nviews, v0, wide_view=False):
    ds = synth.smeared_dataset(nframes=nframes, nviews=nviews, v0=v0, params=p)
    if wide_view:
        # one non-epoch view of frame 0 spinning fast enough that its
        # Doppler footprint is too wide for the bin limit: badradar for that
        # view only
        w = ds.views[0][0]
        for j in range(3):
            w.spin[j] *= 300.0
    fits = orc.eval_deldop(m, ds, p)["fits"]
    rng = np.random.default_rng(5)
    for f in range(ds.nframes):
        ft = fits[f]
        ds.obs[ds.offsets[f]:ds.offsets[f + 1]] = 20.0 * ft / max(ft.max(), 1e-30) + rng.standard_normal(ft.size)
    return ds


def _ref_eval(ref, m, p, ds):
    s = ref.session(m, p, deldops=[ds])
    s.evaluate()
    frames = [s.deldop_frame(0, f, fr) for f, fr in enumerate(ds.frames)]
    return s, frames


CASES = [(2, 3, 1, False), (3, 2, 0, False), (2, 4, 3, True)]


@pytest.mark.parametrize("nframes,nviews,v0,wide", CASES)
def test_oracle_smearing_matches_reference(nframes, nviews, v0, wide):
    ref = _ref()
    orc = cases.orc()
    m = cases.c1()[0]
    p = synth.eval_params()
    if wide:
        p.nsinc2 = 3
    ds = _dataset(orc, m, p, nframes, nviews, v0, wide)
    o = orc.eval_deldop(m, ds, p, keep_pos=True)
    s, rf = _ref_eval(ref, m, p, ds)
    for f in range(ds.nframes):
        assert np.array_equal(o["fits"][f], rf[f]["fit"]), f
        assert np.array_equal(o["pos"][f]["z"], rf[f]["z"]), f
        assert np.array_equal(o["pos"][f]["f"].astype(np.int32), rf[f]["f"]), f
        ro, rr = o["results"][f], rf[f]["res"]
        for k in ("xlim", "ylim", "idellim", "idoplim"):
            assert list(ro[k]) == list(rr[k]), (f, k)
        assert ro["chi2"] == rr["chi2"], f
        assert ro["posbnd_logfactor"] == rr["posbnd_logfactor"], f
    assert np.array_equal(o["seen"], s.seen())
    fl = s.flags()
    dof = sum(fr.dof for fr in ds.frames)
    bany = any(r["badradar_any"] for r in o["results"])
    bterm = 0.0
    for r in o["results"]:
        bterm += r["badradar_term"]
    assert fl["badradar"] == int(bany)
    assert fl["badradar_logfactor"] == bterm / dof
    if wide:
        assert bany and not o["results"][0]["badradar"], "only a non-epoch view is too wide"


def test_smearing_changes_the_fit():
    """A smeared frame is not its epoch view alone."""
    orc = cases.orc()
    m = cases.c1()[0]
    p = synth.eval_params()
    ds = synth.smeared_dataset(nframes=1, nviews=3, v0=1, params=p)
    smeared = orc.eval_deldop(m, ds, p)["fits"][0]
    ds.views = None
    single = orc.eval_deldop(m, ds, p)["fits"][0]
    assert not np.array_equal(smeared, single)
    assert math.isclose(smeared.sum(), single.sum(), rel_tol=0.2)


def test_views_layout():
    ds = synth.smeared_dataset(nframes=2, nviews=3, v0=1)
    assert ds.nviews == 3
    arr = ds.view_array()
    assert len(arr) == 6
    for f in range(2):
        # the epoch view closes each frame's list
        assert list(arr[3 * f + 2].ae) == list(ds.frames[f].ae)


@pytest.mark.gpu
@pytest.mark.parametrize("nframes,nviews,v0,wide", CASES)
def test_engine_smearing_matches_reference(cuda_device, nframes, nviews, v0, wide):
    from shape_b200 import engine as eng
    ref = _ref()
    orc = cases.orc()
    m = cases.c1()[0]
    p = synth.eval_params()
    if wide:
        p.nsinc2 = 3
    ds = _dataset(orc, m, p, nframes, nviews, v0, wide)
    s, rf = _ref_eval(ref, m, p, ds)
    fl = s.flags()
    chi2_ref = sum(r["res"]["chi2"] for r in rf)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
        sm = e.evaluate(form)
        res = e.results()
        for f in range(ds.nframes):
            rr = rf[f]["res"]
            for k in ("xlim", "ylim", "idellim", "idoplim"):
                assert list(res[f][k]) == list(rr[k]), (form, f, k)
            assert abs(res[f]["chi2"] - rr["chi2"]) <= 1e-10 * abs(rr["chi2"]), (form, f)
            fit = e.fit(f)
            assert np.abs(fit - rf[f]["fit"]).max() <= 1e-11 * np.abs(rf[f]["fit"]).max(), (form, f)
            pg = e.pos(f)
            assert np.array_equal(pg["z"], rf[f]["z"]), (form, f)
            assert np.array_equal(pg["f"], rf[f]["f"]), (form, f)
        assert abs(sm["chi2"] - chi2_ref) <= 1e-10 * chi2_ref, form
        assert sm["badradar"] == fl["badradar"], form
        assert abs(sm["badradar_logfactor"] - fl["badradar_logfactor"]) <= 1e-13 * max(1.0, fl["badradar_logfactor"])
        assert np.array_equal(e.seen(), s.seen()), form
    s32 = e.evaluate(eng.FORM_BATCHED_FP32)
    assert abs(s32["chi2"] - chi2_ref) <= 1e-6 * chi2_ref
    e.close()


@pytest.mark.gpu
def test_engine_smearing_refuses_frame_views(cuda_device):
    from shape_b200 import engine as eng
    orc = cases.orc()
    m = cases.c1()[0]
    p = synth.eval_params()
    ds = _dataset(orc, m, p, 1, 3, 1)
    e = eng.make_engine(m, p, deldops=[ds])
    fr = ds.frames[0]
    with pytest.raises(eng.EngineError, match="several views"):
        e.set_frame_view(0, np.array(fr.ae).reshape(3, 3), np.array(fr.oe).reshape(3, 3), np.array(fr.spin), 0.0, 0.0)
    e.close()
