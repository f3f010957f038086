"""Plane-of-sky sets (shape_engine_add_poset_set) against the reference's own
calc_poset and chi2_poset (calc_fits + chi2 of oracle/_ref on the same
poset_t): each frame rendered from the observer and the sun, shadowed by
posmask, its brightness taken by apply_photo, resampled onto the fit grid by
resampim (no interpolation, nearest neighbour, bilinear and cubic
convolution, with and without rebinning, turned by the north angle and
shifted by the COM offsets), checked by checkposet, and compared with the
observed image under a floating calibration.

Bars: brightness images and fit images to 1e-12 of their peak (FP64 forms;
1e-9 in the FP32 form, whose lightcurve-view cosines are the FP64 form's),
calibration and frame chi-square to relative 1e-10 (1e-6 in FP32), the
badposet flag exactly and its log factor to 1e-12, the evaluation's chi2 and
objective to 1e-10 (1e-6)."""
import numpy as np
import pytest

from shape_b200 import engine as eng
from shape_b200 import synth

pytestmark = pytest.mark.gpu

FORMS = (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64, eng.FORM_BATCHED_FP32)

# (resample, rebin, fit-pixel width in rendering pixels, north angle)
CASES = {
    "bilinear_badposet": (2, False, 1.9, 0.35),
    "cubicconv_rebin": (4, True, 2.6, 0.35),
    "nearest_rebin": (1, True, 3.1, -0.5),
    "none_upright": (0, False, 1.0, 0.0),       # no interpolation: north up or a quarter turn
    "bilinear_rebin_small": (2, True, 0.6, 1.1),
}


def _ref():
    from oracle.bindings import Reference
    try:
        return Reference()
    except RuntimeError:
        pytest.skip("reference CPU build (oracle/_ref) not present")


def _dataset(R, m, p, case):
    mode, rebin, fs, na = CASES[case]

    def syn(ds, params):
        s = R.session(m, params, posets=[ds])
        s.evaluate()
        return [s.poset_frame(0, k, fr)[0] for k, fr in enumerate(ds.frames)]
    step = 0.5 * np.pi if mode == 0 else 0.2
    return synth.poset_dataset(synthesize=syn, params=p, resample=mode, rebin=rebin, fit_scale=fs, northangle=na,
                               northangle_step=step)


@pytest.mark.parametrize("case", sorted(CASES))
def test_poset_matches_reference(cuda_device, case):
    R = _ref()
    m = synth.ellipsoid_model()
    p = synth.eval_params()
    ds = _dataset(R, m, p, case)
    s = R.session(m, p, posets=[ds])
    chi2_ref = s.evaluate()
    bad_ref, badlf_ref = s.badposet()
    refs = [s.poset_frame(0, k, fr) for k, fr in enumerate(ds.frames)]
    e = eng.make_engine(m, p, posets=[ds])
    for form in FORMS:
        fp32 = form == eng.FORM_BATCHED_FP32
        tol_img, tol_chi = (1e-9, 1e-6) if fp32 else (1e-12, 1e-10)
        sm = e.evaluate(form)
        for k, fr in enumerate(ds.frames):
            fit, b, res = e.poset(0, k)
            rfit, rb, rcal, rchi2 = refs[k]
            assert np.abs(b - rb).max() <= tol_img * rb.max(), (case, form, k)
            assert np.abs(fit - rfit).max() <= tol_img * max(rfit.max(), 1e-300), (case, form, k)
            assert abs(res["cal"] - rcal) <= tol_chi * rcal, (case, form, k, res["cal"], rcal)
            assert abs(res["chi2"] - rchi2) <= tol_chi * rchi2, (case, form, k, res["chi2"], rchi2)
        assert abs(sm["chi2"] - chi2_ref) <= tol_chi * chi2_ref, (case, form, sm["chi2"], chi2_ref)
        assert abs(sm["chi2_poset"] - chi2_ref) <= tol_chi * chi2_ref
        assert sm["badposet"] == bad_ref, (case, form)
        if bad_ref:
            assert abs(sm["badposet_logfactor"] - badlf_ref) <= 1e-12 * abs(badlf_ref), (case, form)
            want = sm["chi2"] / sm["dof"] * 2.0 * np.exp(sm["badposet_logfactor"])
            assert abs(sm["objective"] - want) <= 1e-12 * want
    e.close()
    if case == "bilinear_badposet":
        assert bad_ref == 1
    if case == "cubicconv_rebin":
        assert bad_ref == 0


def test_poset_beside_radar_and_trial(cuda_device):
    """A delay-Doppler set and a plane-of-sky set in one evaluation: the
    chi-square sums in dataset order and each part equals the reference's;
    after a scale trial the same."""
    R = _ref()
    m = synth.ellipsoid_model()
    p = synth.eval_params()
    ds = _dataset(R, m, p, "cubicconv_rebin")
    dd = synth.config1_frames(1, None, p)
    s = R.session(m, p, deldops=[dd], posets=[ds])
    e = eng.make_engine(m, p, deldops=[dd], posets=[ds])
    for trial, scale in enumerate((None, 1.04)):
        if scale is not None:
            e.set_scale(1, scale)
            R.lib.ref_set_scale(s.h, 1, scale)
        chi2_ref = s.evaluate()
        for form in FORMS:
            tol = 1e-6 if form == eng.FORM_BATCHED_FP32 else 1e-10
            sm = e.evaluate(form)
            assert abs(sm["chi2"] - chi2_ref) <= tol * chi2_ref, (trial, form, sm["chi2"], chi2_ref)
            _, _, _, rchi2 = s.poset_frame(1, 0, ds.frames[0])
            _, _, res = e.poset(1, 0)
            assert abs(res["chi2"] - rchi2) <= tol * rchi2, (trial, form)
    e.close()


def test_poset_refusals(cuda_device):
    m = synth.ellipsoid_model()
    p = synth.eval_params()
    ds = synth.poset_dataset(resample=3)
    e = eng.Engine(0)
    e.set_model(m)
    e.set_params(p)
    with pytest.raises(eng.EngineError):
        e.add_poset(ds)
    e.close()
