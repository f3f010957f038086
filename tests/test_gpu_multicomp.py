"""Models of several VERTEX components (shape_model_desc.ncomp > 1) against
the reference's realize_mod and calc_fits on the same components: each
component's vertices scaled by its own factors, rotated by its Euler angles
and translated by its offset (src/shape/realize_mod.c:444-512), posvis over
the components in order (src/shape/calc_fits.c:507-513).

Bars: realized vertices, normals and areas bit-exact; facet (model-wide
index), z and cos(e) maps bit-exact; chi-square to 1e-10 in the FP64 forms
and 1e-6 in FP32; after a scale change of the second component the same."""
import numpy as np
import pytest

import cases
from shape_b200 import engine as eng
from shape_b200 import synth

pytestmark = pytest.mark.gpu


def _ref():
    from oracle.bindings import Reference
    try:
        return Reference()
    except RuntimeError:
        pytest.skip("reference CPU build (oracle/_ref) not present")


def _dataset(ref, m, p):
    ds = synth.config1_frames(2, None, p)
    s = ref.session(m, p, deldops=[ds])
    s.evaluate()
    rng = np.random.default_rng(9)
    for f, fr in enumerate(ds.frames):
        fit = s.deldop_frame(0, f, fr)["fit"]
        ds.obs[ds.offsets[f]:ds.offsets[f + 1]] = 20.0 * fit / max(fit.max(), 1e-30) + rng.standard_normal(fit.size)
    return ds


def _check(e, s, m, ds, forms):
    rg, rr = e.realized(), s.realized()
    for k in ("x", "vn", "fn", "area"):
        assert np.array_equal(rg[k], rr[k]), k
    for form in forms:
        sm = e.evaluate(form)
        chi2_ref = s.evaluate()
        tol = 1e-6 if form == eng.FORM_BATCHED_FP32 else 1e-10
        assert abs(sm["chi2"] - chi2_ref) <= tol * chi2_ref, (form, sm["chi2"], chi2_ref)
        if form == eng.FORM_BATCHED_FP32:
            continue
        for f, fr in enumerate(ds.frames):
            rf = s.deldop_frame(0, f, fr)
            pg = e.pos(f)
            assert np.array_equal(pg["f"], rf["f"]), (form, f)
            assert np.array_equal(pg["z"], rf["z"]), (form, f)
            assert np.array_equal(pg["cose"], rf["cose"]), (form, f)
        assert np.array_equal(e.seen(), s.seen()), form


def test_two_components_match_reference(cuda_device):
    ref = _ref()
    m = synth.two_component_model()
    p = synth.eval_params()
    ds = _dataset(ref, m, p)
    s = ref.session(m, p, deldops=[ds])
    s.evaluate()
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    e.evaluate(eng.FORM_PLAIN_FP64)
    forms = (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64, eng.FORM_BATCHED_FP32)
    _check(e, s, m, ds, forms)
    # a size trial on the second component (SIZEPAR index 3..5)
    e.set_scale(4, 1.08)
    ref.lib.ref_set_scale(s.h, 4, 1.08)
    e.evaluate(eng.FORM_PLAIN_FP64)
    s.evaluate()
    _check(e, s, m, ds, forms)
    with pytest.raises(eng.EngineError):
        e.set_scale(6, 1.0)
    e.close()


def test_two_components_lightcurve(cuda_device):
    """A lightcurve of the two-component model: brightnesses (observer and
    sun views over both components, shadowing across them) to 1e-12."""
    ref = _ref()
    m = synth.two_component_model()
    p = synth.eval_params(mask_tol=0.0)
    lc = synth.lightcurve_dataset(12, (129, 161), None, p, set_index=0)
    s = ref.session(m, p, lghtcrvs=[lc])
    s.evaluate()
    want = s.lghtcrv(0, lc)
    e = eng.make_engine(m, p, lghtcrvs=[lc])
    for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64, eng.FORM_BATCHED_FP32):
        e.evaluate(form)
        got = e.lghtcrv(0, lc)
        np.testing.assert_allclose(got["y"], want["y"], rtol=1e-12, err_msg=str(form))
    e.close()
