"""Penalty terms of the objective (shape_engine_set_penalties) against the
reference's own penalties() (ref_penalties, compiled from the reference's
sources and run on the CPU) on the same realized model: every supported
penalty's value to 1e-9 relative (1e-14 absolute; the engine sums the
moments and edge terms in another order and diagonalizes the inertia
tensor with its own Jacobi rotations), in every form; and the objective
equal to the reference's chi2/dof + penalties to 1e-10."""
import numpy as np
import pytest

import cases
from oracle.bindings import Reference
from shape_b200 import engine as eng

pytestmark = pytest.mark.gpu

FORMS = (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64, eng.FORM_BATCHED_FP32)
T0 = 2458000.0

SHAPE_PENS = [(eng.PEN_NONSMOOTH, 1e3), (eng.PEN_CONCAVITY, 10.0), (eng.PEN_RDEV, 0.5), (eng.PEN_MAXRDEV, 0.2),
              (eng.PEN_VOLUME, 0.01), (eng.PEN_COMDEV, 2.0), (eng.PEN_INERTIADEV_UNI, 1.0),
              (eng.PEN_PA3TILT, 3.0), (eng.PEN_NONPA_UNI, 0.1), (eng.PEN_EULEROFFS, 0.05),
              (eng.PEN_FLATTENING, 0.3), (eng.PEN_VOLUME, -0.01)]
SPIN_PENS = [(eng.PEN_INERTIADEV, 1.0), (eng.PEN_NONPA, 0.1), (eng.PEN_IMPULSE, 0.02)]


def _model():
    """The config-1 ellipsoid with random vertex deviations and unequal
    scale factors: every shape penalty nonzero."""
    m, p, ds = cases.c1()
    mm = m.copy()
    mm.r = np.random.default_rng(77).normal(0.0, 0.03, mm.nv)
    mm.scale = np.array([1.02, 0.97, 1.01])
    return mm, p, ds


def test_penalties_match_reference(cuda_device):
    m, p, ds = _model()
    spin = eng.spin_state(1, T0, (0.3, 0.8, 0.1), (0.0, 0.0, 20.0), impulses=[(T0 + 0.2, (0.0, 0.0, 0.01))],
                          inertia=(1.0, 1.4, 1.35))
    aoff, ooff = np.array([[0.01, -0.02, 0.005]]), np.array([[0.0, 0.0, 0.001]])
    pens = SHAPE_PENS + SPIN_PENS
    e = eng.make_engine(m, p, deldops=[ds])
    k0 = e.kernels_per_eval(eng.FORM_BATCHED_FP64)
    e.set_spin_model(spin, T0 + 0.01 * np.arange(ds.nframes), None, aoff, ooff)
    e.set_penalties(pens)
    assert e.kernels_per_eval(eng.FORM_BATCHED_FP64) == k0 + 2
    rtot, rbase = Reference().session(m, p, deldops=[ds]).penalties(pens, spin, aoff, ooff)
    nz = [i for i, (t, _) in enumerate(pens) if t != eng.PEN_NONPA_UNI]   # 0: I_z is this body's largest
    assert np.all(rbase[nz] > 0.0), rbase
    for form in FORMS:
        s = e.evaluate(form)
        np.testing.assert_allclose(e.penalties(), rbase, rtol=1e-9, atol=1e-14, err_msg=str(form))
        assert abs(s["penalties"] - rtot) <= 1e-9 * rtot, (form, s["penalties"], rtot)
        assert s["posbnd"] == 0 and s["badradar"] == 0
        assert s["objective"] == s["chi2"] / s["dof"] + s["penalties"]
    e.close()


def test_objective_with_penalties_matches_reference(cuda_device):
    m, p, ds = _model()
    ref = Reference().session(m, p, deldops=[ds])
    chi2 = ref.evaluate()
    rtot, _ = ref.penalties(SHAPE_PENS)
    dof = sum(fr.dof for fr in ds.frames)
    want = chi2 / dof + rtot
    e = eng.make_engine(m, p, deldops=[ds])
    e.set_penalties(SHAPE_PENS)
    for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
        s = e.evaluate(form)
        assert abs(s["objective"] - want) <= 1e-10 * want, (form, s["objective"], want)
    e.set_penalties([])
    s = e.evaluate(eng.FORM_BATCHED_FP64)
    assert s["penalties"] == 0.0 and abs(s["objective"] - chi2 / dof) <= 1e-10 * chi2 / dof
    e.close()


def test_penalty_errors(cuda_device):
    m, p, ds = _model()
    e = eng.make_engine(m, p, deldops=[ds])
    with pytest.raises(eng.EngineError):
        e.set_penalties([(22, 1.0)])                   # maxellipdev: not supported
    e.set_penalties([(eng.PEN_NONPA, 1.0)])            # needs the spin model
    with pytest.raises(eng.EngineError):
        e.evaluate(eng.FORM_BATCHED_FP64)
    e.set_penalties([(eng.PEN_VOLUME, 1.0)])
    s = e.evaluate(eng.FORM_BATCHED_FP64)              # the engine is still usable
    assert s["penalties"] > 0.0
    e.close()


def test_penalties_two_components(cuda_device):
    """A model of two VERTEX components, the second mostly inside the
    first: check_surface's active flags equal the reference's realize_mod
    (vertices, and facets by their centroids), and every shape penalty,
    which leaves inactive facets, edges and vertices out, matches the
    reference's penalties() in every form."""
    from shape_b200 import synth
    m = synth.two_component_model()
    m.r = np.random.default_rng(78).normal(0.0, 0.02, m.nv)
    p = synth.eval_params()
    ds = synth.config1_frames(2, None, p)
    ref = Reference().session(m, p, deldops=[ds])
    rtot, rbase = ref.penalties(SHAPE_PENS)
    rv, rf = ref.active()
    assert 0 < rv.sum() < m.nv and 0 < rf.sum() < m.nf, (rv.sum(), rf.sum())
    e = eng.make_engine(m, p, deldops=[ds])
    k0 = e.kernels_per_eval(eng.FORM_BATCHED_FP64)
    e.set_penalties(SHAPE_PENS)
    assert e.kernels_per_eval(eng.FORM_BATCHED_FP64) == k0 + 3
    for form in FORMS:
        s = e.evaluate(form)
        gv, gf = e.active()
        assert np.array_equal(gv, rv) and np.array_equal(gf, rf), form
        np.testing.assert_allclose(e.penalties(), rbase, rtol=1e-9, atol=1e-14, err_msg=str(form))
        assert abs(s["penalties"] - rtot) <= 1e-9 * rtot, (form, s["penalties"], rtot)
    # a trial that moves the second component: the flags follow it
    e.set_scale(3, 1.2)
    R = Reference()
    ref2 = R.session(m, p, deldops=[ds])
    R.lib.ref_set_scale(ref2.h, 3, 1.2)
    rtot2, rbase2 = ref2.penalties(SHAPE_PENS)
    rv2, rf2 = ref2.active()
    s = e.evaluate(eng.FORM_BATCHED_FP64)
    gv, gf = e.active()
    assert np.array_equal(gv, rv2) and np.array_equal(gf, rf2)
    np.testing.assert_allclose(e.penalties(), rbase2, rtol=1e-9, atol=1e-14)
    e.close()
