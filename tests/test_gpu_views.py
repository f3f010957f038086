"""View updates between evaluations (shape_engine_set_frame_view and
shape_engine_set_point_view), as spin, pole and delay-correction trials make
them: after new views, every form gives what the oracle gives on datasets
carrying those views, at the parity tests' bars (FP64 forms: facet, z and
cos(e) maps bit-exact, chi-square to 1e-10; FP32 form: chi-square to 1e-6),
through graphs captured before the change; setting the old views back
restores the first results."""
import copy

import numpy as np
import pytest

import cases
import golden_cases as gc
from shape_b200 import ctypes_defs as cd
from shape_b200 import engine as eng
from test_gpu_parity import CHI2_RTOL, FP32_CHI2_RTOL, _frame_checks

pytestmark = pytest.mark.gpu

FORMS = (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64, eng.FORM_BATCHED_FP32)


def _rz(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])


def _rx(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]])


def _m(v):
    return np.array(v[:], dtype=np.float64).reshape(3, 3)


def _new_view(fr, k):
    """A spin-phase step, a pole tilt and a faster spin for frame k."""
    ae = _rz(0.15 + 0.05 * k) @ _m(fr.ae) @ _rx(0.08)
    spin = 1.08 * (_rx(0.08).T @ np.array(fr.spin[:]))
    return ae, spin


def test_frame_views_deldop(cuda_device):
    m, p, ds = cases.c2(12)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    base = {f: e.evaluate(f)["chi2"] for f in FORMS}      # tuned, graphs captured
    ds2 = copy.copy(ds)
    ds2.frames = []
    for k, fr in enumerate(ds.frames):
        g = cd.DeldopFrame.from_buffer_copy(fr)
        ae, spin = _new_view(fr, k)
        cd.fill9(g.ae, ae)
        for j in range(3):
            g.spin[j] = spin[j]
        g.deloff, g.dopoff = fr.deloff + 0.37, fr.dopoff - 0.21
        ds2.frames.append(g)
        e.set_frame_view(k, ae, _m(fr.oe), spin, g.deloff, g.dopoff)
    o = cases.orc().eval_deldop(m, ds2, p, keep_pos=True)
    chi2_o = sum(r["chi2"] for r in o["results"])
    for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
        s = e.evaluate(form)
        _frame_checks(e, o, ds2)
        assert abs(s["chi2"] - chi2_o) <= CHI2_RTOL * chi2_o, (form, s["chi2"], chi2_o)
    s = e.evaluate(eng.FORM_BATCHED_FP32)
    assert abs(s["chi2"] - chi2_o) <= FP32_CHI2_RTOL * chi2_o, (s["chi2"], chi2_o)
    for k, fr in enumerate(ds.frames):
        e.set_frame_view(k, _m(fr.ae), _m(fr.oe), fr.spin[:], fr.deloff, fr.dopoff)
    for form in FORMS:       # FP32: the scatter's float atomics may add in another order
        c = e.evaluate(form)["chi2"]
        bar = FP32_CHI2_RTOL if form == eng.FORM_BATCHED_FP32 else CHI2_RTOL
        assert abs(c - base[form]) <= bar * base[form], (form, c, base[form])
    with pytest.raises(eng.EngineError):
        e.set_frame_view(ds.nframes, np.eye(3), np.eye(3), np.zeros(3))
    e.close()


def test_frame_views_doppler(cuda_device):
    model_fn, ds_fn, p = gc.DOPPLER_CASES["dop_nsinc2"]      # nsinc2 = 2: footprint increments
    m = model_fn()
    ds = ds_fn(lambda d, q: cases.orc().eval_doppler(m, d, q)["fits"], p)
    e = eng.make_engine(m, p, dopplers=[ds])
    e.keep_pos(True)
    for f in FORMS:
        e.evaluate(f)
    ds2 = copy.copy(ds)
    ds2.frames = []
    for k, fr in enumerate(ds.frames):
        g = cd.DopplerFrame.from_buffer_copy(fr)
        ae, spin = _new_view(fr, k)
        cd.fill9(g.ae, ae)
        for j in range(3):
            g.spin[j] = spin[j]
        g.dopoff = fr.dopoff + 0.43
        ds2.frames.append(g)
        e.set_frame_view(k, ae, _m(fr.oe), spin, 5.0, g.dopoff)     # deloff: ignored for spectra
    o = cases.orc().eval_doppler(m, ds2, p, keep_pos=True)
    chi2_o = sum(r["chi2"] for r in o["results"])
    for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
        s = e.evaluate(form)
        res = e.results()
        for f in range(len(ds2.frames)):
            assert np.array_equal(e.pos(f)["f"], o["pos"][f]["f"]), (form, f)
            assert list(res[f]["idoplim"]) == list(o["results"][f]["idoplim"]), (form, f)
            assert abs(res[f]["chi2"] - o["results"][f]["chi2"]) <= CHI2_RTOL * abs(o["results"][f]["chi2"])
        assert abs(s["chi2"] - chi2_o) <= CHI2_RTOL * chi2_o
    s = e.evaluate(eng.FORM_BATCHED_FP32)
    assert abs(s["chi2"] - chi2_o) <= FP32_CHI2_RTOL * chi2_o
    e.close()


def test_point_views_lightcurve(cuda_device):
    m, p, sets = cases.c3(12, 2)
    e = eng.make_engine(m, p, lghtcrvs=sets)
    e.keep_pos(True)
    for f in FORMS:
        e.evaluate(f)
    sets2, pt = [], 0
    for ds in sets:
        d2 = copy.copy(ds)
        d2.points = []
        for i, q in enumerate(ds.points):
            g = cd.LghtcrvPoint.from_buffer_copy(q)
            ae = _rz(0.2 + 0.03 * i) @ _m(q.ae)
            cd.fill9(g.ae, ae)
            d2.points.append(g)
            e.set_point_view(pt, ae, _m(q.oe), _m(q.se))
            pt += 1
        sets2.append(d2)
    o = cases.orc()
    outs = [o.eval_lghtcrv(m, d, p, keep_pos=True) for d in sets2]
    tot = sum(oo["chi2"] for oo in outs)
    for form in FORMS:
        s = e.evaluate(form)
        for k, d in enumerate(sets2):
            for i, q in enumerate(d.points):
                pg, po = e.lghtcrv_pos(k, i, q), outs[k]["pos"][i]
                assert np.array_equal(pg["f"], po["f"]), (form, k, i)
                assert np.array_equal(pg["fill"], po["fill"]), (form, k, i)
            if form != eng.FORM_BATCHED_FP32:
                g = e.lghtcrv(k, d)
                np.testing.assert_allclose(g["y"], outs[k]["y"], rtol=1e-12)
        bar = FP32_CHI2_RTOL if form == eng.FORM_BATCHED_FP32 else CHI2_RTOL
        assert abs(s["chi2"] - tot) <= bar * tot, (form, s["chi2"], tot)
    e.close()


def _spin_views(ds, spin, t, angleoff=(0.0, 0.0, 0.0)):
    """ds with every frame's ae and spin vector realized from `spin` at the
    view epochs t (shape_realize_spin, checked against the reference's
    realize_spin on the CPU)."""
    ae, sp = eng.realize_spin(spin, t, None, angleoff)
    d2 = copy.copy(ds)
    d2.frames = []
    for k, fr in enumerate(ds.frames):
        g = cd.DeldopFrame.from_buffer_copy(fr)
        cd.fill9(g.ae, ae[k])
        for j in range(3):
            g.spin[j] = sp[k][j]
        d2.frames.append(g)
    return d2


T0 = 2458000.0


def _pa_spin(psi0):
    return eng.spin_state(1, T0, (0.5, 0.9, psi0), (0.0, 0.0, 2 * np.pi / 0.25))


def test_spin_model_deldop(cuda_device):
    """set_spin_model realizes the views of an engine whose graphs were
    captured on the dataset's own views; a spin-parameter trial re-realizes
    them. Both against the oracle on the realized views."""
    m, p, ds = cases.c2(12)
    t = T0 + 0.04 * np.arange(ds.nframes)
    e = eng.make_engine(m, p, deldops=[ds])
    e.keep_pos(True)
    for f in FORMS:
        e.evaluate(f)
    e.set_spin_model(_pa_spin(0.3), t)
    for psi0 in (0.3, 0.35):
        if psi0 != 0.3:
            e.set_spin_param(eng.PAR_SPIN_ANGLE, 2, psi0)
        assert e.get_spin_param(eng.PAR_SPIN_ANGLE, 2) == psi0
        ds2 = _spin_views(ds, _pa_spin(psi0), t)
        o = cases.orc().eval_deldop(m, ds2, p, keep_pos=True)
        chi2_o = sum(r["chi2"] for r in o["results"])
        for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
            s = e.evaluate(form)
            _frame_checks(e, o, ds2)
            assert abs(s["chi2"] - chi2_o) <= CHI2_RTOL * chi2_o, (psi0, form, s["chi2"], chi2_o)
        s = e.evaluate(eng.FORM_BATCHED_FP32)
        assert abs(s["chi2"] - chi2_o) <= FP32_CHI2_RTOL * chi2_o, (psi0, s["chi2"], chi2_o)
    for kind, index in ((eng.PAR_SPIN_ANGLE, 3), (eng.PAR_ANGLEOFF, 3), (eng.PAR_SPIN_IMPULSE, 0), (99, 0)):
        with pytest.raises(eng.EngineError):
            e.set_spin_param(kind, index, 0.0)
    e.close()


def test_spin_model_lightcurve_offsets(cuda_device):
    """Lightcurve points realized at their sets' calculated epochs, with a
    per-dataset angle offset on the second set."""
    m, p, sets = cases.c3(12, 2)
    e = eng.make_engine(m, p, lghtcrvs=sets)
    e.keep_pos(True)
    e.evaluate(eng.FORM_BATCHED_FP64)
    spin = eng.spin_state(1, float(sets[0].x[0]), (0.2, 1.1, 0.4), (0.0, 0.0, 2 * np.pi / 0.3))
    aoff = np.array([[0.0, 0.0, 0.0], [0.01, -0.02, 0.03]])
    e.set_spin_model(spin, None, None, aoff)
    o = cases.orc()
    tot = 0.0
    outs, sets2 = [], []
    for k, ds in enumerate(sets):
        ae, _ = eng.realize_spin(spin, ds.x, None, tuple(aoff[k]))
        d2 = copy.copy(ds)
        d2.points = []
        for i, q in enumerate(ds.points):
            g = cd.LghtcrvPoint.from_buffer_copy(q)
            cd.fill9(g.ae, ae[i])
            d2.points.append(g)
        sets2.append(d2)
        outs.append(o.eval_lghtcrv(m, d2, p, keep_pos=True))
        tot += outs[-1]["chi2"]
    for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
        s = e.evaluate(form)
        for k, d in enumerate(sets2):
            np.testing.assert_allclose(e.lghtcrv(k, d)["y"], outs[k]["y"], rtol=1e-12)
            for i, q in enumerate(d.points):
                assert np.array_equal(e.lghtcrv_pos(k, i, q)["f"], outs[k]["pos"][i]["f"]), (form, k, i)
        assert abs(s["chi2"] - tot) <= CHI2_RTOL * tot, (form, s["chi2"], tot)
    e.close()


def test_spin_fit_recovers_rotation_phase(cuda_device):
    """bestfit over spin.angle[2] (SHAPE_PAR_SPIN_ANGLE) on noise-free data
    made from a known spin state: every trial is a spin realization of all
    views plus a graph replay; the fit returns to the true phase."""
    m, p, ds = cases.c2(12)
    t = T0 + 0.04 * np.arange(ds.nframes)
    truth = _spin_views(ds, _pa_spin(0.3), t)
    fits = cases.orc().eval_deldop(m, truth, p)["fits"]
    obs = np.concatenate([np.asarray(f, dtype=np.float64).ravel() for f in fits])
    data = copy.copy(truth)
    data.obs = obs
    e = eng.make_engine(m, p, deldops=[data])
    e.set_spin_model(_pa_spin(0.3), t)
    at_truth = e.evaluate(eng.FORM_BATCHED_FP64)["chi2"]
    e.set_spin_param(eng.PAR_SPIN_ANGLE, 2, 0.32)
    at_start = e.evaluate(eng.FORM_BATCHED_FP64)["chi2"]
    assert at_truth <= 1e-6 * at_start, (at_truth, at_start)
    res, trace = e.bestfit([(eng.PAR_SPIN_ANGLE, 2, 0.005, 1e-7, 1e-7)], term_prec=1e-9, term_maxiter=4,
                           trace_max=400)
    psi = e.get_spin_param(eng.PAR_SPIN_ANGLE, 2)
    assert abs(psi - 0.3) < 1e-4, psi
    assert res["final_objective"] < 1e-3 * res["initial_objective"], res
    assert len(trace) == res["trace_len"] > 5
    e.close()


def test_device_spin_matches_host_realization(cuda_device):
    """shape_engine_set_spin_device: views realized inside the evaluation
    graph from the spin state. Against host realization (shape_realize_spin,
    bit-exact with the reference) of the same trials: ae and spin vectors to
    a few units in the last place (CUDA's sin / cos against the C
    library's), chi-square to 1e-10 in the FP64 forms and 1e-6 in FP32, and
    a spin trial costs no host realization (set_spin_param only records the
    value)."""
    m, p, ds = cases.c2(12)
    t = T0 + 0.04 * np.arange(ds.nframes)
    host = eng.make_engine(m, p, deldops=[ds])
    dev = eng.make_engine(m, p, deldops=[ds])
    for e in (host, dev):
        e.set_spin_model(_pa_spin(0.3), t, None, None)
    dev.set_spin_device(True)
    n0 = host.kernels_per_eval(eng.FORM_BATCHED_FP64)
    assert dev.kernels_per_eval(eng.FORM_BATCHED_FP64) == n0 + 1
    trials = [(eng.PAR_SPIN_ANGLE, 2, 0.37), (eng.PAR_SPIN_OMEGA, 2, 2 * np.pi / 0.26),
              (eng.PAR_SPIN_ANGLE, 0, 0.55), (eng.PAR_ANGLEOFF, 1, 0.01), (eng.PAR_OMEGAOFF, 2, 0.2)]
    for kind, index, value in [(None, None, None)] + trials:
        if kind is not None:
            host.set_spin_param(kind, index, value)
            dev.set_spin_param(kind, index, value)
        for form in FORMS:
            sh, sd = host.evaluate(form), dev.evaluate(form)
            tol = FP32_CHI2_RTOL if form == eng.FORM_BATCHED_FP32 else CHI2_RTOL
            assert abs(sd["chi2"] - sh["chi2"]) <= tol * abs(sh["chi2"]), (kind, index, form)
        for f in range(ds.nframes):
            ah, wh = host.frame_view(f)
            ad, wd = dev.frame_view(f)
            assert np.max(np.abs(ad - ah)) <= 4e-16, (kind, f)
            assert np.max(np.abs(wd - wh)) <= 4e-15 * np.max(np.abs(wh)), (kind, f)
    with pytest.raises(eng.EngineError, match="realized on the device"):
        dev.set_frame_view(0, np.eye(3), np.eye(3), np.zeros(3))
    # back to host realization: the host views catch up with the trials
    dev.set_spin_device(False)
    a, b = dev.evaluate(eng.FORM_BATCHED_FP64)["chi2"], host.evaluate(eng.FORM_BATCHED_FP64)["chi2"]
    assert abs(a - b) <= 1e-12 * abs(b)
    for f in range(ds.nframes):
        assert np.array_equal(dev.frame_view(f)[0], host.frame_view(f)[0])
    host.close()
    dev.close()


def test_device_spin_lightcurves(cuda_device):
    """Device spin realization of lightcurve points (observer and sun views)
    against host realization, with dataset angle offsets."""
    m, p, sets = cases.c3(12, 2)
    spin = eng.spin_state(1, float(sets[0].x[0]), (0.2, 1.1, 0.4), (0.0, 0.0, 2 * np.pi / 0.3))
    aoff = np.array([[0.0, 0.0, 0.0], [0.01, -0.02, 0.03]])
    host = eng.make_engine(m, p, lghtcrvs=sets)
    dev = eng.make_engine(m, p, lghtcrvs=sets)
    for e in (host, dev):
        e.set_spin_model(spin, None, None, aoff)
    dev.set_spin_device(True)
    for kind, index, value in [(None, None, None), (eng.PAR_SPIN_ANGLE, 2, 0.45), (eng.PAR_ANGLEOFF, 4, -0.01)]:
        if kind is not None:
            host.set_spin_param(kind, index, value)
            dev.set_spin_param(kind, index, value)
        for form in FORMS:
            sh, sd = host.evaluate(form), dev.evaluate(form)
            tol = FP32_CHI2_RTOL if form == eng.FORM_BATCHED_FP32 else CHI2_RTOL
            assert abs(sd["chi2"] - sh["chi2"]) <= tol * abs(sh["chi2"]), (kind, form)
            for k, d in enumerate(sets):
                np.testing.assert_allclose(dev.lghtcrv(k, d)["y"], host.lghtcrv(k, d)["y"], rtol=1e-12)
    host.close()
    dev.close()


def test_device_spin_refusals(cuda_device):
    m, p, ds = cases.c2(4)
    e = eng.make_engine(m, p, deldops=[ds])
    with pytest.raises(eng.EngineError, match="no spin model"):
        e.set_spin_device(True)
    t = T0 + 0.04 * np.arange(ds.nframes)
    npa = eng.spin_state(0, T0, (0.5, 0.9, 0.3), (0.1, 0.2, 2 * np.pi / 0.25), inertia=(1.0, 1.1, 1.2))
    e.set_spin_model(npa, t)
    with pytest.raises(eng.EngineError, match="principal-axis"):
        e.set_spin_device(True)
    e.close()
