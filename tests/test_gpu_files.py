"""Model and fit files with the engine: a model read from a .mod file
evaluates exactly like the same model given directly; after parameter
changes, shape_mod_take_engine carries the engine's values into the file
written next; shape_engine_write_fitdat writes the frame's listfit file
(cal * fit / sdev, "%13.6e" per line) from the last evaluation."""
import numpy as np
import pytest

import cases
from shape_b200 import engine as eng
from test_modfile import write_mod

pytestmark = pytest.mark.gpu


def test_mod_file_engine_round_trip(cuda_device, tmp_path):
    m, p, ds = cases.c1()
    path = tmp_path / "c1.mod"
    write_mod(path, m, seed=2)
    mf = eng.ModFile(path)
    e1 = eng.make_engine(mf.model(), p, deldops=[ds])
    e2 = eng.make_engine(m, p, deldops=[ds])
    for form in (eng.FORM_PLAIN_FP64, eng.FORM_BATCHED_FP64):
        assert e1.evaluate(form)["chi2"] == e2.evaluate(form)["chi2"]
    e1.set_scale(1, 1.07)
    e1.set_vertex_r(5, 0.0123)
    mf.take_engine(e1)
    out = tmp_path / "fitted.mod"
    mf.write(out)
    back = eng.ModFile(out).model()
    assert back.scale[1] == 1.07 and back.r[5] == 0.0123 and np.array_equal(back.fv, m.fv)
    s = e1.evaluate(eng.FORM_BATCHED_FP64)
    sdev = 0.8
    e1.write_fitdat(0, sdev, tmp_path / "f0.fitdat")
    cal = e1.results()[0]["cal"]
    want = ["%13.6e" % (cal * x / sdev) for x in np.asarray(e1.fit(0)).ravel()]
    assert (tmp_path / "f0.fitdat").read_text().splitlines() == want
    assert s["chi2"] > 0.0
    e1.close()
    e2.close()


def test_two_component_mod_file(cuda_device, tmp_path):
    """A two-component model read from a .mod file evaluates like the same
    components given directly; a second-component scale change carries into
    the written file."""
    from shape_b200 import synth
    m = synth.two_component_model(rot=(0.3, 0.5, -0.2))
    nv1, nf1 = int(m.comp_nv[0]), int(m.comp_nf[0])

    def part(c):
        v0, v1 = (0, nv1) if c == 0 else (nv1, m.nv)
        f0, f1 = (0, nf1) if c == 0 else (nf1, m.nf)
        sub = synth.Model(m.a[v0:v1], m.u[v0:v1], m.r[v0:v1], m.fv[f0:f1] - v0,
                          m.af_ptr[v0:v1 + 1] - m.af_ptr[v0], m.af_idx[m.af_ptr[v0]:m.af_ptr[v1]] - f0,
                          m.comp_scale[c].copy())
        return sub

    comps = [(part(0), m.comp_off[0], np.degrees(m.comp_rot[0]), "fff"),
             (part(1), m.comp_off[1], np.degrees(m.comp_rot[1]), "fff")]
    path = tmp_path / "two.mod"
    write_mod(path, None, seed=3, comps=comps)
    mf = eng.ModFile(path)
    got = mf.model()
    _, p, ds = cases.c1()
    e1 = eng.make_engine(got, p, deldops=[ds])
    e2 = eng.make_engine(m, p, deldops=[ds])
    c1, c2 = e1.evaluate(eng.FORM_PLAIN_FP64)["chi2"], e2.evaluate(eng.FORM_PLAIN_FP64)["chi2"]
    # the file carries the angles in degrees: the radians read back can
    # differ from the direct ones in the last bit
    assert abs(c1 - c2) <= 1e-9 * c2
    e1.set_scale(4, 1.11)
    mf.take_engine(e1)
    out = tmp_path / "back.mod"
    mf.write(out)
    back = eng.ModFile(out).model()
    assert back.comp_scale[1][1] == 1.11 and back.comp_scale[0][1] == 1.0
    e1.close()
    e2.close()
    mf.close()
