"""Model files (.mod): shape_mod_read against the reference's own read_mod
(oracle/_ref/libshape_ref.so via ref_mod_read), on the CPU. Files are
written here from seeded models, with comments in curly braces between
tokens; the shape arrays, the attached-facet lists, the scattering laws and
the spin state (epochs, angles folded over the pole, rad and rad/day
conversions, impulses, the principal-axis flag) must equal the
reference's to the last bit. Unsupported content and syntax errors are
refused with their line."""
import numpy as np
import pytest

import cases
from oracle.bindings import Reference
from shape_b200 import engine as eng


@pytest.fixture(scope="module")
def ref():
    return Reference()


class Writer:
    """Tokens with a comment after some of them (seeded)."""

    def __init__(self, seed):
        self.rng = np.random.default_rng(seed)
        self.out = []

    def tok(self, *items):
        for t in items:
            self.out.append(t if isinstance(t, str) else repr(t))
            r = self.rng.random()
            if r < 0.05:
                self.out.append("{ a comment\nover two lines }")
            elif r < 0.1:
                self.out.append("\n")

    def par(self, state, value):
        self.tok(state, float(value))

    def text(self):
        return " ".join(self.out) + "\n"


def write_mod(path, m, seed=0, states=None, radar=("cosine", 0.1, 1.0), optical=("kaasalainen",),
              spin=None, ctype="vertex", rstate="f", comps=None):
    """comps: several components, (model, offset km, rotation deg, scale
    states) each, in place of m."""
    w = Writer(seed)
    st = states or {}
    comps = comps or [(m, (0.0,) * 3, (0.0,) * 3, st.get("scale", "fcf"))]
    w.tok(len(comps))
    for cm, off, rot, sst in comps:
        for x in tuple(off) + tuple(rot):
            w.par("c", x)
        w.tok(ctype, cm.nv)
        for j in range(3):
            w.par(sst[j], cm.scale[j])
        for v in range(cm.nv):
            w.par(rstate if v % 7 else "c", cm.r[v])
            w.tok(*[float(x) for x in cm.u[v]], *[float(x) for x in cm.a[v]])
        w.tok(cm.nf)
        for f in range(cm.nf):
            w.tok(*[int(x) for x in cm.fv[f]])
    w.tok(1, radar[0])
    if radar[0] == "cosine":
        w.par("f", radar[1]); w.par("c", radar[2])
    elif radar[0] in ("gaussian", "hagfors", "cosine_qs"):
        w.par("f", 0.2); w.par("c", 3.0); w.tok(55.0)
    else:
        w.par("f", 0.2); w.par("c", 3.0); w.tok(40.0); w.par("f", 0.05); w.par("c", 1.5)
    w.tok(2, optical[0])
    if optical[0] == "kaasalainen":
        w.par("f", 0.45); w.par("c", 0.3); w.par("c", 0.5); w.par("c", 7.0); w.par("c", -0.004)
    else:
        w.par("f", 0.2)
    w.tok("lommel")
    w.par("c", 0.1)
    sp = spin or {}
    w.tok(*sp.get("t0", (2018, 3, 14, 5, 6, 7)))
    for a in sp.get("angle", (30.0, 250.0, -10.0)):
        w.par("f", a)
    for i, o in enumerate(sp.get("omega", (0.0, 0.0, 1440.0))):
        w.par(sp.get("omega_state", "ccf")[i], o)
    for x in sp.get("inertia", (1.0, 1.1, 1.2)):
        w.par("c", x)
    for x in sp.get("omegadot", (0.0, 0.0, 1e-6)):
        w.par("c", x)
    for x in sp.get("lib", (0.0, 0.0, 0.0)):
        w.par("c", x)
    imps = sp.get("impulses", [((2018, 3, 15, 0, 0, 0), (0.0, 0.0, 2.0))])
    w.tok(len(imps))
    for date, vec in imps:
        w.tok(*date)
        for x in vec:
            w.par("f" if x else "c", x)
    path.write_text(w.text())


def _compare(path, ref):
    mf = eng.ModFile(path)
    m = mf.model()
    arrays, radar, optical, spin = ref.read_mod(str(path))
    for k in ("a", "u", "r", "scale"):
        assert np.array_equal(np.asarray(getattr(m, k)), arrays[k]), k
    for k in ("fv", "af_ptr", "af_idx"):
        assert np.array_equal(np.asarray(getattr(m, k)), arrays[k]), k
    for mine, theirs in zip(mf.radar_laws(), radar):
        assert bytes(mine) == bytes(theirs)
    for mine, theirs in zip(mf.optical_laws(), optical):
        assert bytes(mine) == bytes(theirs)
    assert len(mf.radar_laws()) == len(radar) and len(mf.optical_laws()) == len(optical)
    s = mf.spin()
    for k in ("pa", "t0", "n_impulse", "lib_amp", "lib_freq", "lib_phase"):
        assert getattr(s, k) == getattr(spin, k), k
    for k in ("angle", "omega", "omegadot", "inertia"):
        assert list(getattr(s, k)) == list(getattr(spin, k)), k
    for n in range(s.n_impulse):
        assert s.t_impulse[n] == spin.t_impulse[n]
        assert list(s.impulse[n]) == list(spin.impulse[n])
    return mf, m


@pytest.mark.parametrize("seed", range(3))
def test_mod_matches_reference_read_mod(tmp_path, ref, seed):
    base = cases.c1()[0]
    m = base.copy()
    rng = np.random.default_rng(seed)
    m.r = rng.normal(0, 0.02, m.nv)
    m.scale = np.array([1.0, 1.05, 0.95]) + rng.normal(0, 1e-3, 3)
    radar = [("cosine", 0.1, 1.0), ("hagfors",), ("cosine+cosine",)][seed]
    spin = {"angle": [(30.0, 250.0, -10.0), (-400.0, 95.0, 720.5), (10.0, 181.0, 3.0)][seed]}
    path = tmp_path / ("m%d.mod" % seed)
    write_mod(path, m, seed=seed, radar=radar, optical=[("kaasalainen",), ("lambertian",), ("lommel",)][seed],
              spin=spin)
    mf, got = _compare(path, ref)
    assert np.array_equal(got.a, m.a) and np.array_equal(got.r, m.r) and np.array_equal(got.fv, m.fv)
    assert mf.spin().pa == 1
    assert mf.spin().angle[1] <= np.pi
    # free parameters in the reference's order: scale 0 and 2, the floating
    # vertex deviations, the three angles, omega z, the z impulse
    fp = mf.free_params()
    nr = sum(1 for v in range(m.nv) if v % 7)
    assert fp[:2] == [(eng.PAR_SCALE, 0), (eng.PAR_SCALE, 2)]
    assert all(k == eng.PAR_VERTEX_R for k, _ in fp[2:2 + nr]) and len(fp) == 2 + nr + 5
    assert fp[2 + nr:] == [(eng.PAR_SPIN_ANGLE, 0), (eng.PAR_SPIN_ANGLE, 1), (eng.PAR_SPIN_ANGLE, 2),
                           (eng.PAR_SPIN_OMEGA, 2), (eng.PAR_SPIN_IMPULSE, 2)]
    mf.close()


def test_mod_two_components(tmp_path, ref):
    """Two vertex components: vertices, facets and attached-facet lists
    concatenated with model-wide indices, each component's scale factors,
    offsets and rotations (degrees wrapped into (-180, 180], then radians)
    equal to the reference's; free parameters per component (its scale
    factors, then its vertex deviations); the file written back reads the
    same."""
    from shape_b200 import synth
    m1 = cases.c1()[0].copy()
    m1.r = np.random.default_rng(1).normal(0, 0.02, m1.nv)
    dirs, fv2 = synth.ring_sphere(6, 10)
    m2 = synth.make_model(dirs, fv2, None, base=0.3 * dirs, name="small")
    m2.scale = np.array([1.05, 0.97, 1.0])
    comps = [(m1, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), "fcc"),
             (m2, (0.6, -0.1, 0.05), (200.0, -190.0, 30.5), "cff")]
    path = tmp_path / "two.mod"
    write_mod(path, None, seed=11, comps=comps)
    mf, got = _compare(path, ref)
    arrays = ref.read_mod(str(path))[0]
    assert got.ncomp == 2 and len(arrays["comps"]) == 2
    for c, rc in enumerate(arrays["comps"]):
        assert got.comp_nv[c] == rc["nv"] and got.comp_nf[c] == rc["nf"]
        assert np.array_equal(got.comp_scale[c], rc["scale"])
        assert np.array_equal(got.comp_off[c], rc["off"])
        assert np.array_equal(got.comp_rot[c], rc["rot"])
    assert got.comp_rot[1][0] < 0 and got.comp_rot[1][1] > 0
    assert np.array_equal(got.fv[m1.nf:], m2.fv + m1.nv)
    fp = mf.free_params()
    n1 = sum(1 for v in range(m1.nv) if v % 7)
    n2 = sum(1 for v in range(m2.nv) if v % 7)
    assert fp[0] == (eng.PAR_SCALE, 0)
    assert fp[1 + n1:3 + n1] == [(eng.PAR_SCALE, 4), (eng.PAR_SCALE, 5)]
    assert fp[3 + n1][1] == m1.nv + 1 and len(fp) == 3 + n1 + n2 + 5
    out = tmp_path / "two_back.mod"
    mf.write(out)
    mb, back = _compare(out, ref)
    for k in ("a", "u", "r", "fv", "af_ptr", "af_idx", "comp_nv", "comp_nf", "comp_scale", "comp_off", "comp_rot"):
        assert np.array_equal(np.asarray(getattr(back, k)), np.asarray(getattr(got, k))), k
    assert mb.free_params() == fp
    mf.close()
    mb.close()


def test_mod_non_principal_axis(tmp_path, ref):
    m = cases.c1()[0]
    path = tmp_path / "npa.mod"
    write_mod(path, m, seed=5, spin={"omega": (12.0, -30.0, 900.0), "omega_state": "fff",
                                     "omegadot": (0.0, 0.0, 0.0), "t0": (1999, 12, 31, 23, 59, 59),
                                     "impulses": [((2000, 1, 2, 0, 0, 0), (1.0, 0.0, -2.0)),
                                                  ((2000, 1, 5, 12, 0, 0), (0.0, 0.5, 0.0))]})
    mf, _ = _compare(path, ref)
    assert mf.spin().pa == 0 and mf.spin().n_impulse == 2


def _err(path):
    with pytest.raises(eng.EngineError) as ei:
        eng.ModFile(path)
    return str(ei.value)


def test_mod_refusals(tmp_path):
    m = cases.c1()[0]
    p = tmp_path / "e.mod"
    write_mod(p, m, ctype="ellipse")
    assert "error -4" in _err(p) and "vertex" in _err(p)
    write_mod(p, m, rstate="=")
    assert "error -4" in _err(p)
    write_mod(p, m, radar=("tabular",))
    assert "error -4" in _err(p)
    write_mod(p, m)
    text = p.read_text()
    p.write_text(text.replace("vertex", "vertex x", 1))
    msg = _err(p)
    assert "error -1" in msg and "line" in msg
    p.write_text(text + " { unclosed")
    # the spin section ends before the comment; the reader stops there
    eng.ModFile(p).close()
    p.write_text(text.rsplit(" ", 8)[0])
    assert "end of file" in _err(p)
    p.write_text("1 c 0 c 0 c 0 c 0 c 0 c 0 vertex 4 { unclosed")
    assert "unclosed comment" in _err(p)


def test_mod_write_round_trip(tmp_path, ref):
    """shape_mod_write: the written file reads back (with this reader and
    with the reference's read_mod, identically) to the same shape, states,
    epochs and impulses; angles, rates and law constants written in degrees
    return to within a few ulps."""
    m = cases.c1()[0].copy()
    m.r = np.random.default_rng(9).normal(0, 0.02, m.nv)
    a, b = tmp_path / "a.mod", tmp_path / "b.mod"
    write_mod(a, m, seed=4, radar=("gauss+cosine",),
              spin={"angle": (33.3, 120.7, 359.9), "lib": (0.5, 20.0, 45.0),
                    "impulses": [((2019, 5, 6, 7, 8, 9), (0.0, 0.0, 1.25)),
                                 ((2019, 6, 1, 23, 59, 59), (0.0, 0.0, -0.5))]})
    ma = eng.ModFile(a)
    ma.write(b)
    mb, gb = _compare(b, ref)
    ga = ma.model()
    for k in ("a", "u", "r", "scale", "fv", "af_ptr", "af_idx"):
        assert np.array_equal(np.asarray(getattr(ga, k)), np.asarray(getattr(gb, k))), k
    assert mb.free_params() == ma.free_params()
    sa, sb = ma.spin(), mb.spin()
    assert sa.t0 == sb.t0 and sa.n_impulse == sb.n_impulse and sa.pa == sb.pa
    assert [sa.t_impulse[n] for n in range(2)] == [sb.t_impulse[n] for n in range(2)]
    for k in ("angle", "omega", "omegadot", "inertia"):
        np.testing.assert_allclose(list(getattr(sb, k)), list(getattr(sa, k)), rtol=4e-16, atol=1e-300)
    np.testing.assert_allclose([sb.impulse[n][2] for n in range(2)], [sa.impulse[n][2] for n in range(2)],
                               rtol=4e-16)
    for x, y in zip(ma.radar_laws() + ma.optical_laws(), mb.radar_laws() + mb.optical_laws()):
        assert x.type == y.type
        for f, _ in type(x)._fields_[1:]:
            assert abs(getattr(x, f) - getattr(y, f)) <= 4e-16 * abs(getattr(x, f)) + 1e-300, f


def test_fitdat_format(tmp_path):
    rng = np.random.default_rng(3)
    fit = rng.normal(0, 1, (7, 11)) * 10.0 ** rng.integers(-8, 8, (7, 11))
    cal, sdev = 1.7342, 0.913
    p = tmp_path / "f.fitdat"
    eng.write_fitdat(p, fit, cal, sdev)
    lines = p.read_text().splitlines()
    assert lines == ["%13.6e" % (cal * x / sdev) for x in fit.ravel()]
