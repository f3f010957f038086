"""Observation files (.obs): shape_obs_read + shape_obs_frames against the
reference's own read_dat, realize_delcor and realize_spin (via
ref_obs_read) on the CPU, for a delay-Doppler set with an ephemeris, a
delay-correction polynomial, dataset angle and spin offsets and ASCII and
big-endian binary data files: every frame's observer and body matrices,
spin vector, delay and Doppler offsets, COM bins, weight, dof,
calibration, sdev, and its obs and 1/variance images, bit for bit."""
import math

import numpy as np
import pytest

import cases
from oracle.bindings import Reference
from shape_b200 import ctypes_defs as cd
from shape_b200 import engine as eng
from test_modfile import write_mod

OBS = """{ one delay-Doppler set }
1
0
c 0.5 c -0.3 c 190.0   { angle offsets (deg) }
c 0 c 0 c 0.2          { spin offsets (deg/day) }
delay-doppler
0                      { radar law }
3
2018 3 14 0 0 0  359.5 10.2 0.031
2018 3 15 0 0 0  0.4 10.0 0.030
2018 3 16 0 0 0  1.1 9.8 0.029
2380.0 20 0.5 1 1 long_orig
30 0.1 15.5 15.0 64
2018 3 14 12 0 0  2 c 0.25 c 0.01 c -0.002
c 1.0
1 0.0 center
d
3
f0.dat 2018 3 14 5 6 7  1.5  f 1.0  4 10.0 1.0 0
f1.dat 2018 3 14 17 0 0  1.2  c 2.0  0  9.5 0.8 0
f2.dat 2018 3 15 9 30 0  0.9  f 1.0  9 11.0 1.2 0
"""


@pytest.mark.parametrize("ltc,gamma,speckle", [(1, 1.0, 0), (0, 1.4, 1)])
def test_obs_matches_reference(tmp_path, monkeypatch, ltc, gamma, speckle):
    monkeypatch.chdir(tmp_path)
    m = cases.c1()[0]
    write_mod(tmp_path / "m.mod", m, seed=3)
    (tmp_path / "d").mkdir()
    rng = np.random.default_rng(12)
    for f in range(3):
        img = rng.normal(0, 1, (20, 30))
        img[0, 0] = -1.5
        if f == 2:
            (tmp_path / "d" / "f2.dat").write_bytes(img.astype(">f4").tobytes())
        else:
            (tmp_path / "d" / ("f%d.dat" % f)).write_text("\n".join(repr(float(x)) for x in img.ravel()) + "\n")
    (tmp_path / "t.obs").write_text(OBS)
    spin = eng.ModFile("m.mod").spin()
    o = eng.ObsFile("t.obs")
    info = o.set_info(0)
    assert o.nsets() == 1 and info["nframes"] == 3 and info["iradlaw"] == 0
    assert info["set"].codemethod == 1 and info["set"].Ftx == 2380.0
    frames, obs, oov, sdev = o.frames(0, spin, 75, 0.02, perform_ltc=ltc, dd_gamma=gamma, speckle=speckle)
    ref = Reference()
    h = ref.lib.ref_obs_read(b"m.mod", b"t.obs", ltc, gamma, speckle, 1)
    D = 20 * 30
    for f in range(3):
        g, nd = np.zeros(34), (eng.C.c_int * 2)()
        ro, rv = np.zeros(D), np.zeros(D)
        ref.lib.ref_obs_frame(h, 0, f, cd.as_dptr(g), nd, cd.as_dptr(ro), cd.as_dptr(rv))
        fr = frames[f]
        assert (nd[0], nd[1]) == (fr.ndel, fr.ndop) == (20, 30)
        assert list(fr.oe) == list(g[1:10]), f
        assert list(fr.ae) == list(g[13:22]), f
        assert list(fr.spin) == list(g[22:25]), f
        assert (fr.deloff, fr.dopoff) == (g[25], g[26]), f
        assert (fr.delcom_vig, fr.dopcom_vig, fr.dopDC_vig) == (g[27], g[28], g[29])
        assert (fr.weight, fr.dof, fr.cal, sdev[f]) == (g[30], g[31], g[32], g[33])
        assert fr.cal_floating == (f != 1)
        assert np.array_equal(obs[f * D:(f + 1) * D], ro) and np.array_equal(oov[f * D:(f + 1) * D], rv), f
        assert fr.pos_n == 75 and fr.km_per_pixel == 0.02


DOPPLER_SET = """0
c 0 c 0 c 0
c 0 c 0 c -0.1
doppler
0
2
2018 3 14 0 0 0  359.5 10.2 0.031
2018 3 16 0 0 0  1.1 9.8 0.029
2380.0 64 0.25 31.5
2018 3 14 12 0 0  1 c 0.25 c 0.03
f 1.0
1 0.0 first
d
2
s0.dat 2018 3 14 8 0 0  1.1  f 1.0  6  1.0 0
s1.dat 2018 3 15 2 0 0  0.7  c 1.5  0  0.5 0
"""


@pytest.mark.parametrize("speckle", [0, 1])
def test_obs_doppler_set_matches_reference(tmp_path, monkeypatch, speckle):
    """A delay-Doppler set followed by a Doppler set: the Doppler frames'
    view, offsets and spectra against the reference's read_doppler,
    dopoffs and realize_spin."""
    monkeypatch.chdir(tmp_path)
    write_mod(tmp_path / "m.mod", cases.c1()[0], seed=3)
    (tmp_path / "d").mkdir()
    rng = np.random.default_rng(5)
    for f in range(3):
        (tmp_path / "d" / ("f%d.dat" % f)).write_bytes(rng.normal(0, 1, (20, 30)).astype(">f4").tobytes())
    (tmp_path / "d" / "s0.dat").write_text("\n".join(repr(float(x)) for x in rng.normal(0, 1, 64)) + "\n")
    (tmp_path / "d" / "s1.dat").write_bytes((-np.abs(rng.normal(0, 1, 64))).astype(">f4").tobytes())
    (tmp_path / "t.obs").write_text(OBS.replace("{ one delay-Doppler set }\n1\n", "2\n", 1) + DOPPLER_SET)
    o = eng.ObsFile("t.obs")
    assert o.nsets() == 2 and o.set_type(0) == 0 and o.set_type(1) == 1
    spin = eng.ModFile("m.mod").spin()
    st, frames, obs, oov = o.doppler(1, spin, 60, 0.03, 2, 64, perform_ltc=1, speckle=speckle)
    assert st.dop_per_bin == 0.25 and st.Ftx == 2380.0 and st.dopscale == 1.0
    ref = Reference()
    h = ref.lib.ref_obs_read(b"m.mod", b"t.obs", 1, 1.0, speckle, 1)
    for f in range(2):
        g, nd = np.zeros(31), (eng.C.c_int * 1)()
        ro, rv = np.zeros(64), np.zeros(64)
        ref.lib.ref_obs_doppler_frame(h, 1, f, cd.as_dptr(g), nd, cd.as_dptr(ro), cd.as_dptr(rv))
        fr = frames[f]
        assert nd[0] == fr.ndop == 64
        assert list(fr.oe) == list(g[1:10]) and list(fr.ae) == list(g[13:22]) and list(fr.spin) == list(g[22:25])
        assert (fr.dopoff, fr.dopcom_vig, fr.weight, fr.dof, fr.cal, fr.sdev) == tuple(g[25:31]), f
        assert np.array_equal(obs[64 * f:64 * (f + 1)], ro) and np.array_equal(oov[64 * f:64 * (f + 1)], rv), f


def test_obs_refusals(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    p = tmp_path / "u.obs"
    p.write_text(OBS.replace("delay-doppler", "radar-image"))
    with pytest.raises(eng.EngineError, match="error -4"):
        eng.ObsFile(p)
    p.write_text(OBS.replace("1 0.0 center", "0 60.0 center"))
    with pytest.raises(eng.EngineError, match="error -1"):
        eng.ObsFile(p)
    p.write_text("1\n" + DOPPLER_SET.replace("1 0.0 first", "3 60.0 first"))
    with pytest.raises(eng.EngineError, match="error -4"):
        eng.ObsFile(p)
    # a weighted frame whose mask file is missing: refused when its sizes
    # are asked for
    p.write_text(OBS.replace("1.0 0\nf1", "1.0 1\nf1"))
    with pytest.raises(eng.EngineError, match="mask"):
        eng.ObsFile(p).set_info(0)
    p.write_text(OBS.replace("long_orig", "long9"))
    with pytest.raises(eng.EngineError, match="error -1"):
        eng.ObsFile(p)


TIED_DOPPLER_SET = """0
= 0 c 0.3 = 0
= 0 c 0 = 0
doppler
0
2
2018 3 14 0 0 0  359.5 10.2 0.031
2018 3 16 0 0 0  1.1 9.8 0.029
2380.0 64 0.25 31.5
2018 3 14 12 0 0  2 = 9.0 = 9.0 = 9.0
f 1.0
1 0.0 first
d
2
s0.dat 2018 3 14 8 0 0  1.1  f 1.0  6  1.0 0
s1.dat 2018 3 15 2 0 0  0.7  c 1.5  0  0.5 0
"""


def test_obs_tied_sets_match_reference(tmp_path, monkeypatch):
    """A Doppler set that ties components of its angle and spin offsets and
    its delay-correction polynomial (same epoch) to the delay-Doppler
    set before it with the = state: the tied values are the earlier set's,
    as the reference's realize_angleoff / realize_omegaoff / realize_delcor
    make them, so the Doppler frames' body matrices, spin vectors and
    Doppler offsets equal the reference's bit for bit."""
    monkeypatch.chdir(tmp_path)
    write_mod(tmp_path / "m.mod", cases.c1()[0], seed=3)
    (tmp_path / "d").mkdir()
    rng = np.random.default_rng(8)
    for f in range(3):
        (tmp_path / "d" / ("f%d.dat" % f)).write_bytes(rng.normal(0, 1, (20, 30)).astype(">f4").tobytes())
    for f in range(2):
        (tmp_path / "d" / ("s%d.dat" % f)).write_bytes(rng.normal(0, 1, 64).astype(">f4").tobytes())
    (tmp_path / "t.obs").write_text(OBS.replace("{ one delay-Doppler set }\n1\n", "2\n", 1) + TIED_DOPPLER_SET)
    o = eng.ObsFile("t.obs")
    a0, a1 = o.set_info(0), o.set_info(1)
    assert a1["angleoff"][0] == a0["angleoff"][0] and a1["angleoff"][2] == a0["angleoff"][2]
    assert a1["omegaoff"][0] == a0["omegaoff"][0] and a1["omegaoff"][2] == a0["omegaoff"][2]
    assert a1["angleoff"][1] != a0["angleoff"][1]
    spin = eng.ModFile("m.mod").spin()
    st, frames, obs, oov = o.doppler(1, spin, 60, 0.03, 2, 64, perform_ltc=1)
    ref = Reference()
    h = ref.lib.ref_obs_read(b"m.mod", b"t.obs", 1, 1.0, 0, 1)
    for f in range(2):
        g, nd = np.zeros(31), (eng.C.c_int * 1)()
        ro, rv = np.zeros(64), np.zeros(64)
        ref.lib.ref_obs_doppler_frame(h, 1, f, cd.as_dptr(g), nd, cd.as_dptr(ro), cd.as_dptr(rv))
        fr = frames[f]
        assert list(fr.oe) == list(g[1:10]) and list(fr.ae) == list(g[13:22]) and list(fr.spin) == list(g[22:25])
        assert (fr.dopoff, fr.dopcom_vig, fr.weight, fr.dof, fr.cal, fr.sdev) == tuple(g[25:31]), f


def test_obs_tie_refusals(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    p = tmp_path / "u.obs"
    p.write_text(OBS.replace("c 0.5 c -0.3 c 190.0", "= 0.5 c -0.3 c 190.0"))
    with pytest.raises(eng.EngineError, match="first dataset's angle offsets"):
        eng.ObsFile(p)
    two = OBS.replace("{ one delay-Doppler set }\n1\n", "2\n", 1)
    p.write_text(two + TIED_DOPPLER_SET.replace("2 = 9.0 = 9.0 = 9.0", "1 = 9.0 = 9.0"))
    with pytest.raises(eng.EngineError, match="same degree"):
        eng.ObsFile(p)
    p.write_text(two + TIED_DOPPLER_SET.replace("12 0 0  2 =", "12 0 1  2 ="))
    with pytest.raises(eng.EngineError, match="same epoch"):
        eng.ObsFile(p)
    p.write_text(OBS.replace("0                      { radar law }", "-1"))
    with pytest.raises(eng.EngineError, match="observation file line .*negative radar law"):
        eng.ObsFile(p)


LC_SETS = """0
c 0 c 0 c 10.0
c 0 c 0 c 0.05
lightcurve
0
3
2018 3 14 0 0 0  359.5 10.2 0.031
2018 3 15 0 0 0  0.4 10.0 0.030
2018 3 16 0 0 0  1.1 9.8 0.029
3
2018 3 14 0 0 0  170.0 -5.0 0.99
2018 3 15 0 0 0  171.0 -5.4 0.99
2018 3 16 0 0 0  172.0 -5.8 0.99
{CALC}
1 0.0 center
5 lc{K}.dat f 1.0 1.5
"""

HELIO_SET = """0
= 0 c -2.0 c 0
c 0 c 0 c 0
heliocurve
1
3
2018 3 14 0 0 0  10.0 2.0 1.02
2018 3 15 0 0 0  10.5 2.1 1.02
2018 3 16 0 0 0  11.0 2.2 1.02
3
2018 3 14 0 0 0  8.0 1.0 1.0
2018 3 15 0 0 0  8.9 1.1 1.0
2018 3 16 0 0 0  9.8 1.2 1.0
-1
1 0.0 first
5 lc9.dat c 2.5 0.8
"""


@pytest.mark.parametrize("ltc", [1, 0])
def test_obs_lightcurve_sets_match_reference(tmp_path, monkeypatch, ltc):
    """Lightcurve sets with explicit, evenly spaced and observation-derived
    calculated epochs, and a heliocurve set, against the reference's
    read_lghtcrv and realize_spin (which read a heliocurve set's tables as a
    lightcurve set's): epochs, observer / Sun / body matrices,
    solar phases, intensities, 1/variance, weight, dof and calibration bit
    for bit."""
    monkeypatch.chdir(tmp_path)
    write_mod(tmp_path / "m.mod", cases.c1()[0], seed=3)
    rng = np.random.default_rng(31)
    calcs = ["3\n2458191.8 2458192.3 2458192.9", "0\n2458191.75 2458193.0 0.25", "-1"]
    text = "%d\n" % (len(calcs) + 1)
    for k, calc in enumerate(calcs):
        ep = np.sort(rng.uniform(2458191.8, 2458192.8, 5))
        if k == 2:
            ep[3] = ep[2]                       # a repeated epoch: calculated once
        (tmp_path / ("lc%d.dat" % k)).write_text("".join("%.9f %.6f %.6f\n" % (e, 14 + rng.normal(0, 0.2), 0.02)
                                                      for e in ep))
        text += LC_SETS.replace("{CALC}", calc).replace("{K}", str(k))
    (tmp_path / "lc9.dat").write_text("".join("%.9f %.6f %.6f\n" % (e, 13.5, 0.03)
                                              for e in np.sort(rng.uniform(2458191.8, 2458192.8, 5))))
    text += HELIO_SET
    (tmp_path / "t.obs").write_text(text)
    o = eng.ObsFile("t.obs")
    spin = eng.ModFile("m.mod").spin()
    ref = Reference()
    h = ref.lib.ref_obs_read(b"m.mod", b"t.obs", ltc, 1.0, 0, 1)
    for s in range(4):
        assert o.set_type(s) == 2
        info = o.lghtcrv_info(s)
        sizes = (eng.C.c_int * 3)()
        ref.lib.ref_obs_lghtcrv(h, s, sizes, None, None, None, None, None, None)
        assert (info["ioptlaw"], info["ncalc"], info["n"]) == tuple(sizes), s
        nc, n = info["ncalc"], info["n"]
        x, pt, t, ob, ov, tail = (np.zeros(nc), np.zeros(28 * nc), np.zeros(n), np.zeros(n), np.zeros(n),
                                  np.zeros(3))
        ref.lib.ref_obs_lghtcrv(h, s, sizes, cd.as_dptr(x), cd.as_dptr(pt), cd.as_dptr(t), cd.as_dptr(ob),
                                cd.as_dptr(ov), cd.as_dptr(tail))
        ds = o.lghtcrv(s, spin, 60, 0.03, sun_appmag=-26.75, perform_ltc=ltc)
        assert np.array_equal(ds.x, x), s
        assert np.array_equal(ds.t, t) and np.array_equal(ds.obs, ob) and np.array_equal(ds.oneovervar, ov), s
        for i, p in enumerate(ds.points):
            g = pt[28 * i:28 * (i + 1)]
            assert list(p.oe) == list(g[0:9]) and list(p.se) == list(g[9:18]) and list(p.ae) == list(g[18:27]), (s, i)
            assert p.solar_phase == g[27], (s, i)
        assert (ds.set.weight, ds.set.dof, ds.set.cal) == tuple(tail), s
        assert ds.set.cal_floating == (s < 3)
    assert o.lghtcrv_info(2)["ncalc"] == 4          # five epochs, one repeated


def _smeared_files(tmp_path, mode, nviews):
    m = cases.c1()[0]
    write_mod(tmp_path / "m.mod", m, seed=3)
    (tmp_path / "d").mkdir()
    rng = np.random.default_rng(21)
    for f in range(3):
        img = rng.normal(0, 1, (20, 30))
        if f == 2:
            (tmp_path / "d" / "f2.dat").write_bytes(img.astype(">f4").tobytes())
        else:
            (tmp_path / "d" / ("f%d.dat" % f)).write_text("\n".join(repr(float(x)) for x in img.ravel()) + "\n")
    (tmp_path / "t.obs").write_text(OBS.replace("1 0.0 center", "%d 1800.0 %s" % (nviews, mode)))
    return m


@pytest.mark.parametrize("mode,nviews,ltc", [("center", 3, 1), ("first", 4, 0), ("center", 4, 1)])
def test_obs_smeared_views_match_reference(tmp_path, monkeypatch, mode, nviews, ltc):
    """Every view of every frame of a smeared set (read_deldop's view
    epochs t0 + (k - v0) * interval, light-time corrected, each view's
    observer matrix, orbital spin, delay / Doppler offsets and realized
    spin), listed in rendering order, bit for bit against read_dat."""
    monkeypatch.chdir(tmp_path)
    _smeared_files(tmp_path, mode, nviews)
    spin = eng.ModFile("m.mod").spin()
    o = eng.ObsFile("t.obs")
    nv, v0 = o.views(0)
    assert nv == nviews and v0 == (nviews // 2 if mode == "center" else 0)
    with pytest.raises(eng.EngineError, match="error -4"):
        o.frames(0, spin, 75, 0.02, perform_ltc=ltc)
    views, obs, oov, sdev = o.frame_views(0, spin, 75, 0.02, perform_ltc=ltc)
    ref = Reference()
    h = ref.lib.ref_obs_read(b"m.mod", b"t.obs", ltc, 1.0, 0, 1)
    rv = (eng.C.c_int * 2)()
    ref.lib.ref_obs_views(h, 0, rv)
    assert (rv[0], rv[1]) == (nv, v0)
    D = 20 * 30
    for f in range(3):
        assert len(views[f]) == nv
        for j, V in enumerate(views[f]):
            k = (v0 + 1 + j) % nv
            g, nd = np.zeros(34), (eng.C.c_int * 2)()
            ro, rvv = np.zeros(D), np.zeros(D)
            ref.lib.ref_obs_frame_view(h, 0, f, k, cd.as_dptr(g), nd, cd.as_dptr(ro), cd.as_dptr(rvv))
            assert list(V.oe) == list(g[1:10]), (f, k)
            assert list(V.ae) == list(g[13:22]), (f, k)
            assert list(V.spin) == list(g[22:25]), (f, k)
            assert (V.deloff, V.dopoff) == (g[25], g[26]), (f, k)
            assert (V.delcom_vig, V.dopcom_vig, V.dopDC_vig, V.weight, V.dof, V.cal) == tuple(g[27:33])
            assert np.array_equal(obs[f * D:(f + 1) * D], ro) and np.array_equal(oov[f * D:(f + 1) * D], rvv)
        # the epoch view closes the list, and the views differ
        assert list(views[f][-1].ae) != list(views[f][0].ae)


def _mask(nd, np_, rng, rows, cols):
    w = np.zeros((nd, np_))
    w[rows[0]:rows[1], cols[0]:cols[1]] = rng.uniform(0.2, 1.5, (rows[1] - rows[0], cols[1] - cols[0]))
    w[min(rows[0] + 1, nd - 1), cols[0] + 2] = 0.0     # a hole inside the window
    return w


def test_obs_masks_match_reference(tmp_path, monkeypatch):
    """Pixel-weighting masks (mask_SS_FF.txt in the data directory) on two
    of three delay-Doppler frames and on one Doppler frame: each frame's
    window of positive weights, its COM and DC bins counted from the window,
    dof (weight per positive weight) and 1/variance times the weights, bit
    for bit against read_dat; then the same masks from a mask directory."""
    monkeypatch.chdir(tmp_path)
    m = cases.c1()[0]
    write_mod(tmp_path / "m.mod", m, seed=3)
    (tmp_path / "d").mkdir()
    rng = np.random.default_rng(31)
    for f in range(3):
        img = rng.normal(0, 1, (20, 30))
        (tmp_path / "d" / ("f%d.dat" % f)).write_text("\n".join(repr(float(x)) for x in img.ravel()) + "\n")
    for f in range(2):
        spec = rng.normal(0, 1, 64)
        (tmp_path / "d" / ("s%d.dat" % f)).write_text("\n".join(repr(float(x)) for x in spec) + "\n")
    masks = {(0, 0): _mask(20, 30, rng, (3, 15), (4, 27)), (0, 2): _mask(20, 30, rng, (0, 20), (10, 30)),
             (1, 1): _mask(1, 64, np.random.default_rng(2), (0, 1), (5, 50))}
    mdir = tmp_path / "masks"
    mdir.mkdir()
    for (s_, f), w in masks.items():
        txt = "{ weights }\n" + "\n".join("%.6f" % x for x in w.ravel()) + "\n"
        (tmp_path / "d" / ("mask_%02d_%02d.txt" % (s_, f))).write_text(txt)
        (mdir / ("mask_%02d_%02d.txt" % (s_, f))).write_text(txt)
    def swap(t, a, b):
        assert t.count(a) == 1, a
        return t.replace(a, b)
    obs = swap(OBS, "f0.dat 2018 3 14 5 6 7  1.5  f 1.0  4 10.0 1.0 0", "f0.dat 2018 3 14 5 6 7  1.5  f 1.0  4 10.0 1.0 1")
    obs = swap(obs, "9 11.0 1.2 0", "9 11.0 1.2 1")
    dop = swap(DOPPLER_SET, "s1.dat 2018 3 15 2 0 0  0.7  c 1.5  0  0.5 0", "s1.dat 2018 3 15 2 0 0  0.7  c 1.5  0  0.5 1")
    text = obs.replace("{ one delay-Doppler set }\n1\n", "{ two sets }\n2\n") + dop
    (tmp_path / "t.obs").write_text(text)
    spin = eng.ModFile("m.mod").spin()
    ref = Reference()
    h = ref.lib.ref_obs_read(b"m.mod", b"t.obs", 1, 1.0, 0, 1)
    for maskdir in (None, mdir):
        o = eng.ObsFile("t.obs")
        if maskdir is not None:
            o.set_maskdir(maskdir)
        frames, ob, ov, sdev = o.frames(0, spin, 75, 0.02)
        off = 0
        for f in range(3):
            g, nd = np.zeros(34), (eng.C.c_int * 2)()
            D = 20 * 30
            ro, rv = np.zeros(D), np.zeros(D)
            ref.lib.ref_obs_frame(h, 0, f, cd.as_dptr(g), nd, cd.as_dptr(ro), cd.as_dptr(rv))
            fr = frames[f]
            n = nd[0] * nd[1]
            assert (fr.ndel, fr.ndop) == (nd[0], nd[1]), f
            assert (fr.delcom_vig, fr.dopcom_vig, fr.dopDC_vig) == (g[27], g[28], g[29]), f
            assert (fr.weight, fr.dof) == (g[30], g[31]), f
            assert np.array_equal(ob[off:off + n], ro[:n]) and np.array_equal(ov[off:off + n], rv[:n]), f
            off += n
        assert (frames[0].ndel, frames[0].ndop) == (12, 23) and frames[1].ndel == 20
        st, dfr, dob, dov = o.doppler(1, spin, 75, 0.02)
        off = 0
        for f in range(2):
            g, nd = np.zeros(31), (eng.C.c_int * 1)()
            ro, rv = np.zeros(64), np.zeros(64)
            ref.lib.ref_obs_doppler_frame(h, 1, f, cd.as_dptr(g), nd, cd.as_dptr(ro), cd.as_dptr(rv))
            n = nd[0]
            assert dfr[f].ndop == n
            assert (dfr[f].dopcom_vig, dfr[f].dof) == (g[26], g[28]), f
            assert np.array_equal(dob[off:off + n], ro[:n]) and np.array_equal(dov[off:off + n], rv[:n]), f
            off += n
        assert dfr[1].ndop == 45


POS_SET = """0
c 0 c 0 c 10.0
c 0 c 0 c 0.05
plane-of-sky
0
3
2018 3 14 0 0 0  359.5 10.2 0.031
2018 3 15 0 0 0  0.4 10.0 0.030
2018 3 16 0 0 0  1.1 9.8 0.029
3
2018 3 14 0 0 0  170.0 -5.0 0.99
2018 3 15 0 0 0  171.0 -5.4 0.99
2018 3 16 0 0 0  172.0 -5.8 0.99
0.25
1 0.0 center
imgs
2
f0.fits 2018 3 14 12 0 0  30.0  c 1.5 c -0.5  1.0 0
f1.fits 2018 3 15 6 0 0  -12.5 f 0.25 c 0  2.0 1
"""


@pytest.mark.parametrize("ltc", [0, 1])
def test_obs_poset_geometry(tmp_path, monkeypatch, ltc):
    """A plane-of-sky set in the .obs grammar (read_poset): its frames'
    observer, Sun and body matrices and solar phases equal those of a
    lightcurve set with the same ephemerides and offsets whose calculated
    epochs are the frames' epochs (a reader pinned to the reference's
    read_lghtcrv); north angles to radians, COM offsets, weights, image
    files and mask flags as written; the fit grid's km per pixel is the
    angular pixel size times the distance before the light-time
    correction."""
    monkeypatch.chdir(tmp_path)
    write_mod(tmp_path / "m.mod", cases.c1()[0], seed=3)
    (tmp_path / "lc0.dat").write_text("".join("%.3f 14.0 0.02\n" % (2458192.0 + 0.2 * k) for k in range(5)))
    lc = LC_SETS.replace("{CALC}", "2\n2458192.0 2458192.75").replace("{K}", "0")
    (tmp_path / "t.obs").write_text("2\n" + POS_SET + lc)
    o = eng.ObsFile("t.obs")
    spin = eng.ModFile("m.mod").spin()
    assert o.set_type(0) == 3 and o.set_type(1) == 2
    frames, files, law = o.poset(0, spin, perform_ltc=ltc)
    ds = o.lghtcrv(1, spin, 60, 0.03, perform_ltc=ltc)
    assert law == 0 and len(frames) == 2
    assert files == [("imgs/f0.fits", 0), ("imgs/f1.fits", 1)]
    D2R = math.pi / 180.0
    for f, (fr, p) in enumerate(zip(frames, ds.points)):
        assert list(fr.oe) == list(p.oe) and list(fr.se) == list(p.se) and list(fr.ae) == list(p.ae), f
        assert fr.solar_phase == p.solar_phase, f
    np.testing.assert_allclose([frames[0].northangle, frames[1].northangle], [30.0 * D2R, -12.5 * D2R],
                               rtol=1e-15)
    assert (frames[0].xoff, frames[0].yoff, frames[1].xoff, frames[1].yoff) == (1.5, -0.5, 0.25, 0.0)
    assert (frames[0].weight, frames[1].weight) == (1.0, 2.0)
    rows = [(2458191.5 + k, r * D2R, d * D2R, a) for k, (r, d, a) in
            enumerate([(359.5, 10.2, 0.031), (0.4, 10.0, 0.030), (1.1, 9.8, 0.029)])]
    for fr, t0 in zip(frames, (2458192.0, 2458192.75)):
        dist = eng.ephem_view(rows, t0)["dist"]
        want = (0.25 / 3600) * D2R * (dist * 1.4959787061e8)
        assert abs(fr.fit_km_per_pixel - want) <= 1e-15 * want
