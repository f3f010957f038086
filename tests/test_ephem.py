"""View geometry from ephemerides (shape_ephem_view) against the reference's
own ephem2mat (via ref_ephem2mat), on the CPU: observer matrices, the
plane-of-sky spin contribution, the distance, and in the bistatic case the
solar matrix, phase and azimuth, bit for bit, over seeded tables whose RA
crosses the 0/360 line and epochs at table entries and between them."""
import numpy as np
import pytest

from oracle.bindings import Reference
from shape_b200 import ctypes_defs as cd
from shape_b200 import engine as eng


@pytest.fixture(scope="module")
def ref():
    return Reference()


def _table(rng, n, t0, ra0, dist0):
    t = t0 + np.cumsum(rng.uniform(0.2, 1.5, n))
    ra = np.mod(ra0 + np.cumsum(rng.normal(0.02, 0.05, n)), 2 * np.pi)
    dec = np.clip(rng.normal(0.2, 0.01, n).cumsum() / np.arange(1, n + 1) * 3, -1.4, 1.4)
    dist = dist0 + np.cumsum(rng.normal(0, 0.003, n))
    return np.stack([t, ra, dec, dist], 1)


def _ref(ref, ast, sun, t):
    oe, se, s, pa = np.zeros(9), np.zeros(9), np.zeros(3), np.zeros(2)
    a = np.ascontiguousarray(ast, dtype=np.float64)
    b = np.ascontiguousarray(sun if sun is not None else np.zeros((1, 4)), dtype=np.float64)
    d = ref.lib.ref_ephem2mat(cd.as_dptr(a), len(a), cd.as_dptr(b), 0 if sun is None else len(b), t,
                              cd.as_dptr(oe), cd.as_dptr(se), cd.as_dptr(s), cd.as_dptr(pa))
    return oe.reshape(3, 3), se.reshape(3, 3), s, pa, d


@pytest.mark.parametrize("seed", range(4))
def test_ephem_view_matches_reference(ref, seed):
    rng = np.random.default_rng(300 + seed)
    ast = _table(rng, 12, 2458000.0, 6.2 if seed % 2 else 1.0, 0.05)
    sun = _table(rng, 12, 2457999.5, 3.0, 1.0)
    sun[-1, 0] = ast[-1, 0] + 1.0
    ts = list(ast[1:-1, 0]) + list(rng.uniform(ast[0, 0], ast[-1, 0], 10))
    for t in ts:
        for bistatic in (False, True):
            got = eng.ephem_view(ast, t, sun if bistatic else None)
            oe, se, s, pa, d = _ref(ref, ast, sun if bistatic else None, t)
            assert np.array_equal(got["oe"], oe) and np.array_equal(got["s"], s) and got["dist"] == d
            if bistatic:
                assert np.array_equal(got["se"], se)
                assert (got["solar_phase"], got["solar_azimuth"]) == (pa[0], pa[1])
            else:
                assert got["solar_phase"] == 0.0 and got["solar_azimuth"] == 0.0
            assert np.allclose(got["oe"] @ got["oe"].T, np.eye(3), atol=1e-14)


def test_ephem_view_out_of_range():
    rng = np.random.default_rng(1)
    ast = _table(rng, 5, 2458000.0, 1.0, 0.05)
    with pytest.raises(eng.EngineError):
        eng.ephem_view(ast, ast[0, 0] - 0.1)
    with pytest.raises(eng.EngineError):
        eng.ephem_view(ast, ast[-1, 0] + 0.1)
    with pytest.raises(eng.EngineError):
        eng.ephem_view(ast[:1], ast[0, 0])


def test_radar_view_light_time(ref):
    """The light-time-corrected view: the reference's sequence of two
    ephem2mat calls with the epoch moved by 5.775518328e-3 day per AU."""
    rng = np.random.default_rng(77)
    ast = _table(rng, 10, 2458000.0, 2.0, 0.03)
    for t in rng.uniform(ast[1, 0], ast[-1, 0], 8):
        _, _, _, _, d = _ref(ref, ast, None, t)
        tl = t - 5.775518328e-3 * d
        oe, _, s, _, _ = _ref(ref, ast, None, tl)
        tv, goe, gs = eng.ephem_radar_view(ast, t, True)
        assert tv == tl and np.array_equal(goe, oe) and np.array_equal(gs, s)
        tv0, goe0, _ = eng.ephem_radar_view(ast, t, False)
        assert tv0 == t and np.array_equal(goe0, _ref(ref, ast, None, t)[0])


@pytest.mark.parametrize("order", [0, 1, 3])
def test_delcor_offsets_match_reference(ref, order):
    rng = np.random.default_rng(40 + order)
    a = rng.normal(0, 1, order + 1) * 10.0 ** -np.arange(order + 1)
    t0 = 2458000.5
    t = t0 + rng.uniform(-3, 3, 9)
    delpp, doppp, ftx = 0.125, 0.0763, 2380.0
    d_ref, p_ref = np.zeros(9), np.zeros(9)
    ref.lib.ref_deldopoffs(cd.as_dptr(a), order, t0, 9, cd.as_dptr(t), delpp, doppp, ftx, cd.as_dptr(d_ref),
                           cd.as_dptr(p_ref))
    for k in range(9):
        assert eng.delcor_offsets(a, t0, t[k], delpp, doppp, ftx) == (d_ref[k], p_ref[k])
