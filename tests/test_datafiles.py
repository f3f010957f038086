"""Radar data files (shape_read_radar_data) against the reference's own
readers (read_deldop_ascii / _binary / _rdf and read_doppler_*, via
ref_read_radar_data), on the CPU: float32 images written as ASCII (with
comments, line breaks and numbers carrying more digits than a float, so the
rounding to float matters), as big- and little-endian raw float32 and as
RDF, cropped to windows; the kept values times sdev must equal the
reference's bit for bit. The gamma transform and the 1/variance with
speckle and pixel weights follow read_deldop's formulas."""
import math

import numpy as np
import pytest

from oracle.bindings import Reference
from shape_b200 import engine as eng


@pytest.fixture(scope="module")
def ref():
    return Reference()


def _image(seed, ndel, ndop):
    rng = np.random.default_rng(seed)
    img = rng.normal(0.0, 1.0, (ndel, ndop)) * 10.0 ** rng.integers(-3, 4, (ndel, ndop))
    img.flat[0] = -abs(img.flat[0]) - 1.0            # a byte >= 128 at the start of raw float32
    return img


def _ascii(path, img, rng):
    parts = []
    for x in img.ravel():
        parts.append(repr(float(x)))                 # up to 17 digits: rounded to float on reading
        r = rng.random()
        if r < 0.03:
            parts.append("{ comment }")
        parts.append("\n" if r < 0.2 else " ")
    path.write_text("".join(parts))


def _rdf(path, img):
    header = "type = delay-doppler image\n" + "".join("{ header line %d }\n" % i for i in range(8)) + ".\n"
    assert len(header) > 128
    path.write_bytes(header.encode() + img.astype(">f4").tobytes())


@pytest.mark.parametrize("doppler", [False, True])
def test_radar_data_matches_reference(tmp_path, ref, doppler):
    ndel, ndop = (1, 301) if doppler else (37, 53)
    img = _image(4 + doppler, ndel, ndop)
    rng = np.random.default_rng(11)
    windows = [((1, ndel), (1, ndop)), ((1, 1) if doppler else (5, 30), (10, ndop - 7))]
    sdev = 0.37
    files = {}
    _ascii(tmp_path / "a.dat", img, rng)
    files["ascii"] = (tmp_path / "a.dat", 0, True)
    (tmp_path / "b.dat").write_bytes(img.astype(">f4").tobytes())
    files["binary_big"] = (tmp_path / "b.dat", 1, True)
    (tmp_path / "l.dat").write_bytes(img.astype("<f4").tobytes())
    files["binary_little"] = (tmp_path / "l.dat", 1, False)
    _rdf(tmp_path / "r.rdf", img)
    files["rdf"] = (tmp_path / "r.rdf", 2, True)
    for name, (path, kind, big) in files.items():
        for dl, dp in windows:
            mine, oov = eng.read_radar_data(path, ndel, ndop, dl, dp, big_endian=big, sdev=sdev)
            theirs = ref.read_radar_data(str(path), kind + 3 * doppler, ndel, ndop, dl, dp,
                                         1 if big else 0, sdev)   # this host is little-endian
            assert np.array_equal(mine.ravel(), theirs), (name, dl, dp)
            want = img[dl[0] - 1:dl[1], dp[0] - 1:dp[1]].astype(np.float32).astype(np.float64) * sdev
            assert np.array_equal(mine, want), name
            assert np.all(oov == 1 / math.pow(sdev, 2.0))


def test_radar_data_gamma_speckle_weights(tmp_path):
    img = _image(7, 9, 40)
    p = tmp_path / "b.dat"
    p.write_bytes(img.astype(">f4").tobytes())
    w = np.random.default_rng(2).uniform(0.5, 1.5, img.shape)
    sdev, gamma, nlooks = 0.9, 1.6, 12.0
    obs, oov = eng.read_radar_data(p, 9, 40, (2, 8), (3, 37), sdev=sdev, gamma=gamma, nlooks=nlooks, pixweight=w)
    look = 1 / math.sqrt(nlooks)
    for j in range(7):
        for k in range(35):
            o = float(np.float32(img[j + 1, k + 2])) * sdev
            if o > 0.0:
                o = math.pow(o, 1 / gamma)
            assert obs[j, k] == o
            assert oov[j, k] == 1 / (math.pow(sdev, 2.0) + math.pow(look * o, 2.0)) * w[j + 1, k + 2]


def test_radar_data_refusals(tmp_path):
    p = tmp_path / "f.fits"
    p.write_text("SIMPLE  =                    T" + " " * 200)
    with pytest.raises(eng.EngineError, match="error -4"):
        eng.read_radar_data(p, 2, 2)
    p.write_text("1 2 3")
    with pytest.raises(eng.EngineError, match="128 bytes"):
        eng.read_radar_data(p, 1, 3)
    p.write_bytes(_image(1, 4, 40).astype(">f4").tobytes())
    with pytest.raises(eng.EngineError, match="too short"):
        eng.read_radar_data(p, 5, 40)
    with pytest.raises(eng.EngineError):
        eng.read_radar_data(p, 4, 40, (0, 4), (1, 40))


def test_lightcurve_data(tmp_path):
    """read_lghtcrv's conversion (src/shape/read_dat.c:1925-1956), restated
    with the same operations: magnitudes to intensities relative to the Sun
    and their 1/variance."""
    rng = np.random.default_rng(8)
    n, sun = 40, -26.74
    rows = [(2458000.0 + 0.01 * i + rng.uniform(0, 1e-3), rng.uniform(12, 16), rng.uniform(0.005, 0.05))
            for i in range(n)]
    p = tmp_path / "lc.dat"
    p.write_text("{ JD mag err }\n" + "".join("%r %r %r\n" % r for r in rows))
    t, obs, oov = eng.read_lghtcrv_data(p, n, sun)
    ln10 = 2.302585092994046
    for i, (jd, mag, err) in enumerate(rows):
        intens = math.exp(-0.4 * ln10 * (mag - sun))
        e = (0.4 * ln10 * err) * intens
        assert t[i] == jd and obs[i] == intens and oov[i] == 1.0 / (e * e)
    with pytest.raises(eng.EngineError, match="end of file"):
        eng.read_lghtcrv_data(p, n + 1, sun)
