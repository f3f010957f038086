"""Seeded synthetic inputs have the benchmark configurations' sizes."""
import numpy as np

from shape_b200 import synth


def _check_model(m, nv, nf):
    assert (m.nv, m.nf) == (nv, nf)
    x = m.a + m.u * m.r[:, None]
    p0, p1, p2 = x[m.fv[:, 0]], x[m.fv[:, 1]], x[m.fv[:, 2]]
    nrm = np.cross(p1 - p0, p2 - p1)
    assert (np.einsum("ij,ij->i", nrm, (p0 + p1 + p2) / 3) > 0).all(), "facets not outward"
    assert m.af_ptr[-1] == 3 * nf
    for i in (0, nv // 2, nv - 1):
        lst = m.af_idx[m.af_ptr[i]:m.af_ptr[i + 1]]
        assert (np.diff(lst) > 0).all() and all(i in m.fv[f] for f in lst)


def test_model_sizes():
    _check_model(synth.ellipsoid_model(), 1152, 2300)
    _check_model(synth.harmonic_model(), 4002, 8000)
    _check_model(synth.noisy_octa_model(), 16386, 32768)


def test_harmonic_deviation_rms():
    m = synth.harmonic_model()
    assert abs(np.sqrt(((m.r - 1.0) ** 2).mean()) - 0.05) < 1e-12


def test_config_datasets_shapes():
    p = synth.eval_params()
    c1 = synth.config1_dataset(None, p)
    assert c1.nframes == 1 and c1.frames[0].pos_n == 75 and (c1.frames[0].ndel, c1.frames[0].ndop) == (100, 100)
    c2 = synth.config2_dataset(None, p)
    assert c2.nframes == 64
    for f in c2.frames:
        assert 101 <= 2 * f.pos_n + 1 <= 301 and 64 <= f.ndel <= 256 and 64 <= f.ndop <= 512
    c4 = synth.config4_dataset(None, p)
    assert c4.nframes == 16 and all(f.pos_n == 255 and f.ndel == 256 and f.ndop == 256 for f in c4.frames)
    lcs = synth.config3_datasets(None, p, npoints=20)
    assert len(lcs) == 4 and all(len(l.points) == 20 for l in lcs)
    for l in lcs:
        ph = l.points[0].solar_phase * 180 / np.pi
        assert 5 <= ph <= 60
