"""The raster autotuner (shape_engine_set_raster_tuning /
shape_engine_get_raster_tuning): every candidate kernel and grid computes
the same images, the tuned form records the candidates' measured times and
runs the fastest, and a second engine of the same size class reuses the
choice without timing again.

Bars: facet, z and cos(e) maps bit-exact between candidates (FP64 batched
form, and the FP32 form's exact variant); fit images and chi-square to
relative 1e-12 in FP64 and 1e-5 / 1e-6 in FP32 (the scatter-add order
differs between kernels and launches, and FP32 images round each add)."""
import numpy as np
import pytest

import cases
from shape_b200 import engine as eng

pytestmark = pytest.mark.gpu


def _run(m, p, ds, mode, form):
    e = eng.make_engine(m, p, deldops=[ds])
    e.set_raster_tuning(mode)
    e.keep_pos(True)
    s = e.evaluate(form)
    maps = [e.pos(f) for f in range(ds.nframes)]
    fits = [e.fit(f) for f in range(ds.nframes)]
    info = e.raster_tuning(form)
    e.close()
    return s, maps, fits, info


@pytest.mark.parametrize("form", [eng.FORM_BATCHED_FP64, eng.FORM_BATCHED_FP32])
def test_candidates_agree(cuda_device, form):
    m, p, ds = cases.c2(12)
    ref = None
    for mode in (0, 1, -1):
        s, maps, fits, info = _run(m, p, ds, mode, form)
        assert info["tuned"]
        if mode >= 0:
            assert info["variant"] == mode and info["persistent"] == 0
        else:
            ms = info["ms"]
            assert all(t > 0 for t in ms), ms
            best = int(np.argmin(ms))
            assert (info["variant"], info["persistent"]) == (best >> 1, best & 1)
        if ref is None:
            ref = (s, maps, fits)
            continue
        fit_tol, chi2_tol = (1e-5, 1e-6) if form == eng.FORM_BATCHED_FP32 else (1e-12, 1e-12)
        for f in range(ds.nframes):
            for k in ("f", "z", "cose"):
                assert np.array_equal(maps[f][k], ref[1][f][k]), (mode, f, k)
            scale = max(np.abs(ref[2][f]).max(), 1e-300)
            assert np.abs(fits[f] - ref[2][f]).max() <= fit_tol * scale, (mode, f)
        assert abs(s["chi2"] - ref[0]["chi2"]) <= chi2_tol * abs(ref[0]["chi2"]), mode


def test_choice_is_shared_by_size_class(cuda_device):
    m, p, ds = cases.c2(12)
    e1 = eng.make_engine(m, p, deldops=[ds])
    e1.evaluate(eng.FORM_BATCHED_FP32)
    a = e1.raster_tuning(eng.FORM_BATCHED_FP32)
    e2 = eng.make_engine(m, p, deldops=[ds])
    e2.evaluate(eng.FORM_BATCHED_FP32)
    b = e2.raster_tuning(eng.FORM_BATCHED_FP32)
    assert a == b
    # the same datasets through both engines: the same chi-square to the
    # FP32 images' scatter-order rounding
    assert e1.evaluate(eng.FORM_BATCHED_FP32)["chi2"] == pytest.approx(
        e2.evaluate(eng.FORM_BATCHED_FP32)["chi2"], rel=1e-6)
    e1.close()
    e2.close()


_TUNE_SNIPPET = r"""
import json, os, sys
sys.path.insert(0, os.environ["REPO"]); sys.path.insert(0, os.path.join(os.environ["REPO"], "tests"))
sys.path.insert(0, os.path.join(os.environ["REPO"], "shape-cuda-v1.2_b200", "python"))
import cases
from shape_b200 import engine as eng
m, p, ds = cases.c2(12)
e = eng.make_engine(m, p, deldops=[ds])
e.evaluate(eng.FORM_BATCHED_FP32)
print(json.dumps(e.raster_tuning(eng.FORM_BATCHED_FP32)))
e.close()
"""


def test_tuning_file_carries_choices(cuda_device, tmp_path):
    """SHAPE_B200_TUNING_CACHE: the first process times the candidates and
    writes its choice for the size class; a second process reads the file
    and takes the same choice and times without timing again."""
    import json
    import os
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    path = tmp_path / "tuning.jsonl"
    env = dict(os.environ, REPO=repo, SHAPE_B200_TUNING_CACHE=str(path))
    runs = []
    for _ in range(2):
        out = subprocess.run([sys.executable, "-c", _TUNE_SNIPPET], env=env, capture_output=True, text=True,
                             timeout=600)
        assert out.returncode == 0, out.stderr[-2000:]
        runs.append(json.loads(out.stdout.strip().splitlines()[-1]))
    lines = path.read_text().splitlines()
    assert len(lines) == 1, lines
    rec = json.loads(lines[0])
    assert rec["form"] == eng.FORM_BATCHED_FP32 and rec["views"] == ds_views(), rec
    a, b = runs
    assert a["tuned"] and b["tuned"]
    assert (a["variant"], a["persistent"]) == (b["variant"], b["persistent"]) == (rec["variant"], rec["persistent"])
    np.testing.assert_allclose(b["ms"], rec["ms"], rtol=1e-5)


def ds_views():
    return cases.c2(12)[2].nframes
