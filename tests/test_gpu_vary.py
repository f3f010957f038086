"""vary_params (shape_engine_vary_params) against the reference's own
vary_params (src/shape/vary_params.c) on the same session, after an
evaluation of the same model: the subradar distance mean (delay-Doppler
frames with a floating 0th delay-correction coefficient), the radar
cross-section mean (frames with a fixed calibration), the optical
brightness mean (a lightcurve with a fixed calibration) and the
cos(subradar latitude) mean (sets with a floating Doppler scale), each
normalised by read_dat's weight sums over every dataset; only the first
dataset contributes, as in the reference.

Bars: distances (from bit-exact depth maps) and cosines exact; the cross
section (a sum over a fit image the engine scatters in parallel) to 1e-10
relative; the brightness to 1e-12."""
import copy

import numpy as np
import pytest

import cases
import golden_cases as gc
from shape_b200 import ctypes_defs as cd
from shape_b200 import engine as eng

pytestmark = pytest.mark.gpu


def _ref():
    from oracle.bindings import Reference
    try:
        return Reference()
    except RuntimeError:
        pytest.skip("reference CPU build (oracle/_ref) not present")


def _with_fixed_cal(ds, frames, kind=cd.DeldopFrame, cal=1.5):
    """A copy of ds (frames copied too) whose listed frames have a fixed
    calibration."""
    out = copy.copy(ds)
    out.frames = [kind.from_buffer_copy(f) for f in ds.frames]
    for f in frames:
        out.frames[f].cal_floating = 0
        out.frames[f].cal = cal
    return out


def _compare(m, p, deldops=(), dopplers=(), lghtcrvs=(), flags=(1, 1, 1, 1), d0=None, ds_=None):
    ref = _ref()
    nsets = len(deldops) + len(dopplers) + len(lghtcrvs)
    d0 = d0 if d0 is not None else [1] * nsets
    ds_ = ds_ if ds_ is not None else [1] * nsets
    s = ref.session(m, p, deldops=list(deldops), dopplers=list(dopplers), lghtcrvs=list(lghtcrvs))
    s.evaluate()
    want = s.vary_params(flags, d0, ds_)
    e = eng.make_engine(m, p, deldops=list(deldops), dopplers=list(dopplers), lghtcrvs=list(lghtcrvs))
    got = e.vary_params(flags, d0, ds_)
    e.close()
    return got, want


def test_vary_deldop_first():
    m, p, ds = cases.c2(6)
    ds = _with_fixed_cal(ds, [0, 2, 3])
    got, want = _compare(m, p, deldops=[ds])
    assert got[0] == want[0]
    assert abs(got[1] - want[1]) <= 1e-10 * abs(want[1])
    assert got[2] == want[2] == 0.0
    assert got[3] == want[3]
    assert want[0] != 0.0 and want[1] != 0.0 and want[3] != 0.0


def test_vary_only_the_first_set_and_its_flags():
    """A second delay-Doppler set adds to the weight sums but not to the
    means (the reference's loop stops after set 0); a fixed 0th delay
    coefficient and a fixed Doppler scale drop those means."""
    m, p, ds = cases.c2(6)
    a = _with_fixed_cal(ds, [1])
    b = _with_fixed_cal(ds, [0, 1, 2])
    got, want = _compare(m, p, deldops=[a, b], d0=[1, 0], ds_=[0, 1])
    for k in (0, 2, 3):
        assert got[k] == want[k], k
    assert abs(got[1] - want[1]) <= 1e-10 * abs(want[1])
    got, want = _compare(m, p, deldops=[a, b], flags=(0, 1, 0, 0))
    assert got[0] == want[0] == 0.0 and got[3] == want[3] == 0.0


def test_vary_doppler_first():
    name = sorted(gc.DOPPLER_CASES)[0]
    model_fn, ds_fn, p = gc.DOPPLER_CASES[name]
    m = model_fn()
    ds = ds_fn(lambda d, pp: cases.orc().eval_doppler(m, d, pp)["fits"], p)
    dop = _with_fixed_cal(ds, [0], kind=cd.DopplerFrame, cal=1.2)
    got, want = _compare(m, p, dopplers=[dop])
    assert got[0] == want[0] == 0.0
    assert abs(got[1] - want[1]) <= 1e-10 * abs(want[1])
    assert got[3] == want[3] and want[3] != 0.0


def test_vary_lightcurve_first():
    m, p, sets = cases.c3(12, 1)
    lc = copy.copy(sets[0])
    lc.set = cd.LghtcrvSet.from_buffer_copy(sets[0].set)
    lc.set.cal_floating = 0
    lc.set.cal = 1.0
    lc.bind()
    got, want = _compare(m, p, lghtcrvs=[lc])
    assert abs(got[2] - want[2]) <= 1e-12 * abs(want[2])
    assert want[2] != 0.0
