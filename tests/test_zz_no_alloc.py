"""shape_chi2_frames_noalloc: chi-square sums without any device allocation.

That entry point serves callers that cannot call cudaMalloc (their device
memory belongs to another allocator, or they run where an allocation could
stall the device). They pass images they already hold on the device; the
entry point keeps its partial sums in a fixed device array instead of
allocating scratch. This test runs last (file name) so that a stop at the
first failure has already run every other test.

Every check is against the CPU oracle's chi2_deldop restatement
(orc_chi2_frame, the reference's row-major sums) on the same images:
o2, m2 and om to relative 1e-12 (the device sums are compensated, the
oracle's sequential), calibration and chi-square to 1e-10 (chi-square is a
difference of those sums). The images are the oracle's own fit images of
config-2 frames, two calls in a row, then small frames that exercise an
empty frame between non-empty ones, offsets that start above 0 and the
element limit.
"""
import ctypes as C

import numpy as np
import pytest

import cases
from shape_b200 import ctypes_defs as cd
from shape_b200 import engine as eng

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-12
CHI2_RTOL = 1e-10


def _oracle_frames(obs, oov, fit, offs, weight, calf, cal):
    """Per-frame (o2, m2, om, cal, chi2) of the oracle's chi2_deldop."""
    lib = cases.orc().lib
    out = []
    for f in range(len(offs) - 1):
        a, b = int(offs[f]), int(offs[f + 1])
        v = [C.c_double() for _ in range(5)]
        o, w, ft = (np.ascontiguousarray(x[a:b]) for x in (obs, oov, fit))
        lib.orc_chi2_frame(cd.as_dptr(o), cd.as_dptr(w), cd.as_dptr(ft), b - a, float(weight[f]),
                           int(calf[f]), float(cal[f]), *[C.byref(x) for x in v])
        out.append([x.value for x in v])
    return np.array(out)


def _call(dev, obs, oov, fit, offs, weight, calf, cal):
    import torch
    L = eng.load_library()
    d = [torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(dev) for x in (obs, oov, fit)]
    torch.cuda.synchronize()
    n = len(offs) - 1
    offs = np.ascontiguousarray(offs, dtype=np.int64)
    out = np.full(5 * n, np.nan)
    rc = L.shape_chi2_frames_noalloc(dev.index, n, offs.ctypes.data_as(C.POINTER(C.c_longlong)),
                                     C.c_void_p(d[0].data_ptr()), C.c_void_p(d[1].data_ptr()),
                                     C.c_void_p(d[2].data_ptr()),
                                     cd.as_dptr(np.ascontiguousarray(weight, dtype=np.float64)),
                                     cd.as_iptr(np.ascontiguousarray(calf, dtype=np.int32)),
                                     cd.as_dptr(np.ascontiguousarray(cal, dtype=np.float64)), cd.as_dptr(out))
    assert rc == 0, L.shape_last_error().decode()
    return out.reshape(n, 5)


def _check(got, want, tag):
    for f in range(len(want)):
        for k, key in enumerate(("o2", "m2", "om", "cal", "chi2")):
            tol = (SUM_RTOL if k < 3 else CHI2_RTOL) * abs(want[f, k])
            assert abs(got[f, k] - want[f, k]) <= tol, (tag, f, key, got[f, k], want[f, k])


def test_noalloc_chi2_matches_oracle_twice(cuda_device):
    import torch
    m, p, ds = cases.c2(12)
    o = cases.orc().eval_deldop(m, ds, p)
    fits = np.concatenate(o["fits"])
    weight = np.array([fr.weight for fr in ds.frames])
    calf = np.array([fr.cal_floating for fr in ds.frames], dtype=np.int32)
    cal = np.array([fr.cal for fr in ds.frames])
    want = _oracle_frames(ds.obs, ds.oneovervar, fits, ds.offsets, weight, calf, cal)
    # the oracle's frame chi-square (orc_deldop_frame) is the same number
    for f, r in enumerate(o["results"]):
        assert abs(want[f, 4] - r["chi2"]) <= CHI2_RTOL * abs(r["chi2"])
    dev = torch.device("cuda", cuda_device)
    for call in range(2):
        _check(_call(dev, ds.obs, ds.oneovervar, fits, ds.offsets, weight, calf, cal), want, "call %d" % call)


def test_noalloc_empty_frame_and_offset_start(cuda_device):
    """Frames of 3000, 0, 5000 and 2048 elements whose offsets start at 100
    (the first 100 elements of the arrays belong to no frame), fixed and
    floating calibration."""
    import torch
    rng = np.random.default_rng(5)
    sizes = [3000, 0, 5000, 2048]
    offs = np.concatenate([[100], 100 + np.cumsum(sizes)])
    n = int(offs[-1])
    fit = np.abs(rng.standard_normal(n))
    fit[rng.random(n) < 0.3] = 0.0
    obs = 3.0 * fit + rng.standard_normal(n)
    oov = rng.uniform(0.5, 2.0, n)
    weight = np.array([1.0, 2.0, 0.5, 1.5])
    calf = np.array([1, 1, 0, 1], dtype=np.int32)
    cal = np.array([1.0, 1.0, 2.5, 1.0])
    want = _oracle_frames(obs, oov, fit, offs, weight, calf, cal)
    got = _call(torch.device("cuda", cuda_device), obs, oov, fit, offs, weight, calf, cal)
    _check(got, want, "ragged")
    assert got[1, 4] == 0.0 and got[1, 0] == 0.0


def _rejected(cuda_device, nframes, offs):
    import torch
    L = eng.load_library()
    buf = torch.zeros(16, dtype=torch.float64, device=torch.device("cuda", cuda_device))
    offs = np.ascontiguousarray(offs, dtype=np.int64)
    w = np.ones(nframes); cf = np.zeros(nframes, dtype=np.int32); cal = np.ones(nframes)
    out = np.zeros(5 * nframes)
    ptr = C.c_void_p(buf.data_ptr())
    rc = L.shape_chi2_frames_noalloc(cuda_device, nframes, offs.ctypes.data_as(C.POINTER(C.c_longlong)),
                                     ptr, ptr, ptr, cd.as_dptr(w), cd.as_iptr(cf), cd.as_dptr(cal),
                                     cd.as_dptr(out))
    return rc, L.shape_last_error()


def test_noalloc_rejects_oversize(cuda_device):
    """More frames, or more elements, than the fixed scratch array holds: a
    clear error before any work (the arrays are never read)."""
    n = 4097
    rc, msg = _rejected(cuda_device, n, np.arange(n + 1))
    assert rc == -1 and b"exceed the maximum" in msg
    rc, msg = _rejected(cuda_device, 1, [0, 65536 * 2048 + 1])
    assert rc == -1 and b"elements exceed the maximum" in msg
