"""shape_chi2_frames_noalloc: chi-square sums without any device allocation.

That entry point serves callers that cannot call cudaMalloc (their device
memory belongs to another allocator, or they run where an allocation could
stall the device). They pass images they already hold on the device; the
entry point keeps its partial sums in a fixed device array instead of
allocating scratch. This test runs last (file name) so that a stop at the
first failure has already run every other test.

It checks the per-frame o2, m2, om, calibration and chi-square of two
consecutive calls against the engine's own evaluation of the same frames
(shape_engine_evaluate + shape_engine_get_deldop_results), to the relative
1e-12 that FP64 chi-square sums of the same images meet.
"""
import ctypes as C

import numpy as np
import pytest

import cases
from shape_b200 import ctypes_defs as cd
from shape_b200 import engine as eng

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def test_noalloc_chi2_matches_engine_twice(cuda_device):
    import torch
    m, p, ds = cases.c2(12)
    e = eng.make_engine(m, p, deldops=[ds])
    e.evaluate(eng.FORM_BATCHED_FP64)
    ref = e.results()
    fits = np.concatenate([e.fit(f) for f in range(ds.nframes)])
    e.close()

    dev = torch.device("cuda", cuda_device)
    d_obs = torch.from_numpy(ds.obs).to(dev)
    d_oov = torch.from_numpy(ds.oneovervar).to(dev)
    d_fit = torch.from_numpy(fits).to(dev)
    torch.cuda.synchronize()
    offs = np.ascontiguousarray(ds.offsets, dtype=np.int64)
    weight = np.array([fr.weight for fr in ds.frames])
    calf = np.array([fr.cal_floating for fr in ds.frames], dtype=np.int32)
    cal = np.array([fr.cal for fr in ds.frames])
    L = eng.load_library()
    for call in range(2):
        out = np.full(5 * ds.nframes, np.nan)
        rc = L.shape_chi2_frames_noalloc(cuda_device, ds.nframes,
                                         offs.ctypes.data_as(C.POINTER(C.c_longlong)),
                                         C.c_void_p(d_obs.data_ptr()), C.c_void_p(d_oov.data_ptr()),
                                         C.c_void_p(d_fit.data_ptr()), cd.as_dptr(weight), cd.as_iptr(calf),
                                         cd.as_dptr(cal), cd.as_dptr(out))
        assert rc == 0, L.shape_last_error().decode()
        got = out.reshape(ds.nframes, 5)
        for f, r in enumerate(ref):
            for k, key in enumerate(("o2", "m2", "om", "cal", "chi2")):
                assert abs(got[f, k] - r[key]) <= RTOL * abs(r[key]), (call, f, key, got[f, k], r[key])


def test_noalloc_rejects_oversize(cuda_device):
    """More frames than the fixed scratch array holds: a clear error, no work."""
    import torch
    L = eng.load_library()
    n = 4097
    buf = torch.zeros(n, dtype=torch.float64, device=torch.device("cuda", cuda_device))
    offs = np.arange(n + 1, dtype=np.int64)
    w = np.ones(n); cf = np.zeros(n, dtype=np.int32); cal = np.ones(n); out = np.zeros(5 * n)
    ptr = C.c_void_p(buf.data_ptr())
    rc = L.shape_chi2_frames_noalloc(cuda_device, n, offs.ctypes.data_as(C.POINTER(C.c_longlong)),
                                     ptr, ptr, ptr, cd.as_dptr(w), cd.as_iptr(cf), cd.as_dptr(cal),
                                     cd.as_dptr(out))
    assert rc == -1 and b"exceed the maximum" in L.shape_last_error()
