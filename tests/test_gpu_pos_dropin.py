"""The plane-of-sky drop-ins (shape-cuda-v1.2_b200/dropin/shape_b200_pos.c:
posvis, pos2deldop, posclr, posmask, apply_photo with the reference's
signatures, running on the device through shape_posvis & co.) beside the
reference's own routines, on POS frames and datasets allocated the
reference's way, in one process (oracle/_ref/libshape_dropin.so).

Bars: posvis's images (z, cos(e), cos(i), facet, body, component, and the
sun view's), limits, posbnd_logfactor and return value bit-exact, including
accumulation over further bodies at orbit offsets; posclr and posmask
bit-exact; apply_photo's brightness image and sum bit-exact (the device
computes each pixel as the reference does, the sum runs in its order);
pos2deldop's fit image to 1e-12 of its peak (parallel scatter-add), its
bin limits, delay / Doppler limits and badradar terms exact, with and
without orbit offsets.
"""
import ctypes as C
import os

import numpy as np
import pytest

import cases
import golden_cases as gc
from shape_b200 import ctypes_defs as cd
from shape_b200 import synth

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN_SO = os.path.join(REPO, "oracle", "_ref", "libshape_dropin.so")
IMAGES = ("b", "cose", "cosi", "z", "body", "comp", "f", "cosill", "zill", "bodyill", "compill", "fill")
INT_IMAGES = ("body", "comp", "f", "bodyill", "compill", "fill")


@pytest.fixture(scope="module")
def lib():
    from oracle.bindings import Reference
    ref = Reference()
    if not os.path.exists(DROPIN_SO):
        pytest.fail("oracle/_ref/libshape_dropin.so missing: run oracle/build_dropin.sh")
    L = C.CDLL(DROPIN_SO)
    vp, d3 = C.c_void_p, cd.dptr
    L.dh_pos_new.restype = vp
    L.dh_pos_new.argtypes = [C.c_int, C.c_double, d3, d3, d3, C.c_int]
    L.dh_pos_free.argtypes = [vp]
    L.dh_posclr.argtypes = [vp, C.c_int]
    L.dh_posvis.argtypes = [vp, vp, C.c_int, d3, C.c_int, C.c_int, C.c_int, C.c_int]
    L.dh_posmask.argtypes = [vp, C.c_int, C.c_double]
    L.dh_apply_photo.restype = C.c_double
    L.dh_apply_photo.argtypes = [vp, vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]
    L.dh_pos_get.argtypes = [vp] + [cd.dptr] * 4 + [cd.iptr] * 3 + [cd.dptr] * 2 + [cd.iptr] * 3 + \
        [cd.iptr, cd.dptr]
    L.dh_pos2deldop.argtypes = [vp, C.c_int, C.c_int, C.c_int, d3, C.c_double, C.c_double, C.c_double, C.c_int]
    return ref, L


def _pos_get(L, p, n):
    P = (2 * n + 1) ** 2
    out = {k: (np.zeros(P, dtype=np.int32) if k in INT_IMAGES else np.zeros(P)) for k in IMAGES}
    lims = np.zeros(8, dtype=np.int32)
    lf = C.c_double()
    L.dh_pos_get(p, *[cd.as_iptr(out[k]) if k in INT_IMAGES else cd.as_dptr(out[k]) for k in IMAGES],
                 cd.as_iptr(lims), C.byref(lf))
    out["lims"] = lims
    out["logfactor"] = lf.value
    return out


def _same_pos(a, b, tag):
    for k in IMAGES:
        assert np.array_equal(a[k], b[k]), (tag, k, int(np.sum(a[k] != b[k])))
    assert np.array_equal(a["lims"], b["lims"]), (tag, a["lims"], b["lims"])
    assert a["logfactor"] == b["logfactor"], (tag, a["logfactor"], b["logfactor"])


def _pair(L, n, kmpp, ae, oe, se, bistatic):
    mk = lambda: L.dh_pos_new(n, kmpp, cd.as_dptr(np.ascontiguousarray(ae, dtype=np.float64)),
                              cd.as_dptr(np.ascontiguousarray(oe, dtype=np.float64)),
                              cd.as_dptr(np.ascontiguousarray(se, dtype=np.float64)), bistatic)
    return mk(), mk()


def _view(n=75, kmpp=2.25 / 150.0, phase=0.7, alpha=0.0):
    pole = synth.ecl_dir(30.0, 60.0)
    to_earth = synth.ecl_dir(0.0, 10.0)
    ae = synth.body_matrix(pole, phase)
    oe = synth.observer_matrix(to_earth)
    axis = np.cross(to_earth, [0.0, 0.0, 1.0])
    se = synth.observer_matrix(synth.rotate_about(to_earth, axis, alpha))
    return n, kmpp, ae, oe, se


@pytest.mark.parametrize("case", ["c1_smooth", "c1_flat", "c1_outbnd", "octa3_bistatic", "three_bodies"])
def test_posvis_matches_reference(cuda_device, lib, case):
    ref, L = lib
    m = gc.octa3_model() if case == "octa3_bistatic" else synth.ellipsoid_model()
    S = ref.session(m, synth.eval_params())
    ref.lib.ref_realize(S.h)
    n, kmpp, ae, oe, se = _view(n=40 if case == "c1_outbnd" else 75, alpha=0.6 if case == "octa3_bistatic" else 0.0)
    if case == "octa3_bistatic":
        kmpp = 2.6 / 150.0
    bistatic = 1 if case == "octa3_bistatic" else 0
    a, b = _pair(L, n, kmpp, ae, oe, se, bistatic)
    L.dh_posclr(a, 0)
    L.dh_posclr(b, 1)
    _same_pos(_pos_get(L, a, n), _pos_get(L, b, n), "posclr")
    smooth = 0 if case == "c1_flat" else 1
    zero = np.zeros(3)
    calls = [(zero, 0, 0, 0)]
    if bistatic:
        calls.append((zero, 1, 0, 0))                            # the sun view
    if case == "three_bodies":
        calls.append((np.array([0.31, -0.22, 0.47]), 0, 1, 0))  # a second body in front, partly
        calls.append((np.array([-0.9, 0.75, -0.6]), 0, 2, 1))   # and one behind, partly outside
    for off, src, body, comp in calls:
        ra = L.dh_posvis(S.h, a, 0, cd.as_dptr(off), smooth, src, body, comp)
        rb = L.dh_posvis(S.h, b, 1, cd.as_dptr(off), smooth, src, body, comp)
        assert ra == rb, (case, src, body, ra, rb)
        _same_pos(_pos_get(L, a, n), _pos_get(L, b, n), (case, src, body))
    pa = _pos_get(L, a, n)
    assert (pa["f"] >= 0).sum() > 100
    if case == "c1_outbnd":
        assert ra == 1 and pa["logfactor"] > 0
    if case == "three_bodies":
        assert set(np.unique(pa["body"])) >= {0, 1, 2}
    L.dh_pos_free(a)
    L.dh_pos_free(b)
    S.close()


@pytest.mark.parametrize("case,offsets", [("c1", False), ("small_long_orig", False), ("small_short", False),
                                          ("small_long_mod_spb3_nsinc3", False), ("c1", True)])
def test_pos2deldop_matches_reference(cuda_device, lib, case, offsets):
    ref, L = lib
    mk, build, p = gc.DELDOP_CASES[case]
    m = mk()
    ds = build(cases.dd_synth(m), p)
    S = ref.session(m, p, deldops=[ds])
    for f, fr in enumerate(ds.frames):
        if offsets:
            off2, xo, yo, do, bodies = np.array([0.3, -0.2, 0.4]), 3.5, -2.25, 1.75, (0, 1)
        else:
            off2, xo, yo, do, bodies = None, 0.0, 0.0, 0.0, (0,)
        for body in bodies:
            po = cd.as_dptr(off2) if off2 is not None else None
            ba = L.dh_pos2deldop(S.h, 0, f, 0, po, xo, yo, do, body)
            ra = S.deldop_frame(0, f, fr)
            bb = L.dh_pos2deldop(S.h, 0, f, 1, po, xo, yo, do, body)
            rb = S.deldop_frame(0, f, fr)
            assert ba == bb
            scale = max(np.abs(ra["fit"]).max(), 1e-300)
            assert np.abs(ra["fit"] - rb["fit"]).max() <= 1e-12 * scale, (case, f, body)
            assert ra["fit"].max() > 0
            for k in ("idellim", "idoplim", "dellim", "doplim", "badradar_logfactor"):
                assert ra["res"][k] == rb["res"][k], (case, f, body, k, ra["res"][k], rb["res"][k])
    S.close()


@pytest.mark.parametrize("law_type,tol", [(11, 0.0), (2, 0.0), (3, 0.002)])
def test_posmask_apply_photo_match_reference(cuda_device, lib, law_type, tol):
    """A lightcurve point's two views filled by the reference's posvis, then
    the reference's or the drop-in's posmask and apply_photo."""
    ref, L = lib
    m = gc.octa3_model()
    p = synth.eval_params(mask_tol=tol)
    ls = synth.lightcurve_dataset(3, (81, 101), None, p, seed=5, law_type=law_type)
    S = ref.session(m, p, lghtcrvs=[ls])
    ref.lib.ref_realize(S.h)
    for pt in ls.points:
        n = pt.pos_n
        ae = np.array(pt.ae).reshape(3, 3)
        oe = np.array(pt.oe).reshape(3, 3)
        se = np.array(pt.se).reshape(3, 3)
        a, b = _pair(L, n, pt.km_per_pixel, ae, oe, se, 1)
        zero = np.zeros(3)
        for q in (a, b):
            L.dh_posclr(q, 0)
            L.dh_posvis(S.h, q, 0, cd.as_dptr(zero), 1, 0, 0, 0)
            L.dh_posvis(S.h, q, 0, cd.as_dptr(zero), 1, 1, 0, 0)
        L.dh_posmask(a, 0, tol)
        L.dh_posmask(b, 1, tol)
        _same_pos(_pos_get(L, a, n), _pos_get(L, b, n), "posmask")
        intensity = (pt.km_per_pixel / 1.4959787061e8) ** 2
        sa = L.dh_apply_photo(S.h, a, 0, 0, pt.solar_phase, intensity, 0)
        sb = L.dh_apply_photo(S.h, b, 1, 0, pt.solar_phase, intensity, 0)
        assert sa == sb and sa > 1e-40, (sa, sb)
        _same_pos(_pos_get(L, a, n), _pos_get(L, b, n), "apply_photo")
        L.dh_pos_free(a)
        L.dh_pos_free(b)
    S.close()
