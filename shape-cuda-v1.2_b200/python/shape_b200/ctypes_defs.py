"""ctypes mirrors of include/shape_types.h (plain C structs of the C ABI).

The field order and types must match the header exactly; tests check the
struct sizes against the C compiler's (``shape_abi_sizes`` in the library).
"""
import ctypes as C

import numpy as np

dptr = C.POINTER(C.c_double)
iptr = C.POINTER(C.c_int)


class ModelDesc(C.Structure):
    _fields_ = [
        ("nv", C.c_int), ("nf", C.c_int),
        ("a", dptr), ("u", dptr), ("r", dptr),
        ("scale", C.c_double * 3),
        ("fv", iptr), ("af_ptr", iptr), ("af_idx", iptr),
        ("ncomp", C.c_int),
        ("comp_nv", iptr), ("comp_nf", iptr),
        ("comp_scale", dptr), ("comp_rot", dptr), ("comp_off", dptr),
    ]


class RadarLaw(C.Structure):
    _fields_ = [
        ("type", C.c_int),
        ("diff_R", C.c_double), ("diff_C", C.c_double),
        ("qs_R", C.c_double), ("qs_C", C.c_double), ("qs_cos_cutoff", C.c_double),
    ]


class OpticalLaw(C.Structure):
    _fields_ = [
        ("type", C.c_int), ("R", C.c_double), ("wt", C.c_double),
        ("A0", C.c_double), ("D", C.c_double), ("k", C.c_double),
    ]


class EvalParams(C.Structure):
    _fields_ = [
        ("pos_smooth", C.c_int), ("nsinc2", C.c_int), ("sinc2width", C.c_int),
        ("mask_tol", C.c_double), ("mincosine_seen", C.c_double), ("mark_seen", C.c_int),
    ]


class DeldopFrame(C.Structure):
    _fields_ = [
        ("pos_n", C.c_int), ("km_per_pixel", C.c_double),
        ("ae", C.c_double * 9), ("oe", C.c_double * 9), ("spin", C.c_double * 3),
        ("deloff", C.c_double), ("dopoff", C.c_double),
        ("ndel", C.c_int), ("ndop", C.c_int),
        ("delcom_vig", C.c_double), ("dopcom_vig", C.c_double), ("dopDC_vig", C.c_double),
        ("weight", C.c_double), ("dof", C.c_double),
        ("cal_floating", C.c_int), ("cal", C.c_double),
    ]


class DeldopSet(C.Structure):
    _fields_ = [
        ("del_per_pixel", C.c_double), ("dop_per_pixel", C.c_double),
        ("Ftx", C.c_double), ("dopscale", C.c_double),
        ("codemethod", C.c_int), ("spb", C.c_int), ("stride", C.c_int),
        ("dopfftlen", C.c_int),
        ("law", RadarLaw),
    ]


class DopplerFrame(C.Structure):
    _fields_ = [
        ("pos_n", C.c_int), ("km_per_pixel", C.c_double),
        ("ae", C.c_double * 9), ("oe", C.c_double * 9), ("spin", C.c_double * 3),
        ("dopoff", C.c_double), ("ndop", C.c_int), ("dopcom_vig", C.c_double),
        ("weight", C.c_double), ("dof", C.c_double),
        ("cal_floating", C.c_int), ("cal", C.c_double), ("sdev", C.c_double),
    ]


class DopplerSet(C.Structure):
    _fields_ = [
        ("dop_per_bin", C.c_double), ("Ftx", C.c_double), ("dopscale", C.c_double),
        ("law", RadarLaw),
    ]


MAX_IMPULSES = 10


class EphemPoint(C.Structure):
    _fields_ = [("t", C.c_double), ("ra", C.c_double), ("dec", C.c_double), ("dist", C.c_double)]


class SpinState(C.Structure):
    """shape_spin_state (include/shape_types.h)."""
    _fields_ = [
        ("pa", C.c_int), ("t0", C.c_double),
        ("angle", C.c_double * 3), ("omega", C.c_double * 3), ("omegadot", C.c_double * 3),
        ("n_impulse", C.c_int), ("t_impulse", C.c_double * MAX_IMPULSES),
        ("impulse", (C.c_double * 3) * MAX_IMPULSES),
        ("lib_amp", C.c_double), ("lib_freq", C.c_double), ("lib_phase", C.c_double),
        ("inertia", C.c_double * 3),
    ]


class LghtcrvPoint(C.Structure):
    _fields_ = [
        ("pos_n", C.c_int), ("km_per_pixel", C.c_double),
        ("ae", C.c_double * 9), ("oe", C.c_double * 9), ("se", C.c_double * 9),
        ("solar_phase", C.c_double),
    ]


class LghtcrvSet(C.Structure):
    _fields_ = [
        ("ncalc", C.c_int), ("n", C.c_int),
        ("x", dptr), ("t", dptr), ("obs", dptr), ("oneovervar", dptr),
        ("weight", C.c_double), ("dof", C.c_double),
        ("cal_floating", C.c_int), ("cal", C.c_double),
        ("law", OpticalLaw),
    ]


class PosetFrame(C.Structure):
    _fields_ = [
        ("pos_n", C.c_int), ("km_per_pixel", C.c_double),
        ("ae", C.c_double * 9), ("oe", C.c_double * 9), ("se", C.c_double * 9),
        ("solar_phase", C.c_double),
        ("ncol", C.c_int), ("nrow", C.c_int), ("fit_km_per_pixel", C.c_double),
        ("colcom_vig", C.c_double), ("rowcom_vig", C.c_double),
        ("xoff", C.c_double), ("yoff", C.c_double), ("northangle", C.c_double),
        ("weight", C.c_double), ("dof", C.c_double),
    ]


class PosetSet(C.Structure):
    _fields_ = [("law", OpticalLaw), ("resample", C.c_int), ("rebin", C.c_int)]


class PosetResult(C.Structure):
    _fields_ = [
        ("outbnd", C.c_int), ("posbnd_logsum", C.c_double),
        ("badposet", C.c_int), ("badposet_logfactor", C.c_double),
        ("o2", C.c_double), ("m2", C.c_double), ("om", C.c_double),
        ("cal", C.c_double), ("chi2", C.c_double),
    ]


class DeldopResult(C.Structure):
    _fields_ = [
        ("outbnd", C.c_int), ("posbnd_logfactor", C.c_double),
        ("badradar", C.c_int), ("badradar_logfactor", C.c_double),
        ("xlim", C.c_int * 2), ("ylim", C.c_int * 2),
        ("idellim", C.c_int * 2), ("idoplim", C.c_int * 2),
        ("dellim", C.c_double * 2), ("doplim", C.c_double * 2),
        ("o2", C.c_double), ("m2", C.c_double), ("om", C.c_double),
        ("cal", C.c_double), ("chi2", C.c_double),
    ]


STRUCTS = {
    "shape_model_desc": ModelDesc, "shape_radar_law": RadarLaw,
    "shape_optical_law": OpticalLaw, "shape_eval_params": EvalParams,
    "shape_deldop_frame": DeldopFrame, "shape_deldop_set": DeldopSet,
    "shape_lghtcrv_point": LghtcrvPoint, "shape_lghtcrv_set": LghtcrvSet,
    "shape_deldop_result": DeldopResult,
    "shape_doppler_frame": DopplerFrame, "shape_doppler_set": DopplerSet,
}


def as_dptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(dptr)


def as_iptr(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(iptr)


def fill9(arr9, m):
    flat = np.asarray(m, dtype=np.float64).reshape(9)
    for i in range(9):
        arr9[i] = float(flat[i])


def result_to_dict(r):
    return {
        "outbnd": r.outbnd, "posbnd_logfactor": r.posbnd_logfactor,
        "badradar": r.badradar, "badradar_logfactor": r.badradar_logfactor,
        "xlim": tuple(r.xlim), "ylim": tuple(r.ylim),
        "idellim": tuple(r.idellim), "idoplim": tuple(r.idoplim),
        "dellim": tuple(r.dellim), "doplim": tuple(r.doplim),
        "o2": r.o2, "m2": r.m2, "om": r.om, "cal": r.cal, "chi2": r.chi2,
    }
