"""Inputs of the golden fixtures (tests/golden/): models, datasets and
evaluation switches, rebuilt deterministically by shape_b200.synth, shared
by tests/golden/make_golden.py and the CPU tests."""
import math

import numpy as np

from shape_b200 import ctypes_defs as cd
from shape_b200 import synth


def octa3_model():
    """512-facet model (octahedron subdivided 3 times), radii with 3% noise."""
    return synth.noisy_octa_model(levels=3, sigma=0.03, seed=42)


def law(kind, R=0.08, C=1.3, qR=0.05, qC=4.0, cut_deg=60.0):
    L = cd.RadarLaw()
    L.type, L.diff_R, L.diff_C = kind, R, C
    L.qs_R, L.qs_C, L.qs_cos_cutoff = qR, qC, math.cos(cut_deg * math.pi / 180)
    return L


def _small(codemethod=1, spb=1, stride=1, law_=None, seed=11, pos=(41, 61)):
    return lambda s, p: synth.batched_dataset(3, pos, (32, 48), (32, 64), s, p, seed=seed,
                                              codemethod=codemethod, spb=spb, stride=stride, law=law_)


P_DEFAULT = synth.eval_params()

DELDOP_CASES = {
    "c1": (synth.ellipsoid_model, lambda s, p: synth.config1_dataset(s, p), P_DEFAULT),
    "c1_outbnd": (synth.ellipsoid_model, lambda s, p: synth.config1_dataset(s, p, pos_n=40), P_DEFAULT),
    "c1_nosmooth": (synth.ellipsoid_model, lambda s, p: synth.config1_dataset(s, p),
                    synth.eval_params(pos_smooth=0)),
    "small_long_orig": (octa3_model, _small(), P_DEFAULT),
    "small_short": (octa3_model, _small(codemethod=0), P_DEFAULT),
    "small_long_mod_spb2_nsinc2": (octa3_model, _small(codemethod=2, spb=2), synth.eval_params(nsinc2=2)),
    "small_long_mod_spb3_nsinc3": (octa3_model, _small(codemethod=2, spb=3), synth.eval_params(nsinc2=3)),
    "small_long_orig_spb2": (octa3_model, _small(spb=2, stride=1), P_DEFAULT),
    "law_gaussian": (octa3_model, _small(law_=law(2)), P_DEFAULT),
    "law_hagfors": (octa3_model, _small(law_=law(3)), P_DEFAULT),
    "law_cosine_qs": (octa3_model, _small(law_=law(4)), P_DEFAULT),
    "law_gaussian_cosine": (octa3_model, _small(law_=law(5)), P_DEFAULT),
    "law_hagfors_cosine": (octa3_model, _small(law_=law(6)), P_DEFAULT),
    "law_cosine_cosine": (octa3_model, _small(law_=law(7)), P_DEFAULT),
}

def _dop(span=0.7, law_=None, seed=21, pos=(41, 61), ndop=(32, 64), nframes=3):
    return lambda s, p: synth.doppler_dataset(nframes, pos, ndop, s, p, seed=seed, span=span, law=law_)


# Doppler-only sets: in-frame spectra, spectra whose model spills into the
# overflow spectrum, a model wider than the overflow spectrum (badradar),
# nsinc2 = 2 and a hybrid radar law.
DOPPLER_CASES = {
    "dop_small": (octa3_model, _dop(), P_DEFAULT),
    "dop_overflow": (octa3_model, _dop(span=1.6), P_DEFAULT),
    "dop_overflow_far": (octa3_model, _dop(span=130.0, ndop=(24, 32), nframes=2), P_DEFAULT),
    "dop_nsinc2": (octa3_model, _dop(seed=23), synth.eval_params(nsinc2=2)),
    "dop_law_hagfors_cosine": (octa3_model, _dop(law_=law(6), seed=25), P_DEFAULT),
}

LGHTCRV_CASES = {
    "kaasalainen": (octa3_model, lambda s, p: synth.lightcurve_dataset(6, (41, 61), s, p, seed=5),
                    synth.eval_params(mask_tol=0.0)),
    "lambert": (octa3_model, lambda s, p: synth.lightcurve_dataset(5, (41, 61), s, p, seed=6, law_type=2),
                synth.eval_params(mask_tol=0.0)),
    "lommel": (octa3_model, lambda s, p: synth.lightcurve_dataset(5, (41, 61), s, p, seed=8, law_type=3),
               synth.eval_params(mask_tol=0.002)),
    "c3_short": (synth.harmonic_model, lambda s, p: synth.lightcurve_dataset(4, (129, 141), s, p, seed=7),
                 synth.eval_params(mask_tol=0.0)),
    # observation epochs strictly between the calculated ones: the fit is
    # the natural spline off its knots (NR spline / splint in the reference)
    "kaasalainen_off_knots": (octa3_model,
                              lambda s, p: synth.lightcurve_dataset(9, (41, 61), s, p, seed=13, obs_between=True),
                              synth.eval_params(mask_tol=0.0)),
}


# config-1 fit: the three scale factors from a 10% perturbation
FIT_START = (1.10, 0.90, 1.10)
FIT_PARAMS = [(1, j, 0.02, 1e-4, 1e-6) for j in range(3)]   # kind SCALE, index, step, tol, abstol
FIT_TERM_PREC = 1e-4
FIT_MAXITER = 3


def objective_from(chi2, dof, flags, bad_objfactor=2.0):
    """objective() of src/shape/bestfit.c:789-866 with no penalties."""
    err = chi2 / dof
    if flags["posbnd"]:
        err *= bad_objfactor * math.exp(flags["posbnd_logfactor"])
    if flags["badradar"]:
        err *= bad_objfactor * math.exp(flags["badradar_logfactor"])
    return err


def _quad(x):
    return 3.0 * (x - 1.37) ** 2 + 0.5


def _quart(x):
    return (x - 0.3) ** 4 + 0.1 * (x - 0.3) ** 2 + 2.0


def _cosine(x):
    return -math.cos(2.0 * x) + 0.05 * x


def _asym(x):
    return math.exp(x - 2.0) - x


LINESEARCH_CASES = [
    # name, f, ax, bx, fractional tol, absolute tol
    ("quadratic", _quad, 1.0, 1.1, 1e-6, 1e-9),
    ("quartic", _quart, 2.0, 2.2, 1e-4, 1e-6),
    ("cosine", _cosine, 0.5, 0.6, 1e-8, 0.0),
    ("asymmetric", _asym, 0.0, 0.05, 1e-5, 1e-7),
    ("scale_like", lambda x: 1e4 * (x - 0.95) ** 2 + 1e4 * 0.001 * (x - 0.95) ** 3 + 10070.0, 1.0, 1.02, 1e-5, 1e-7),
]
