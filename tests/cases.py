"""Seeded test cases shared by the CPU and GPU tests. Observed images are
synthesized from the true model with the CPU oracle (tests may use it)."""
import functools
import math

import numpy as np

from oracle.bindings import Oracle
from shape_b200 import ctypes_defs as cd
from shape_b200 import synth

_orc = None


def orc():
    global _orc
    if _orc is None:
        _orc = Oracle()
    return _orc


def dd_synth(model):
    return lambda ds, p: orc().eval_deldop(model, ds, p)["fits"]


def lc_synth(model):
    return lambda ds, p: orc().eval_lghtcrv(model, ds, p)["y"]


@functools.lru_cache(None)
def c1():
    m = synth.ellipsoid_model()
    p = synth.eval_params()
    return m, p, synth.config1_dataset(dd_synth(m), p)


@functools.lru_cache(None)
def c2_model():
    return synth.harmonic_model()


@functools.lru_cache(None)
def c2(nframes=64):
    m = c2_model()
    p = synth.eval_params()
    ds = synth.batched_dataset(nframes, (101, 301), (64, 256), (64, 512), dd_synth(m), p, seed=7)
    return m, p, ds


@functools.lru_cache(None)
def c3(npoints=24, nsets=2):
    m = c2_model()
    p = synth.eval_params(mask_tol=0.0)
    sets = [synth.lightcurve_dataset(npoints, (129, 257), lc_synth(m), p, set_index=k) for k in range(nsets)]
    return m, p, sets


def small_frames(model, params, nframes, pos_range, codemethod=1, spb=1, stride=1, seed=11,
                 law=None, ndel=(48, 96), ndop=(48, 128)):
    ds = synth.batched_dataset(nframes, pos_range, ndel, ndop, dd_synth(model), params, seed=seed,
                               codemethod=codemethod, spb=spb, stride=stride)
    if law is not None:
        ds.set.law = law
        # re-synthesize observations with the new law
        fits = orc().eval_deldop(model, ds, params)["fits"]
        rng = np.random.default_rng(99)
        for f in range(ds.nframes):
            ft = fits[f]
            peak = ft.max() if ft.max() > 0 else 1.0
            ds.obs[ds.offsets[f]:ds.offsets[f + 1]] = 20 * ft / peak + rng.standard_normal(ft.size)
    return ds


def radar_law(kind):
    L = cd.RadarLaw()
    L.type = kind
    L.diff_R, L.diff_C = 0.08, 1.3
    L.qs_R, L.qs_C, L.qs_cos_cutoff = 0.05, 4.0, math.cos(60 * math.pi / 180)
    return L


def scaled_model(m, sc):
    """A copy of model m with scale factors sc (the oracle reads them from the model)."""
    mm = m.copy()
    mm.scale = np.array([float(x) for x in sc])
    return mm
