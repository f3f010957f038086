"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own CPU
code (oracle/_ref/libshape_ref.so, built by oracle/build_ref.sh from the
reference sources). Run in a checkout where the reference tree is present:

    bash oracle/build_ref.sh && python tests/golden/make_golden.py

Every input is rebuilt deterministically by shape_b200.synth; the fixtures
store the reference's outputs (and the observed images it synthesized), so
the CPU tests can pin the oracle restatement without the reference tree.
Large maps are stored as SHA-256 digests of their exact bytes.
"""
import ctypes as C
import hashlib
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "shape-cuda-v1.2_b200", "python"))
sys.path.insert(0, os.path.join(REPO, "tests"))

import numpy as np  # noqa: E402

from oracle.bindings import Reference  # noqa: E402
from shape_b200 import synth  # noqa: E402
import golden_cases as gc  # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def quiet(fn):
    """Run fn with stdout redirected (chi2_lghtcrv prints every point)."""
    sys.stdout.flush()
    saved = os.dup(1)
    dn = os.open(os.devnull, os.O_WRONLY)
    os.dup2(dn, 1)
    try:
        return fn()
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(dn)
        os.close(saved)


def ref_deldop_synth(ref, model):
    def f(ds, p):
        S = ref.session(model, p, deldops=[ds])
        S.evaluate()
        out = [S.deldop_frame(0, k, fr)["fit"] for k, fr in enumerate(ds.frames)]
        S.close()
        return out
    return f


def ref_doppler_synth(ref, model):
    def f(ds, p):
        S = ref.session(model, p, dopplers=[ds])
        S.evaluate()
        out = [S.doppler_frame(0, k, fr)["fit"] for k, fr in enumerate(ds.frames)]
        S.close()
        return out
    return f


def ref_lc_synth(ref, model):
    def f(ds, p):
        S = ref.session(model, p, lghtcrvs=[ds])
        quiet(S.evaluate)
        y = S.lghtcrv(0, ds)["y"]
        S.close()
        return y
    return f


def deldop_record(S, s, ds):
    frames = []
    for k, fr in enumerate(ds.frames):
        r = S.deldop_frame(s, k, fr)
        frames.append({
            "f": digest(r["f"].astype(np.int32)), "z": digest(r["z"]), "cose": digest(r["cose"]),
            "fit": digest(r["fit"]), "fit_sum": float(r["fit"].sum()),
            "covered": int((r["f"] >= 0).sum()),
            "res": {k2: (list(v) if isinstance(v, tuple) else v) for k2, v in r["res"].items()
                    if k2 in ("xlim", "ylim", "idellim", "idoplim", "dellim", "doplim",
                              "posbnd_logfactor", "badradar_logfactor", "cal", "chi2")},
        })
    return frames


def doppler_record(S, s, ds):
    frames = []
    for k, fr in enumerate(ds.frames):
        r = S.doppler_frame(s, k, fr)
        frames.append({
            "f": digest(r["f"].astype(np.int32)), "fit": digest(r["fit"]), "fit_sum": float(r["fit"].sum()),
            "covered": int((r["f"] >= 0).sum()),
            "overflow_o2": r["res"]["o2"], "overflow_m2": r["res"]["m2"],
            "res": {k2: (list(v) if isinstance(v, tuple) else v) for k2, v in r["res"].items()
                    if k2 in ("xlim", "ylim", "idoplim", "doplim", "posbnd_logfactor",
                              "badradar_logfactor", "cal", "chi2")},
        })
    return frames


def main():
    ref = Reference()
    out = {"deldop": {}, "lghtcrv": {}, "realize": {}, "doppler": {}}
    arrays = {}

    # realization digests (bit-exact targets)
    for name, mk in (("c1", synth.ellipsoid_model), ("c2", synth.harmonic_model), ("octa3", gc.octa3_model)):
        m = mk()
        S = ref.session(m, synth.eval_params(), deldops=[], lghtcrvs=[])
        ref.lib.ref_realize(S.h)
        r = S.realized()
        out["realize"][name] = {k: digest(v) for k, v in r.items()}
        S.close()

    # delay-Doppler cases
    for name, (model_fn, ds_fn, params) in gc.DELDOP_CASES.items():
        m = model_fn()
        ds = ds_fn(ref_deldop_synth(ref, m), params)
        S = ref.session(m, params, deldops=[ds])
        chi2 = S.evaluate()
        out["deldop"][name] = {"chi2": chi2, "frames": deldop_record(S, 0, ds), "flags": S.flags(),
                               "seen": digest(S.seen())}
        out["deldop"][name]["obs"] = digest(ds.obs)
        if name == "c1":
            r = S.deldop_frame(0, 0, ds.frames[0])
            cov = r["f"] >= 0
            arrays["c1_f"] = r["f"].astype(np.int16)
            arrays["c1_z"] = r["z"][cov]
            arrays["c1_cose"] = r["cose"][cov]
            arrays["c1_fit"] = r["fit"]
        S.close()

    # Doppler cases
    for name, (model_fn, ds_fn, params) in gc.DOPPLER_CASES.items():
        m = model_fn()
        ds = ds_fn(ref_doppler_synth(ref, m), params)
        S = ref.session(m, params, dopplers=[ds])
        chi2 = S.evaluate()
        out["doppler"][name] = {"chi2": chi2, "frames": doppler_record(S, 0, ds), "flags": S.flags(),
                                "seen": digest(S.seen()), "obs": digest(ds.obs)}
        S.close()

    # lightcurve cases
    for name, (model_fn, ds_fn, params) in gc.LGHTCRV_CASES.items():
        m = model_fn()
        ds = ds_fn(ref_lc_synth(ref, m), params)
        S = ref.session(m, params, lghtcrvs=[ds])
        chi2 = quiet(S.evaluate)
        r = S.lghtcrv(0, ds)
        pos = []
        for i, pt in enumerate(ds.points):
            pr = S.lghtcrv_pos(0, i, pt)
            pos.append({k: digest(pr[k]) for k in ("z", "cose", "cosi", "f", "zill", "fill")})
        out["lghtcrv"][name] = {"chi2": chi2, "y": r["y"].tolist(), "fit": r["fit"].tolist(),
                                "cal": r["cal"], "pos": pos, "flags": S.flags(), "seen": digest(S.seen())}
        out["lghtcrv"][name]["obs"] = digest(ds.obs)
        S.close()

    # line searches of the reference on analytic objectives
    out["linesearch"] = {}
    for name, fn, ax, bx, tol, abstol in gc.LINESEARCH_CASES:
        trials = []

        def obj(x, fn=fn, trials=trials):
            trials.append(x)
            return fn(x)
        a, b, c, fa, fb, fc = ref.mnbrak(obj, ax, bx)
        n_mn = len(trials)
        fmin, xmin = ref.brent_abs(obj, a, b, c, tol, abstol)
        out["linesearch"][name] = {"bracket": [a, b, c, fa, fb, fc], "n_mnbrak": n_mn,
                                   "trials": list(trials), "xmin": xmin, "fmin": fmin}

    # config-1 fit with the reference's line searches and objective; the
    # outer parameter loop follows src/shape/bestfit.c:367-651
    m = synth.ellipsoid_model()
    params = synth.eval_params()
    ds = synth.config1_dataset(ref_deldop_synth(ref, m), params)
    S = ref.session(m, params, deldops=[ds])
    dof = sum(fr.dof for fr in ds.frames)
    values = list(gc.FIT_START)
    trace, state = [], {"flag": 0}

    def objective():
        for j in range(3):
            ref.lib.ref_set_scale(S.h, j, values[j])
        chi2 = S.evaluate()
        fl = S.flags()
        state["flag"] |= fl["posbnd"] | fl["badradar"]
        return gc.objective_from(chi2, dof, fl)
    enderr = objective()
    start = enderr
    it = 0
    while True:
        it += 1
        beginerr = enderr
        for k, (_, j, step, tol, abstol) in enumerate(gc.FIT_PARAMS):
            def f(x, k=k, j=j):
                values[j] = x
                trace.append([k, x])
                return objective()
            state["flag"] = 0
            cur = values[j]
            a, b, c, fa, fb, fc = ref.mnbrak(f, cur, cur + step)
            enderr, xmin = ref.brent_abs(f, a, b, c, tol, abstol)
            values[j] = xmin
            if state["flag"]:
                objective()
        if (beginerr - enderr) / enderr < gc.FIT_TERM_PREC or it >= gc.FIT_MAXITER:
            break
    out["bestfit_c1"] = {"trace": trace, "values": values, "initial": start, "final": enderr,
                         "iterations": it, "obs": digest(ds.obs)}
    S.close()

    with open(os.path.join(HERE, "reference_golden.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "reference_arrays.npz"), **arrays)
    print("wrote", os.path.join(HERE, "reference_golden.json"))


if __name__ == "__main__":
    main()
