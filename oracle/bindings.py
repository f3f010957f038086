"""Python bindings for the CPU checkers. TEST INFRASTRUCTURE ONLY.

- ``Oracle``: the plain-C restatement (oracle/shape_oracle.c -> liboracle.so).
- ``Reference``: the reference's own CPU code compiled in place
  (oracle/build_ref.sh -> oracle/_ref/libshape_ref.so), driven through the
  direct-call harness oracle/ref_harness.c.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm import this module.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "shape-cuda-v1.2_b200", "python"))

from shape_b200 import ctypes_defs as cd  # noqa: E402

ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libshape_ref.so")


class OrcReal(C.Structure):
    _fields_ = [("nv", C.c_int), ("nf", C.c_int), ("x", cd.dptr), ("vn", cd.dptr),
                ("fn", cd.dptr), ("area", cd.dptr), ("fv", cd.iptr)]


class OrcPos(C.Structure):
    _fields_ = [("n", C.c_int), ("kmpp", C.c_double),
                ("ae", C.c_double * 9), ("oe", C.c_double * 9), ("se", C.c_double * 9),
                ("bistatic", C.c_int),
                ("b", cd.dptr), ("cose", cd.dptr), ("cosi", cd.dptr), ("z", cd.dptr),
                ("f", cd.iptr), ("cosill", cd.dptr), ("zill", cd.dptr), ("fill", cd.iptr),
                ("xlim", C.c_int * 2), ("ylim", C.c_int * 2),
                ("xlim2", C.c_int * 2), ("ylim2", C.c_int * 2),
                ("posbnd_logfactor", C.c_double)]


def _load(path, builder):
    if not os.path.exists(path):
        raise RuntimeError("%s missing: run %s" % (path, builder))
    return C.CDLL(path)


class Oracle:
    """CPU restatement of the reference hot path (bit-exact FP64 order)."""

    def __init__(self):
        L = self.lib = _load(ORACLE_SO, "oracle/build_oracle.sh")
        P = C.POINTER
        L.orc_realize_vertex.argtypes = [P(cd.ModelDesc), cd.dptr, cd.dptr, cd.dptr, cd.dptr]
        L.orc_pos_alloc.argtypes = [P(OrcPos), C.c_int, C.c_int]
        L.orc_pos_free.argtypes = [P(OrcPos)]
        L.orc_deldop_frame.argtypes = [P(cd.EvalParams), P(OrcReal), P(cd.DeldopSet),
                                       P(cd.DeldopFrame), cd.dptr, cd.dptr, P(OrcPos),
                                       cd.dptr, C.c_char_p, P(cd.DeldopResult)]
        L.orc_deldop_frame_views.argtypes = [P(cd.EvalParams), P(OrcReal), P(cd.DeldopSet), C.c_int,
                                             P(cd.DeldopFrame), cd.dptr, cd.dptr, P(OrcPos),
                                             cd.dptr, C.c_char_p, P(cd.DeldopResult), P(C.c_int),
                                             P(C.c_double)]
        L.orc_doppler_frame.argtypes = [P(cd.EvalParams), P(OrcReal), P(cd.DopplerSet),
                                        P(cd.DopplerFrame), cd.dptr, cd.dptr, P(OrcPos),
                                        cd.dptr, C.c_char_p, P(cd.DeldopResult)]
        L.orc_lghtcrv_point.restype = C.c_double
        L.orc_lghtcrv_point.argtypes = [P(cd.EvalParams), P(OrcReal), P(cd.OpticalLaw),
                                        P(cd.LghtcrvPoint), P(OrcPos), C.c_char_p,
                                        P(C.c_int), P(C.c_double)]
        L.orc_spline_natural.argtypes = [cd.dptr, cd.dptr, C.c_int, cd.dptr]
        L.orc_splint.restype = C.c_double
        L.orc_splint.argtypes = [cd.dptr, cd.dptr, cd.dptr, C.c_int, C.c_double]
        L.orc_radlaw.restype = C.c_double
        L.orc_radlaw.argtypes = [P(cd.RadarLaw), C.c_double]
        L.orc_chi2_frame.argtypes = [cd.dptr, cd.dptr, cd.dptr, C.c_int, C.c_double, C.c_int, C.c_double,
                                     P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double),
                                     P(C.c_double)]

    def realize(self, model):
        d = model.desc()
        x = np.zeros((model.nv, 3)); vn = np.zeros((model.nv, 3))
        fn = np.zeros((model.nf, 3)); area = np.zeros(model.nf)
        self.lib.orc_realize_vertex(C.byref(d), cd.as_dptr(x), cd.as_dptr(vn),
                                    cd.as_dptr(fn), cd.as_dptr(area))
        return {"x": x, "vn": vn, "fn": fn, "area": area, "fv": model.fv}

    def _real(self, real):
        r = OrcReal()
        r.nv, r.nf = real["x"].shape[0], real["fn"].shape[0]
        r.x, r.vn, r.fn = cd.as_dptr(real["x"]), cd.as_dptr(real["vn"]), cd.as_dptr(real["fn"])
        r.area, r.fv = cd.as_dptr(real["area"]), cd.as_iptr(real["fv"])
        return r

    @staticmethod
    def pos_arrays(pos):
        side = 2 * pos.n + 1
        np_ = side * side
        get = lambda p, ct: np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(np_,)).copy()
        return {"z": get(pos.z, C.c_double), "cose": get(pos.cose, C.c_double),
                "cosi": get(pos.cosi, C.c_double), "f": get(pos.f, C.c_int),
                "zill": get(pos.zill, C.c_double), "fill": get(pos.fill, C.c_int),
                "xlim": tuple(pos.xlim), "ylim": tuple(pos.ylim),
                "xlim2": tuple(pos.xlim2), "ylim2": tuple(pos.ylim2)}

    def eval_deldop(self, model, ds, params, real=None, keep_pos=False):
        """calc_deldop + chi2_deldop over every frame of `ds`. Returns
        per-frame fits, results, seen flags and (optionally) POS maps."""
        real = real or self.realize(model)
        R = self._real(real)
        seen = C.create_string_buffer(model.nf)
        fits, results, poss = [], [], []
        for f, fr in enumerate(ds.frames):
            pos = OrcPos()
            self.lib.orc_pos_alloc(C.byref(pos), fr.pos_n, 0)
            fit = np.zeros(fr.ndel * fr.ndop)
            res = cd.DeldopResult()
            obs = np.ascontiguousarray(ds.frame_obs(f))
            oov = np.ascontiguousarray(ds.oneovervar[ds.offsets[f]:ds.offsets[f + 1]])
            if getattr(ds, "views", None):
                va = (cd.DeldopFrame * ds.nviews)(*ds.views[f])
                bany, bterm = C.c_int(0), C.c_double(0.0)
                self.lib.orc_deldop_frame_views(C.byref(params), C.byref(R), C.byref(ds.set), ds.nviews, va,
                                                cd.as_dptr(obs), cd.as_dptr(oov), C.byref(pos),
                                                cd.as_dptr(fit), seen, C.byref(res), C.byref(bany),
                                                C.byref(bterm))
                rd = cd.result_to_dict(res)
                rd["badradar_any"], rd["badradar_term"] = bany.value, bterm.value
            else:
                self.lib.orc_deldop_frame(C.byref(params), C.byref(R), C.byref(ds.set), C.byref(fr),
                                          cd.as_dptr(obs), cd.as_dptr(oov), C.byref(pos),
                                          cd.as_dptr(fit), seen, C.byref(res))
                rd = cd.result_to_dict(res)
            fits.append(fit)
            results.append(rd)
            if keep_pos:
                poss.append(self.pos_arrays(pos))
            self.lib.orc_pos_free(C.byref(pos))
        return {"fits": fits, "results": results, "pos": poss,
                "seen": np.frombuffer(seen.raw, dtype=np.uint8).copy(), "real": real}

    def eval_doppler(self, model, ds, params, real=None, keep_pos=False):
        """calc_doppler + chi2_doppler over every frame of the Doppler set `ds`."""
        real = real or self.realize(model)
        R = self._real(real)
        seen = C.create_string_buffer(model.nf)
        fits, results, poss = [], [], []
        for f, fr in enumerate(ds.frames):
            pos = OrcPos()
            self.lib.orc_pos_alloc(C.byref(pos), fr.pos_n, 0)
            fit = np.zeros(fr.ndop)
            res = cd.DeldopResult()
            obs = np.ascontiguousarray(ds.frame_obs(f))
            oov = np.ascontiguousarray(ds.oneovervar[ds.offsets[f]:ds.offsets[f + 1]])
            self.lib.orc_doppler_frame(C.byref(params), C.byref(R), C.byref(ds.set), C.byref(fr),
                                       cd.as_dptr(obs), cd.as_dptr(oov), C.byref(pos),
                                       cd.as_dptr(fit), seen, C.byref(res))
            fits.append(fit)
            results.append(cd.result_to_dict(res))
            if keep_pos:
                poss.append(self.pos_arrays(pos))
            self.lib.orc_pos_free(C.byref(pos))
        return {"fits": fits, "results": results, "pos": poss,
                "seen": np.frombuffer(seen.raw, dtype=np.uint8).copy(), "real": real}

    def eval_lghtcrv(self, model, ds, params, real=None, keep_pos=False):
        """calc_lghtcrv + chi2_lghtcrv for one lightcurve dataset."""
        real = real or self.realize(model)
        R = self._real(real)
        seen = C.create_string_buffer(model.nf)
        ys, poss, flags = [], [], []
        for p in ds.points:
            pos = OrcPos()
            self.lib.orc_pos_alloc(C.byref(pos), p.pos_n, 1)
            ob, lg = C.c_int(0), C.c_double(0.0)
            y = self.lib.orc_lghtcrv_point(C.byref(params), C.byref(R), C.byref(ds.set.law),
                                           C.byref(p), C.byref(pos), seen, C.byref(ob), C.byref(lg))
            ys.append(y)
            flags.append((ob.value, lg.value))
            if keep_pos:
                poss.append(self.pos_arrays(pos))
            self.lib.orc_pos_free(C.byref(pos))
        y = np.array(ys)
        fit = self.spline_fit(ds.x, y, ds.t)
        o2 = float(np.sum(ds.obs * ds.obs * ds.oneovervar))
        m2 = float(np.sum(fit * fit * ds.oneovervar))
        om = float(np.sum(fit * ds.obs * ds.oneovervar))
        cal = (om / m2 if om > 0 else 1e-40) if ds.set.cal_floating else ds.set.cal
        chi2 = ds.set.weight * (o2 - 2 * cal * om + cal * cal * m2)
        return {"y": y, "fit": fit, "cal": cal, "chi2": chi2, "pos": poss, "flags": flags,
                "seen": np.frombuffer(seen.raw, dtype=np.uint8).copy()}

    def spline_fit(self, x, y, t):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        y2 = np.zeros_like(y)
        self.lib.orc_spline_natural(cd.as_dptr(x), cd.as_dptr(y), len(x), cd.as_dptr(y2))
        return np.array([self.lib.orc_splint(cd.as_dptr(x), cd.as_dptr(y), cd.as_dptr(y2), len(x), float(tt))
                         for tt in t])


OBJFN = C.CFUNCTYPE(C.c_double, C.c_double)


class Reference:
    """The reference's own CPU code (oracle/_ref/libshape_ref.so)."""

    def __init__(self):
        L = self.lib = _load(REF_SO, "oracle/build_ref.sh")
        P = C.POINTER
        L.ref_spline_eval.argtypes = [cd.dptr, cd.dptr, C.c_int, cd.dptr, C.c_int, cd.dptr]
        L.ref_obs_lghtcrv.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), cd.dptr, cd.dptr, cd.dptr, cd.dptr,
                                      cd.dptr, cd.dptr]
        L.ref_obs_lghtcrv_ephem.argtypes = [C.c_void_p, C.c_int, C.c_int, cd.dptr]
        L.ref_new.restype = C.c_void_p
        L.ref_new.argtypes = [P(cd.ModelDesc), P(cd.EvalParams), C.c_int]
        L.ref_set_radar_law.argtypes = [C.c_void_p, P(cd.RadarLaw)]
        L.ref_set_optical_law.argtypes = [C.c_void_p, P(cd.OpticalLaw)]
        L.ref_add_deldop_set.argtypes = [C.c_void_p, P(cd.DeldopSet), C.c_int,
                                         P(cd.DeldopFrame), cd.dptr, cd.dptr]
        L.ref_add_deldop_set_views.argtypes = [C.c_void_p, P(cd.DeldopSet), C.c_int, C.c_int, C.c_int,
                                               P(cd.DeldopFrame), cd.dptr, cd.dptr]
        L.ref_add_lghtcrv_set.argtypes = [C.c_void_p, P(cd.LghtcrvSet), P(cd.LghtcrvPoint)]
        L.ref_add_doppler_set.argtypes = [C.c_void_p, P(cd.DopplerSet), C.c_int,
                                          P(cd.DopplerFrame), cd.dptr, cd.dptr]
        L.ref_get_doppler_frame.argtypes = [C.c_void_p, C.c_int, C.c_int, cd.dptr, cd.dptr,
                                            cd.dptr, cd.iptr, P(cd.DeldopResult)]
        L.ref_set_scale.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.ref_realize_spin_frames.argtypes = [P(cd.SpinState), cd.dptr, cd.dptr, C.c_int, cd.dptr, cd.dptr,
                                              cd.dptr, cd.dptr, C.c_double]
        L.ref_set_r.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.ref_vary_params.argtypes = [C.c_void_p, P(C.c_int), P(C.c_int), P(C.c_int), cd.dptr]
        L.ref_vary_params.restype = None
        L.ref_realize.argtypes = [C.c_void_p]
        L.ref_evaluate.restype = C.c_double
        L.ref_evaluate.argtypes = [C.c_void_p]
        L.ref_calc_chi2.restype = C.c_double
        L.ref_calc_chi2.argtypes = [C.c_void_p]
        L.ref_evaluate_mt.restype = C.c_double
        L.ref_evaluate_mt.argtypes = [P(C.c_void_p), C.c_int]
        L.ref_get_realized.argtypes = [C.c_void_p, cd.dptr, cd.dptr, cd.dptr, cd.dptr]
        L.ref_get_active.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_add_poset_set.argtypes = [C.c_void_p, C.POINTER(cd.PosetSet), C.c_int, C.POINTER(cd.PosetFrame),
                                        cd.dptr, cd.dptr]
        L.ref_get_poset_frame.argtypes = [C.c_void_p, C.c_int, C.c_int, cd.dptr, cd.dptr, cd.dptr]
        L.ref_get_badposet.argtypes = [C.c_void_p, cd.dptr]
        L.ref_get_flags.argtypes = [C.c_void_p, cd.dptr]
        L.ref_penalties.argtypes = [C.c_void_p, C.c_int, cd.iptr, cd.dptr, P(cd.SpinState), cd.dptr, cd.dptr,
                                    cd.dptr]
        L.ref_penalties.restype = C.c_double
        L.ref_mod_read.argtypes = [C.c_char_p]
        L.ref_mod_read.restype = C.c_void_p
        L.ref_mod_shape.argtypes = [C.c_void_p, P(C.c_int), P(C.c_int), cd.dptr, cd.dptr, cd.dptr, cd.dptr,
                                    cd.iptr, cd.iptr, cd.iptr]
        L.ref_mod_comp.argtypes = [C.c_void_p, C.c_int, P(C.c_int), P(C.c_int), cd.dptr, cd.dptr, cd.dptr]
        L.ref_mod_comp.restype = C.c_int
        L.ref_mod_radar.argtypes = [C.c_void_p, C.c_int, P(cd.RadarLaw)]
        L.ref_mod_optical.argtypes = [C.c_void_p, C.c_int, P(cd.OpticalLaw)]
        L.ref_mod_spin.argtypes = [C.c_void_p, P(cd.SpinState)]
        L.ref_ephem2mat.argtypes = [cd.dptr, C.c_int, cd.dptr, C.c_int, C.c_double, cd.dptr, cd.dptr, cd.dptr,
                                    cd.dptr]
        L.ref_ephem2mat.restype = C.c_double
        L.ref_deldopoffs.argtypes = [cd.dptr, C.c_int, C.c_double, C.c_int, cd.dptr, C.c_double, C.c_double,
                                     C.c_double, cd.dptr, cd.dptr]
        L.ref_deldopoffs.restype = None
        L.ref_obs_read.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_int]
        L.ref_obs_read.restype = C.c_void_p
        L.ref_obs_frame.argtypes = [C.c_void_p, C.c_int, C.c_int, cd.dptr, P(C.c_int), cd.dptr, cd.dptr]
        L.ref_obs_frame.restype = None
        L.ref_obs_frame_view.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, cd.dptr, P(C.c_int), cd.dptr,
                                         cd.dptr]
        L.ref_obs_frame_view.restype = None
        L.ref_obs_views.argtypes = [C.c_void_p, C.c_int, P(C.c_int)]
        L.ref_obs_views.restype = None
        L.ref_obs_doppler_frame.argtypes = [C.c_void_p, C.c_int, C.c_int, cd.dptr, P(C.c_int), cd.dptr, cd.dptr]
        L.ref_obs_doppler_frame.restype = None
        L.ref_read_radar_data.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, P(C.c_int), P(C.c_int), C.c_int,
                                          C.c_double, cd.dptr]
        L.ref_get_seen.argtypes = [C.c_void_p, C.c_char_p]
        L.ref_get_deldop_frame.argtypes = [C.c_void_p, C.c_int, C.c_int, cd.dptr, cd.dptr,
                                           cd.dptr, cd.iptr, P(cd.DeldopResult)]
        L.ref_get_lghtcrv.argtypes = [C.c_void_p, C.c_int, cd.dptr, cd.dptr, cd.dptr]
        L.ref_get_lghtcrv_pos.argtypes = [C.c_void_p, C.c_int, C.c_int, cd.dptr, cd.dptr,
                                          cd.dptr, cd.iptr, cd.dptr, cd.iptr, cd.iptr]
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_mnbrak.argtypes = [cd.dptr, cd.dptr, cd.dptr, cd.dptr, cd.dptr, cd.dptr, OBJFN]
        L.ref_brent_abs.restype = C.c_double
        L.ref_brent_abs.argtypes = [C.c_double, C.c_double, C.c_double, OBJFN,
                                    C.c_double, C.c_double, cd.dptr]

    def session(self, model, params, deldops=(), lghtcrvs=(), radar_law=None, optical_law=None,
                dopplers=(), posets=()):
        """A reference session with the sets in the order deldops, dopplers,
        lightcurves, plane-of-sky sets (all radar sets share one radar law,
        all optical sets one optical law)."""
        d = model.desc()
        h = self.lib.ref_new(C.byref(d), C.byref(params),
                             len(deldops) + len(dopplers) + len(lghtcrvs) + len(posets))
        keep = [d]
        if deldops or dopplers:
            first = deldops[0] if deldops else dopplers[0]
            self.lib.ref_set_radar_law(h, C.byref(radar_law or first.set.law))
        if lghtcrvs or posets:
            law = optical_law or (lghtcrvs[0].set.law if lghtcrvs else posets[0].law)
            self.lib.ref_set_optical_law(h, C.byref(law))
        for ds in deldops:
            if getattr(ds, "views", None):
                arr = ds.view_array()
                keep.append(arr)
                self.lib.ref_add_deldop_set_views(h, C.byref(ds.set), ds.nframes, ds.nviews, ds.v0, arr,
                                                  cd.as_dptr(ds.obs), cd.as_dptr(ds.oneovervar))
                continue
            arr = ds.frame_array()
            keep.append(arr)
            self.lib.ref_add_deldop_set(h, C.byref(ds.set), ds.nframes, arr,
                                        cd.as_dptr(ds.obs), cd.as_dptr(ds.oneovervar))
        for ds in dopplers:
            arr = ds.frame_array()
            keep.append(arr)
            self.lib.ref_add_doppler_set(h, C.byref(ds.set), ds.nframes, arr,
                                         cd.as_dptr(ds.obs), cd.as_dptr(ds.oneovervar))
        for ls in lghtcrvs:
            arr = ls.point_array()
            keep.append(arr)
            self.lib.ref_add_lghtcrv_set(h, C.byref(ls.bind()), arr)
        for ds in posets:
            st, frames, obs, oov = ds.bind()
            keep.extend([st, frames, obs, oov])
            self.lib.ref_add_poset_set(h, C.byref(st), ds.nframes, frames, cd.as_dptr(obs), cd.as_dptr(oov))
        return RefSession(self, h, model, keep)

    def read_mod(self, path):
        """The reference's read_mod on a model file: (arrays, radar laws,
        optical laws, spin state), arrays as shape_model_desc holds them."""
        h = self.lib.ref_mod_read(os.fsencode(path))
        nv, nf = C.c_int(), C.c_int()
        self.lib.ref_mod_shape(h, C.byref(nv), C.byref(nf), None, None, None, None, None, None, None)
        nv, nf = nv.value, nf.value
        a, u, r, sc = np.zeros(3 * nv), np.zeros(3 * nv), np.zeros(nv), np.zeros(3)
        fv, ap, ai = np.zeros(3 * nf, np.int32), np.zeros(nv + 1, np.int32), np.zeros(3 * nf, np.int32)
        i32 = lambda x: x.ctypes.data_as(cd.iptr)
        self.lib.ref_mod_shape(h, C.byref(C.c_int()), C.byref(C.c_int()), cd.as_dptr(a), cd.as_dptr(u),
                               cd.as_dptr(r), cd.as_dptr(sc), i32(fv), i32(ap), i32(ai))
        radar, optical = [], []
        n = self.lib.ref_mod_radar(h, -1, C.byref(cd.RadarLaw()))
        for i in range(n):
            law = cd.RadarLaw()
            self.lib.ref_mod_radar(h, i, C.byref(law))
            radar.append(law)
        n = self.lib.ref_mod_optical(h, -1, C.byref(cd.OpticalLaw()))
        for i in range(n):
            olaw = cd.OpticalLaw()
            self.lib.ref_mod_optical(h, i, C.byref(olaw))
            optical.append(olaw)
        spin = cd.SpinState()
        self.lib.ref_mod_spin(h, C.byref(spin))
        comps = []
        ncomp = self.lib.ref_mod_comp(h, -1, C.byref(C.c_int()), C.byref(C.c_int()), None, None, None)
        for c in range(ncomp):
            cnv, cnf = C.c_int(), C.c_int()
            csc, coff, crot = np.zeros(3), np.zeros(3), np.zeros(3)
            self.lib.ref_mod_comp(h, c, C.byref(cnv), C.byref(cnf), cd.as_dptr(csc), cd.as_dptr(coff),
                                  cd.as_dptr(crot))
            comps.append({"nv": cnv.value, "nf": cnf.value, "scale": csc, "off": coff, "rot": crot})
        arrays = {"a": a.reshape(nv, 3), "u": u.reshape(nv, 3), "r": r, "scale": sc, "fv": fv.reshape(nf, 3),
                  "af_ptr": ap, "af_idx": ai, "comps": comps}
        return arrays, radar, optical, spin

    def read_radar_data(self, path, kind, ndel, ndop, idel_use, idop_use, swap, sdev):
        """The reference's reader of one data file (kind 0-2 delay-Doppler
        ascii / binary / rdf, 3-5 Doppler): the window's obs values."""
        obs = np.zeros((idel_use[1] - idel_use[0] + 1) * (idop_use[1] - idop_use[0] + 1))
        rc = self.lib.ref_read_radar_data(os.fsencode(path), kind, ndel, ndop, (C.c_int * 2)(*idel_use),
                                          (C.c_int * 2)(*idop_use), swap, sdev, cd.as_dptr(obs))
        assert rc == 0
        return obs

    def spline_eval(self, x, y, t):
        """The reference's spline() + splint() at epochs t (natural ends)."""
        x, y, t = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, t))
        out = np.zeros(len(t))
        self.lib.ref_spline_eval(cd.as_dptr(x), cd.as_dptr(y), len(x), cd.as_dptr(t), len(t), cd.as_dptr(out))
        return out

    def mnbrak(self, fn, ax, bx):
        cb = OBJFN(fn)
        a, b, c = C.c_double(ax), C.c_double(bx), C.c_double(0)
        fa, fb, fc = C.c_double(0), C.c_double(0), C.c_double(0)
        self.lib.ref_mnbrak(C.byref(a), C.byref(b), C.byref(c), C.byref(fa), C.byref(fb),
                            C.byref(fc), cb)
        return a.value, b.value, c.value, fa.value, fb.value, fc.value

    def brent_abs(self, fn, ax, bx, cx, tol, abstol):
        cb = OBJFN(fn)
        xmin = C.c_double(0)
        fmin = self.lib.ref_brent_abs(ax, bx, cx, cb, tol, abstol, C.byref(xmin))
        return fmin, xmin.value


class RefSession:
    def __init__(self, ref, h, model, keep):
        self.ref, self.h, self.model, self.keep = ref, h, model, keep
        self.L = ref.lib

    def evaluate(self):
        return self.L.ref_evaluate(self.h)

    def penalties(self, pens, spin=None, angleoff=None, omegaoff=None):
        """The reference's penalties() for [(type, weight), ...]: (sum, bases)."""
        n = len(pens)
        types = np.array([t for t, _ in pens] or [0], dtype=np.int32)
        w = np.array([x for _, x in pens] or [0.0])
        base = np.zeros(max(1, n))
        ao = None if angleoff is None else np.ascontiguousarray(angleoff, dtype=np.float64).ravel()
        oo = None if omegaoff is None else np.ascontiguousarray(omegaoff, dtype=np.float64).ravel()
        tot = self.L.ref_penalties(self.h, n, types.ctypes.data_as(cd.iptr), cd.as_dptr(w),
                                   C.byref(spin) if spin is not None else None,
                                   cd.as_dptr(ao) if ao is not None else None,
                                   cd.as_dptr(oo) if oo is not None else None, cd.as_dptr(base))
        return tot, base[:n].copy()

    def poset_frame(self, s, f, frame):
        """(fit [ncol, nrow], sky brightness [2n+1, 2n+1], cal, chi2) of a
        plane-of-sky frame after evaluate(); frame: its description dict."""
        fit = np.zeros((frame["ncol"], frame["nrow"]))
        side = 2 * frame["pos_n"] + 1
        b = np.zeros((side, side))
        out = np.zeros(2)
        self.L.ref_get_poset_frame(self.h, s, f, cd.as_dptr(fit), cd.as_dptr(b), cd.as_dptr(out))
        return fit, b, out[0], out[1]

    def badposet(self):
        out = np.zeros(2)
        self.L.ref_get_badposet(self.h, cd.as_dptr(out))
        return int(out[0]), out[1]

    def active(self):
        """check_surface's (vertex, facet) act flags after the last realize_mod."""
        m = self.model
        v = np.zeros(m.nv, dtype=np.uint8)
        f = np.zeros(m.nf, dtype=np.uint8)
        self.L.ref_get_active(self.h, v.ctypes.data_as(C.c_void_p), f.ctypes.data_as(C.c_void_p))
        return v, f

    def realized(self):
        m = self.model
        x = np.zeros((m.nv, 3)); vn = np.zeros((m.nv, 3))
        fn = np.zeros((m.nf, 3)); area = np.zeros(m.nf)
        self.L.ref_get_realized(self.h, cd.as_dptr(x), cd.as_dptr(vn), cd.as_dptr(fn), cd.as_dptr(area))
        return {"x": x, "vn": vn, "fn": fn, "area": area}

    def flags(self):
        out = np.zeros(4)
        self.L.ref_get_flags(self.h, cd.as_dptr(out))
        return {"posbnd": int(out[0]), "posbnd_logfactor": out[1],
                "badradar": int(out[2]), "badradar_logfactor": out[3]}

    def seen(self):
        buf = C.create_string_buffer(self.model.nf)
        self.L.ref_get_seen(self.h, buf)
        return np.frombuffer(buf.raw, dtype=np.uint8).copy()

    def vary_params(self, flags, delcor0_free, dopscale_free):
        """The reference's vary_params after evaluate(): the four means."""
        fl = (C.c_int * 4)(*[int(x) for x in flags])
        a = (C.c_int * len(delcor0_free))(*[int(x) for x in delcor0_free])
        b = (C.c_int * len(dopscale_free))(*[int(x) for x in dopscale_free])
        out = np.zeros(4)
        self.L.ref_vary_params(self.h, fl, a, b, cd.as_dptr(out))
        return out

    def deldop_frame(self, s, f, fr):
        side = 2 * fr.pos_n + 1
        fit = np.zeros(fr.ndel * fr.ndop)
        z = np.zeros(side * side); cose = np.zeros(side * side)
        fac = np.zeros(side * side, dtype=np.int32)
        res = cd.DeldopResult()
        self.L.ref_get_deldop_frame(self.h, s, f, cd.as_dptr(fit), cd.as_dptr(z), cd.as_dptr(cose),
                                    cd.as_iptr(fac), C.byref(res))
        return {"fit": fit, "z": z, "cose": cose, "f": fac, "res": cd.result_to_dict(res)}

    def doppler_frame(self, s, f, fr):
        side = 2 * fr.pos_n + 1
        fit = np.zeros(fr.ndop)
        z = np.zeros(side * side); cose = np.zeros(side * side)
        fac = np.zeros(side * side, dtype=np.int32)
        res = cd.DeldopResult()
        self.L.ref_get_doppler_frame(self.h, s, f, cd.as_dptr(fit), cd.as_dptr(z), cd.as_dptr(cose),
                                     cd.as_iptr(fac), C.byref(res))
        return {"fit": fit, "z": z, "cose": cose, "f": fac, "res": cd.result_to_dict(res)}

    def lghtcrv(self, s, ds):
        y = np.zeros(ds.set.ncalc); fit = np.zeros(ds.set.n); out = np.zeros(2)
        self.L.ref_get_lghtcrv(self.h, s, cd.as_dptr(y), cd.as_dptr(fit), cd.as_dptr(out))
        return {"y": y, "fit": fit, "cal": out[0], "chi2": out[1]}

    def lghtcrv_pos(self, s, i, pt):
        side = 2 * pt.pos_n + 1
        np_ = side * side
        z, cose, cosi, zill = (np.zeros(np_) for _ in range(4))
        fac = np.zeros(np_, dtype=np.int32); fill = np.zeros(np_, dtype=np.int32)
        lims = np.zeros(8, dtype=np.int32)
        self.L.ref_get_lghtcrv_pos(self.h, s, i + 1, cd.as_dptr(z), cd.as_dptr(cose), cd.as_dptr(cosi),
                                   cd.as_iptr(fac), cd.as_dptr(zill), cd.as_iptr(fill), cd.as_iptr(lims))
        return {"z": z, "cose": cose, "cosi": cosi, "f": fac, "zill": zill, "fill": fill,
                "lims": lims}

    def close(self):
        if self.h:
            self.L.ref_free(self.h)
            self.h = None

    def __del__(self):
        self.close()
