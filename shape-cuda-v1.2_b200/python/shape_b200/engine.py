"""ctypes binding of libshape_b200.so (C ABI: include/shape_b200.h).

The library is built in-tree by shape-cuda-v1.2_b200/build.py. Loading fails
loudly when it is missing: there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

from . import ctypes_defs as cd

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(os.path.dirname(HERE))
LIB_PATH = os.path.join(PKG, "lib", "libshape_b200.so")

FORM_PLAIN_FP64 = 0
FORM_BATCHED_FP64 = 1
FORM_BATCHED_FP32 = 2
FORMS = {"plain_fp64": 0, "batched_fp64": 1, "batched_fp32": 2}


PAR_SCALE = 1
PAR_VERTEX_R = 2
PAR_SPIN_ANGLE = 3
PAR_SPIN_OMEGA = 4
PAR_SPIN_INERTIA = 5
PAR_SPIN_OMEGADOT = 6
PAR_SPIN_IMPULSE = 7
PAR_SPIN_LIB = 8
PAR_ANGLEOFF = 9
PAR_OMEGAOFF = 10

# penalty types (the reference's numbering)
PEN_NONSMOOTH, PEN_CONCAVITY, PEN_RDEV, PEN_VOLUME, PEN_COMDEV = 9, 10, 11, 12, 13
PEN_INERTIADEV, PEN_INERTIADEV_UNI, PEN_PA3TILT, PEN_NONPA, PEN_NONPA_UNI = 14, 15, 16, 17, 18
PEN_EULEROFFS, PEN_FLATTENING, PEN_MAXRDEV, PEN_IMPULSE = 19, 20, 21, 25


class FitParam(C.Structure):
    _fields_ = [("kind", C.c_int), ("index", C.c_int), ("step", C.c_double), ("tol", C.c_double),
                ("abstol", C.c_double)]


class FitOptions(C.Structure):
    _fields_ = [("form", C.c_int), ("term_prec", C.c_double), ("term_maxiter", C.c_int)]


class FitResult(C.Structure):
    _fields_ = [("initial_objective", C.c_double), ("final_objective", C.c_double),
                ("iterations", C.c_int), ("evaluations", C.c_int), ("trace_len", C.c_int)]


class Request(C.Structure):
    _fields_ = [("workload", C.c_int), ("arrival_s", C.c_double), ("scale", C.c_double * 3)]


class RequestResult(C.Structure):
    _fields_ = [("chi2", C.c_double), ("objective", C.c_double), ("t_start", C.c_double),
                ("t_done", C.c_double), ("latency_s", C.c_double), ("device_ms", C.c_double),
                ("instance", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("span_s", C.c_double), ("requests_per_s", C.c_double), ("frame_evals_per_s", C.c_double),
                ("p50_latency_s", C.c_double), ("p99_latency_s", C.c_double),
                ("mean_concurrency", C.c_double), ("peak_concurrency", C.c_int),
                ("instances_created", C.c_int), ("instances_evicted", C.c_int),
                ("peak_hbm_bytes", C.c_double)]


class EvalSummary(C.Structure):
    _fields_ = [("chi2", C.c_double), ("dof", C.c_double), ("chi2_deldop", C.c_double),
                ("chi2_lghtcrv", C.c_double), ("posbnd", C.c_int), ("posbnd_logfactor", C.c_double),
                ("badradar", C.c_int), ("badradar_logfactor", C.c_double), ("objective", C.c_double),
                ("penalties", C.c_double), ("chi2_poset", C.c_double), ("badposet", C.c_int),
                ("badposet_logfactor", C.c_double)]


ABI_ORDER = ["shape_model_desc", "shape_radar_law", "shape_optical_law", "shape_eval_params",
             "shape_deldop_frame", "shape_deldop_set", "shape_lghtcrv_point", "shape_lghtcrv_set",
             "shape_deldop_result"]

_lib = None


def load_library(path=LIB_PATH):
    """Load the engine library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libshape_b200.so not found at %s: run shape-cuda-v1.2_b200/build.py" % path)
    L = C.CDLL(path)
    P = C.POINTER
    vp = C.c_void_p
    L.shape_last_error.restype = C.c_char_p
    L.shape_version.restype = C.c_char_p
    L.shape_abi_sizes.argtypes = [P(C.c_size_t), C.c_int]
    L.shape_engine_create.argtypes = [C.c_int, P(vp)]
    L.shape_engine_destroy.argtypes = [vp]
    L.shape_engine_set_model.argtypes = [vp, P(cd.ModelDesc)]
    L.shape_engine_set_params.argtypes = [vp, P(cd.EvalParams)]
    L.shape_engine_add_deldop_set.argtypes = [vp, P(cd.DeldopSet), C.c_int, P(cd.DeldopFrame),
                                              cd.dptr, cd.dptr]
    L.shape_engine_add_deldop_set_views.argtypes = [vp, P(cd.DeldopSet), C.c_int, C.c_int, P(cd.DeldopFrame),
                                                    cd.dptr, cd.dptr]
    L.shape_engine_add_lghtcrv_set.argtypes = [vp, P(cd.LghtcrvSet), P(cd.LghtcrvPoint)]
    L.shape_engine_add_doppler_set.argtypes = [vp, P(cd.DopplerSet), C.c_int, P(cd.DopplerFrame),
                                               cd.dptr, cd.dptr]
    L.shape_engine_get_radar_overflow.argtypes = [vp, cd.dptr, C.c_int]
    L.shape_engine_finalize.argtypes = [vp]
    L.shape_engine_get_active.argtypes = [vp, vp, vp]
    L.shape_obs_poset_info.argtypes = [vp, C.c_int, P(C.c_int), P(C.c_int)]
    L.shape_obs_poset_file.argtypes = [vp, C.c_int, C.c_int, C.c_char_p, C.c_int, P(C.c_int)]
    L.shape_obs_poset.argtypes = [vp, C.c_int, P(cd.SpinState), P(ObsOptions), P(cd.PosetFrame)]
    L.shape_engine_add_poset_set.argtypes = [vp, P(cd.PosetSet), C.c_int, P(cd.PosetFrame), cd.dptr, cd.dptr]
    L.shape_engine_get_poset.argtypes = [vp, C.c_int, C.c_int, cd.dptr, cd.dptr, P(cd.PosetResult)]
    L.shape_engine_set_scale.argtypes = [vp, C.c_int, C.c_double]
    L.shape_engine_set_vertex_r.argtypes = [vp, C.c_int, C.c_double]
    L.shape_engine_get_vertex_r.argtypes = [vp, C.c_int, P(C.c_double)]
    L.shape_engine_evaluate.argtypes = [vp, C.c_int, P(EvalSummary)]
    L.shape_engine_get_deldop_results.argtypes = [vp, P(cd.DeldopResult), C.c_int]
    L.shape_engine_get_fit.argtypes = [vp, C.c_int, cd.dptr]
    L.shape_engine_keep_pos.argtypes = [vp, C.c_int]
    L.shape_engine_get_pos.argtypes = [vp, C.c_int, cd.dptr, cd.dptr, cd.iptr]
    L.shape_engine_get_lghtcrv_pos.argtypes = [vp, C.c_int, C.c_int, cd.dptr, cd.dptr, cd.dptr,
                                               cd.iptr, cd.dptr, cd.iptr]
    L.shape_engine_get_lghtcrv.argtypes = [vp, C.c_int, cd.dptr, cd.dptr, P(C.c_double), P(C.c_double)]
    L.shape_engine_get_seen.argtypes = [vp, C.c_char_p]
    L.shape_engine_get_realized.argtypes = [vp, cd.dptr, cd.dptr, cd.dptr, cd.dptr]
    L.shape_engine_last_time_ms.argtypes = [vp, P(C.c_double)]
    L.shape_engine_stage_times.argtypes = [vp, C.c_int, cd.dptr, C.c_int]
    L.shape_engine_set_bin_capacity.argtypes = [vp, C.c_int]
    L.shape_engine_set_fp32_exact.argtypes = [vp, C.c_int]
    L.shape_engine_set_raster_tuning.argtypes = [vp, C.c_int]
    L.shape_engine_vary_params.argtypes = [vp, P(VaryOptions), cd.dptr]
    L.shape_engine_set_spin_device.argtypes = [vp, C.c_int]
    L.shape_engine_get_frame_view.argtypes = [vp, C.c_int, cd.dptr, cd.dptr]
    L.shape_engine_get_raster_tuning.argtypes = [vp, C.c_int, P(C.c_int), P(C.c_int), cd.dptr]
    L.shape_engine_set_frame_view.argtypes = [vp, C.c_int, cd.dptr, cd.dptr, cd.dptr, C.c_double, C.c_double]
    L.shape_engine_set_point_view.argtypes = [vp, C.c_int, cd.dptr, cd.dptr, cd.dptr]
    L.shape_engine_set_spin_model.argtypes = [vp, P(cd.SpinState), cd.dptr, cd.dptr, cd.dptr, cd.dptr]
    L.shape_engine_set_spin_param.argtypes = [vp, C.c_int, C.c_int, C.c_double]
    L.shape_engine_set_penalties.argtypes = [vp, C.c_int, P(C.c_int), cd.dptr]
    L.shape_mod_read.argtypes = [C.c_char_p, P(vp)]
    L.shape_mod_free.argtypes = [vp]
    L.shape_mod_free.restype = None
    L.shape_mod_model.argtypes = [vp, P(cd.ModelDesc)]
    L.shape_mod_radar_law.argtypes = [vp, C.c_int, P(cd.RadarLaw)]
    L.shape_mod_optical_law.argtypes = [vp, C.c_int, P(cd.OpticalLaw)]
    L.shape_mod_spin.argtypes = [vp, P(cd.SpinState)]
    L.shape_mod_free_params.argtypes = [vp, P(FitParam), C.c_int]
    L.shape_mod_write.argtypes = [vp, C.c_char_p]
    L.shape_mod_take_engine.argtypes = [vp, vp]
    L.shape_write_fitdat.argtypes = [C.c_char_p, C.c_int, C.c_int, cd.dptr, C.c_double, C.c_double]
    L.shape_ephem_view.argtypes = [P(cd.EphemPoint), C.c_int, P(cd.EphemPoint), C.c_int, C.c_double, cd.dptr,
                                   cd.dptr, cd.dptr, P(C.c_double), P(C.c_double), P(C.c_double)]
    L.shape_ephem_radar_view.argtypes = [P(cd.EphemPoint), C.c_int, C.c_double, C.c_int, P(C.c_double), cd.dptr,
                                         cd.dptr]
    L.shape_delcor_offsets.argtypes = [cd.dptr, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, P(C.c_double), P(C.c_double)]
    L.shape_obs_read.argtypes = [C.c_char_p, P(vp)]
    L.shape_obs_free.argtypes = [vp]
    L.shape_obs_free.restype = None
    L.shape_obs_nsets.argtypes = [vp]
    L.shape_obs_set_type.argtypes = [vp, C.c_int]
    L.shape_obs_lghtcrv_info.argtypes = [vp, C.c_int, P(C.c_int), P(C.c_int), P(C.c_int)]
    L.shape_obs_lghtcrv.argtypes = [vp, C.c_int, P(cd.SpinState), C.c_int, C.c_double, P(ObsOptions), C.c_double,
                                    P(cd.LghtcrvSet), P(cd.LghtcrvPoint), cd.dptr, cd.dptr, cd.dptr, cd.dptr]
    L.shape_obs_doppler.argtypes = [vp, C.c_int, P(cd.SpinState), C.c_int, C.c_double, P(ObsOptions),
                                    P(cd.DopplerSet), P(cd.DopplerFrame), cd.dptr, cd.dptr]
    L.shape_obs_set.argtypes = [vp, C.c_int, P(cd.DeldopSet), P(C.c_int), P(C.c_int), cd.dptr, cd.dptr,
                                P(C.c_size_t)]
    L.shape_obs_frames.argtypes = [vp, C.c_int, P(cd.SpinState), C.c_int, C.c_double, P(ObsOptions),
                                   P(cd.DeldopFrame), cd.dptr, cd.dptr, cd.dptr]
    L.shape_obs_views.argtypes = [vp, C.c_int, P(C.c_int), P(C.c_int)]
    L.shape_obs_set_maskdir.argtypes = [vp, C.c_char_p]
    L.shape_obs_frames_views.argtypes = [vp, C.c_int, P(cd.SpinState), C.c_int, C.c_double, P(ObsOptions),
                                         P(cd.DeldopFrame), cd.dptr, cd.dptr, cd.dptr]
    L.shape_read_lghtcrv_data.argtypes = [C.c_char_p, C.c_int, C.c_double, cd.dptr, cd.dptr, cd.dptr]
    L.shape_read_radar_data.argtypes = [C.c_char_p, C.c_int, C.c_int, P(C.c_int), P(C.c_int), C.c_int, C.c_double,
                                        C.c_double, C.c_double, cd.dptr, cd.dptr, cd.dptr]
    L.shape_engine_write_fitdat.argtypes = [vp, C.c_int, C.c_double, C.c_char_p]
    L.shape_engine_get_penalties.argtypes = [vp, cd.dptr, C.c_int]
    L.shape_engine_get_spin_param.argtypes = [vp, C.c_int, C.c_int, P(C.c_double)]
    L.shape_realize_spin.argtypes = [P(cd.SpinState), cd.dptr, cd.dptr, C.c_int, cd.dptr, cd.dptr, cd.dptr,
                                     cd.dptr]
    L.shape_engine_get_tuning.argtypes = [vp, P(C.c_int), C.c_int]
    L.shape_engine_bestfit.argtypes = [vp, P(FitParam), C.c_int, P(FitOptions), P(FitResult), cd.dptr, C.c_int]
    L.shape_engine_get_scale.argtypes = [vp, C.c_int, P(C.c_double)]
    L.shape_chi2_frames_noalloc.argtypes = [C.c_int, C.c_int, P(C.c_longlong), C.c_void_p, C.c_void_p,
                                            C.c_void_p, cd.dptr, cd.iptr, cd.dptr, cd.dptr]
    L.shape_engine_kernels_per_eval.argtypes = [vp, C.c_int, P(C.c_int)]
    L.shape_server_create.argtypes = [C.c_int, C.c_size_t, C.c_int, P(vp)]
    L.shape_server_destroy.argtypes = [vp]
    L.shape_server_add_workload.argtypes = [vp, vp, C.c_int]
    L.shape_server_workload_bytes.argtypes = [vp, C.c_int, P(C.c_size_t)]
    L.shape_server_run.argtypes = [vp, P(Request), C.c_int, P(RequestResult), P(ServerStats)]
    L.shape_server_start.argtypes = [vp]
    L.shape_server_submit.argtypes = [vp, C.c_int, cd.dptr, P(C.c_longlong)]
    L.shape_server_poll.argtypes = [vp, C.c_longlong, P(RequestResult)]
    L.shape_server_wait.argtypes = [vp, C.c_longlong, C.c_double, P(RequestResult)]
    L.shape_server_stats_get.argtypes = [vp, P(ServerStats)]
    L.shape_server_stop.argtypes = [vp]
    _lib = L
    return L


def abi_sizes():
    L = load_library()
    out = (C.c_size_t * 32)()
    n = L.shape_abi_sizes(out, 32)
    return [out[i] for i in range(min(n, 32))]


class EngineError(RuntimeError):
    pass


def _chk(rc):
    if rc < 0:
        raise EngineError("shape engine error %d: %s" % (rc, load_library().shape_last_error().decode()))
    return rc


def _summary_dict(s):
    return {k: getattr(s, k) for k, _ in EvalSummary._fields_}


class Engine:
    """One engine handle: device-resident model and datasets."""

    def __init__(self, device=0):
        self.L = load_library()
        h = C.c_void_p()
        _chk(self.L.shape_engine_create(device, C.byref(h)))
        self.h = h
        self.deldops, self.lghtcrvs, self.set_index = [], [], []
        self.posets = []
        self.model = None
        self._keep = []

    def close(self):
        if self.h:
            self.L.shape_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_model(self, model):
        self.model = model
        d = model.desc()
        self._keep.append(d)
        _chk(self.L.shape_engine_set_model(self.h, C.byref(d)))

    def set_params(self, params):
        _chk(self.L.shape_engine_set_params(self.h, C.byref(params)))

    def add_deldop(self, ds):
        if getattr(ds, "views", None):
            arr = ds.view_array()
            self._keep.append(arr)
            idx = _chk(self.L.shape_engine_add_deldop_set_views(self.h, C.byref(ds.set), ds.nframes, ds.nviews,
                                                                arr, cd.as_dptr(ds.obs),
                                                                cd.as_dptr(ds.oneovervar)))
        else:
            arr = ds.frame_array()
            self._keep.append(arr)
            idx = _chk(self.L.shape_engine_add_deldop_set(self.h, C.byref(ds.set), ds.nframes, arr,
                                                          cd.as_dptr(ds.obs), cd.as_dptr(ds.oneovervar)))
        self.deldops.append(ds)
        self.set_index.append(("deldop", len(self.deldops) - 1))
        return idx

    def add_doppler(self, ds):
        """A Doppler set; its frames join the radar frames in call order."""
        arr = ds.frame_array()
        self._keep.append(arr)
        idx = _chk(self.L.shape_engine_add_doppler_set(self.h, C.byref(ds.set), ds.nframes, arr,
                                                       cd.as_dptr(ds.obs), cd.as_dptr(ds.oneovervar)))
        self.deldops.append(ds)
        self.set_index.append(("doppler", len(self.deldops) - 1))
        return idx

    def radar_overflow(self):
        """[overflow_o2, overflow_m2, overflow_xsec, overflow_dopmean] per radar frame."""
        nfr = len(self.frames)
        out = np.zeros(4 * max(1, nfr))
        n = _chk(self.L.shape_engine_get_radar_overflow(self.h, cd.as_dptr(out), nfr))
        return out[:4 * n].reshape(n, 4)

    def add_lghtcrv(self, ds):
        arr = ds.point_array()
        self._keep.append(arr)
        idx = _chk(self.L.shape_engine_add_lghtcrv_set(self.h, C.byref(ds.bind()), arr))
        self.lghtcrvs.append(ds)
        self.set_index.append(("lghtcrv", len(self.lghtcrvs) - 1))
        return idx

    def add_poset(self, ds):
        """A plane-of-sky set (synth.PosetDataset)."""
        st, frames, obs, oov = ds.bind()
        self._keep.extend([frames, obs, oov])
        idx = _chk(self.L.shape_engine_add_poset_set(self.h, C.byref(st), len(ds.frames), frames,
                                                     cd.as_dptr(obs), cd.as_dptr(oov)))
        self.posets.append(ds)
        self.set_index.append(("poset", len(self.posets) - 1))
        return idx

    def poset(self, set_idx, frame):
        """(fit image [ncol, nrow], brightness image [2n+1, 2n+1], results dict)
        of a plane-of-sky frame after the last evaluation."""
        kind, k = self.set_index[set_idx]
        assert kind == "poset", kind
        ds = self.posets[k]
        fr = ds.frames[frame]
        fit = np.zeros((fr["ncol"], fr["nrow"]))
        side = 2 * fr["pos_n"] + 1
        b = np.zeros((side, side))
        r = cd.PosetResult()
        _chk(self.L.shape_engine_get_poset(self.h, int(set_idx), int(frame), cd.as_dptr(fit), cd.as_dptr(b),
                                           C.byref(r)))
        return fit, b, {k: getattr(r, k) for k, _ in cd.PosetResult._fields_}

    def finalize(self):
        _chk(self.L.shape_engine_finalize(self.h))

    def set_bin_capacity(self, cap):
        _chk(self.L.shape_engine_set_bin_capacity(self.h, int(cap)))

    def set_fp32_exact(self, exact=True):
        """Batched FP32 form, radar views: True (the default) redoes pixels
        whose decisions lie within FP32 error by the FP64 rules; False keeps
        the FP32 decisions (faster raster)."""
        _chk(self.L.shape_engine_set_fp32_exact(self.h, 1 if exact else 0))

    def set_spin_device(self, on=True):
        """Realize the views from the spin model inside each evaluation
        (principal-axis rotators): spin trials replay the graph only."""
        _chk(self.L.shape_engine_set_spin_device(self.h, 1 if on else 0))

    def frame_view(self, frame):
        """(ae 3x3, spin vector) of radar frame `frame` as last realized."""
        ae, sp = np.zeros(9), np.zeros(3)
        _chk(self.L.shape_engine_get_frame_view(self.h, int(frame), cd.as_dptr(ae), cd.as_dptr(sp)))
        return ae.reshape(3, 3), sp

    def vary_params(self, flags, delcor0_free=None, dopscale_free=None):
        """shape_engine_vary_params: flags = (vary_delcor0, vary_radalb,
        vary_optalb, vary_dopscale); per dataset free flags. Returns the four
        means (deldop_zmax, rad_xsec, opt_brightness, cos_subradarlat)."""
        o = VaryOptions()
        o.vary_delcor0, o.vary_radalb, o.vary_optalb, o.vary_dopscale = (int(x) for x in flags)
        keep = []
        for name, v in (("delcor0_free", delcor0_free), ("dopscale_free", dopscale_free)):
            if v is not None:
                a = (C.c_int * len(v))(*[int(x) for x in v])
                keep.append(a)
                setattr(o, name, C.cast(a, C.POINTER(C.c_int)))
        out = np.zeros(4)
        _chk(self.L.shape_engine_vary_params(self.h, C.byref(o), cd.as_dptr(out)))
        return out

    def set_raster_tuning(self, mode=-1):
        """-1: time the raster candidates at each batched form's first
        evaluation and keep the fastest; 0 / 1: the tile-per-CTA / warp-
        independent kernel, one CTA per tile."""
        _chk(self.L.shape_engine_set_raster_tuning(self.h, int(mode)))

    def raster_tuning(self, form):
        """{'tuned', 'variant', 'persistent', 'ms': [4 candidate times]}."""
        if isinstance(form, str):
            form = FORMS[form]
        v, p, ms = C.c_int(), C.c_int(), np.zeros(4)
        t = _chk(self.L.shape_engine_get_raster_tuning(self.h, form, C.byref(v), C.byref(p), cd.as_dptr(ms)))
        return {"tuned": bool(t), "variant": v.value, "persistent": p.value, "ms": ms.tolist()}

    def set_frame_view(self, frame, ae, oe, spin, deloff=0.0, dopoff=0.0):
        """New view for radar frame `frame` (numbered across sets): 3x3 ae
        and oe, the spin vector and the delay / Doppler offsets."""
        a = np.ascontiguousarray(ae, dtype=np.float64).reshape(9)
        o = np.ascontiguousarray(oe, dtype=np.float64).reshape(9)
        w = np.ascontiguousarray(spin, dtype=np.float64).reshape(3)
        _chk(self.L.shape_engine_set_frame_view(self.h, int(frame), cd.as_dptr(a), cd.as_dptr(o), cd.as_dptr(w),
                                                float(deloff), float(dopoff)))

    def set_point_view(self, point, ae, oe, se):
        """New view for lightcurve point `point` (numbered across sets)."""
        a = np.ascontiguousarray(ae, dtype=np.float64).reshape(9)
        o = np.ascontiguousarray(oe, dtype=np.float64).reshape(9)
        q = np.ascontiguousarray(se, dtype=np.float64).reshape(9)
        _chk(self.L.shape_engine_set_point_view(self.h, int(point), cd.as_dptr(a), cd.as_dptr(o), cd.as_dptr(q)))

    def tuning(self):
        out = (C.c_int * 8)()
        n = _chk(self.L.shape_engine_get_tuning(self.h, out, 8))
        keys = ["bin_capacity", "max_bin", "nonempty_tiles", "tiles", "tile_w"]
        return dict(zip(keys[:n], [out[i] for i in range(n)]))

    def keep_pos(self, keep=True):
        _chk(self.L.shape_engine_keep_pos(self.h, 1 if keep else 0))

    def set_scale(self, j, v):
        _chk(self.L.shape_engine_set_scale(self.h, j, float(v)))

    def set_vertex_r(self, i, v):
        _chk(self.L.shape_engine_set_vertex_r(self.h, i, float(v)))

    def get_scale(self, j):
        v = C.c_double()
        _chk(self.L.shape_engine_get_scale(self.h, j, C.byref(v)))
        return v.value

    def get_vertex_r(self, i):
        v = C.c_double()
        _chk(self.L.shape_engine_get_vertex_r(self.h, i, C.byref(v)))
        return v.value

    def set_spin_model(self, spin, frame_t=None, frame_orbspin=None, angleoff=None, omegaoff=None):
        """Spin model of the views: a spin_state(), per radar frame its view
        epoch and orbital spin (nframes x 3), per dataset its angle and spin
        offsets (nsets x 3). Realizes every view now."""
        self._spin = spin
        keep = [None if v is None else np.ascontiguousarray(v, dtype=np.float64).ravel()
                for v in (angleoff, omegaoff, frame_t, frame_orbspin)]
        ptrs = [cd.as_dptr(v) if v is not None else None for v in keep]
        _chk(self.L.shape_engine_set_spin_model(self.h, C.byref(spin), *ptrs))

    def set_penalties(self, penalties):
        """penalties: list of (type, weight); [] removes them."""
        n = len(penalties)
        types = (C.c_int * max(1, n))(*[int(t) for t, _ in penalties])
        w = np.array([float(x) for _, x in penalties] or [0.0])
        _chk(self.L.shape_engine_set_penalties(self.h, n, types, cd.as_dptr(w)))

    def penalties(self):
        """Each penalty's base value at the last evaluation."""
        out = np.zeros(64)
        n = _chk(self.L.shape_engine_get_penalties(self.h, cd.as_dptr(out), 64))
        return out[:n].copy()

    def active(self):
        """check_surface's (vertex, facet) active flags at the last
        evaluation with penalties."""
        v = np.zeros(self.model.nv, dtype=np.uint8)
        f = np.zeros(self.model.nf, dtype=np.uint8)
        _chk(self.L.shape_engine_get_active(self.h, v.ctypes.data_as(C.c_void_p), f.ctypes.data_as(C.c_void_p)))
        return v, f

    def write_fitdat(self, frame, sdev, path):
        _chk(self.L.shape_engine_write_fitdat(self.h, int(frame), float(sdev), os.fsencode(path)))

    def set_spin_param(self, kind, index, value):
        _chk(self.L.shape_engine_set_spin_param(self.h, int(kind), int(index), float(value)))

    def get_spin_param(self, kind, index):
        v = C.c_double()
        _chk(self.L.shape_engine_get_spin_param(self.h, int(kind), int(index), C.byref(v)))
        return v.value

    def bestfit(self, params, form=FORM_BATCHED_FP64, term_prec=1e-4, term_maxiter=0, trace_max=0):
        """params: list of (kind, index, step, tol, abstol). Returns the
        result dict and the trial trace [(param number, value), ...]."""
        if isinstance(form, str):
            form = FORMS[form]
        arr = (FitParam * len(params))(*[FitParam(*t) for t in params])
        opt = FitOptions(form, term_prec, term_maxiter)
        res = FitResult()
        tr = np.zeros(2 * max(1, trace_max))
        _chk(self.L.shape_engine_bestfit(self.h, arr, len(params), C.byref(opt), C.byref(res),
                                         cd.as_dptr(tr) if trace_max else None, trace_max))
        out = {k: getattr(res, k) for k, _ in FitResult._fields_}
        trace = [(int(tr[2 * i]), tr[2 * i + 1]) for i in range(res.trace_len)]
        return out, trace

    def evaluate(self, form=FORM_PLAIN_FP64):
        if isinstance(form, str):
            form = FORMS[form]
        s = EvalSummary()
        _chk(self.L.shape_engine_evaluate(self.h, form, C.byref(s)))
        return _summary_dict(s)

    def kernels_per_eval(self, form):
        n = C.c_int()
        _chk(self.L.shape_engine_kernels_per_eval(self.h, form, C.byref(n)))
        return n.value

    def last_ms(self):
        v = C.c_double()
        _chk(self.L.shape_engine_last_time_ms(self.h, C.byref(v)))
        return v.value

    STAGES = ["realize", "reset", "transform", "bin", "raster_synth", "chi2", "lc_photo", "finalize"]

    def stage_times(self, form=FORM_BATCHED_FP32):
        """Stage times in ms of one batched evaluation (shape_engine_stage_times);
        with the fused chi-square kernel its time is under "finalize" and
        "chi2" is empty."""
        if isinstance(form, str):
            form = FORMS[form]
        ms = np.zeros(8)
        n = _chk(self.L.shape_engine_stage_times(self.h, form, cd.as_dptr(ms), 8))
        return dict(zip(self.STAGES[:n], ms[:n].tolist()))

    @property
    def frames(self):
        out = []
        for ds in self.deldops:
            out.extend(ds.frames)
        return out

    def results(self):
        nfr = len(self.frames)
        arr = (cd.DeldopResult * max(1, nfr))()
        n = _chk(self.L.shape_engine_get_deldop_results(self.h, arr, nfr))
        return [cd.result_to_dict(arr[i]) for i in range(n)]

    def fit(self, frame):
        fr = self.frames[frame]
        out = np.zeros(getattr(fr, "ndel", 1) * fr.ndop)
        _chk(self.L.shape_engine_get_fit(self.h, frame, cd.as_dptr(out)))
        return out

    def pos(self, frame):
        fr = self.frames[frame]
        side = 2 * fr.pos_n + 1
        z = np.zeros(side * side); cose = np.zeros(side * side)
        f = np.zeros(side * side, dtype=np.int32)
        _chk(self.L.shape_engine_get_pos(self.h, frame, cd.as_dptr(z), cd.as_dptr(cose), cd.as_iptr(f)))
        return {"z": z, "cose": cose, "f": f}

    def lghtcrv_pos(self, set_idx, point, pt):
        side = 2 * pt.pos_n + 1
        np_ = side * side
        z, cose, cosi, zill = (np.zeros(np_) for _ in range(4))
        f = np.zeros(np_, dtype=np.int32); fill = np.zeros(np_, dtype=np.int32)
        _chk(self.L.shape_engine_get_lghtcrv_pos(self.h, set_idx, point, cd.as_dptr(z), cd.as_dptr(cose),
                                                 cd.as_dptr(cosi), cd.as_iptr(f), cd.as_dptr(zill),
                                                 cd.as_iptr(fill)))
        return {"z": z, "cose": cose, "cosi": cosi, "f": f, "zill": zill, "fill": fill}

    def lghtcrv(self, set_idx, ds):
        y = np.zeros(ds.set.ncalc); fit = np.zeros(ds.set.n)
        cal, chi2 = C.c_double(), C.c_double()
        _chk(self.L.shape_engine_get_lghtcrv(self.h, set_idx, cd.as_dptr(y), cd.as_dptr(fit),
                                             C.byref(cal), C.byref(chi2)))
        return {"y": y, "fit": fit, "cal": cal.value, "chi2": chi2.value}

    def seen(self):
        buf = C.create_string_buffer(self.model.nf)
        _chk(self.L.shape_engine_get_seen(self.h, buf))
        return np.frombuffer(buf.raw, dtype=np.uint8).copy()

    def realized(self):
        m = self.model
        x = np.zeros((m.nv, 3)); vn = np.zeros((m.nv, 3))
        fn = np.zeros((m.nf, 3)); area = np.zeros(m.nf)
        _chk(self.L.shape_engine_get_realized(self.h, cd.as_dptr(x), cd.as_dptr(vn), cd.as_dptr(fn),
                                              cd.as_dptr(area)))
        return {"x": x, "vn": vn, "fn": fn, "area": area}


def read_radar_data(path, ndel, ndop, idel_use=None, idop_use=None, big_endian=True, sdev=1.0, gamma=1.0,
                    nlooks=0.0, pixweight=None):
    """One radar data file (shape_read_radar_data): (obs, 1/variance) of the
    window idel_use x idop_use (1-based, inclusive; default the whole
    stored image), each [rows, cols]."""
    dl = idel_use or (1, ndel)
    dp = idop_use or (1, ndop)
    wd, wp = dl[1] - dl[0] + 1, dp[1] - dp[0] + 1
    obs, oov = np.zeros(max(1, wd * wp)), np.zeros(max(1, wd * wp))
    pw = None if pixweight is None else np.ascontiguousarray(pixweight, dtype=np.float64).ravel()
    _chk(load_library().shape_read_radar_data(os.fsencode(path), ndel, ndop, (C.c_int * 2)(*dl), (C.c_int * 2)(*dp),
                                              1 if big_endian else 0, float(sdev), float(gamma), float(nlooks),
                                              cd.as_dptr(pw) if pw is not None else None, cd.as_dptr(obs),
                                              cd.as_dptr(oov)))
    return obs.reshape(wd, wp), oov.reshape(wd, wp)


def ephem_view(ast, t, sun=None):
    """View geometry at epoch t from ephemeris rows (t, ra, dec, dist):
    dict of oe (3x3), se (3x3, bistatic), s, solar_phase, solar_azimuth,
    dist."""
    def table(rows):
        a = np.ascontiguousarray(rows, dtype=np.float64).reshape(-1, 4)
        return (cd.EphemPoint * len(a))(*[cd.EphemPoint(*r) for r in a]), len(a)
    A, na = table(ast)
    S, ns = table(sun) if sun is not None else (None, 0)
    oe, se, s = np.zeros(9), np.zeros(9), np.zeros(3)
    ph, az, d = C.c_double(), C.c_double(), C.c_double()
    _chk(load_library().shape_ephem_view(A, na, S, ns, float(t), cd.as_dptr(oe), cd.as_dptr(se), cd.as_dptr(s),
                                         C.byref(ph), C.byref(az), C.byref(d)))
    return {"oe": oe.reshape(3, 3), "se": se.reshape(3, 3), "s": s, "solar_phase": ph.value,
            "solar_azimuth": az.value, "dist": d.value}


def ephem_radar_view(ast, t_obs, perform_ltc=True):
    """(view epoch, oe 3x3, orbital spin) of a radar view (shape_ephem_radar_view)."""
    a = np.ascontiguousarray(ast, dtype=np.float64).reshape(-1, 4)
    A = (cd.EphemPoint * len(a))(*[cd.EphemPoint(*r) for r in a])
    tv, oe, s = C.c_double(), np.zeros(9), np.zeros(3)
    _chk(load_library().shape_ephem_radar_view(A, len(a), float(t_obs), 1 if perform_ltc else 0, C.byref(tv),
                                               cd.as_dptr(oe), cd.as_dptr(s)))
    return tv.value, oe.reshape(3, 3), s


def delcor_offsets(a, t0, t_view, del_per_pixel, dop_per_pixel, Ftx):
    """(deloff, dopoff) of a view from a delay-correction polynomial a[0..n]."""
    c = np.ascontiguousarray(a, dtype=np.float64)
    d, p = C.c_double(), C.c_double()
    _chk(load_library().shape_delcor_offsets(cd.as_dptr(c), len(c) - 1, float(t0), float(t_view),
                                             float(del_per_pixel), float(dop_per_pixel), float(Ftx), C.byref(d),
                                             C.byref(p)))
    return d.value, p.value


def read_lghtcrv_data(path, n, sun_appmag):
    """A lightcurve data file (shape_read_lghtcrv_data): (t, obs, 1/variance)."""
    t, obs, oov = np.zeros(n), np.zeros(n), np.zeros(n)
    _chk(load_library().shape_read_lghtcrv_data(os.fsencode(path), n, float(sun_appmag), cd.as_dptr(t),
                                                cd.as_dptr(obs), cd.as_dptr(oov)))
    return t, obs, oov


def write_fitdat(path, fit, cal, sdev):
    """The listfit file of one radar frame: cal * fit / sdev, one "%13.6e" per line."""
    f = np.ascontiguousarray(fit, dtype=np.float64)
    ndel, ndop = f.shape if f.ndim == 2 else (1, f.size)
    _chk(load_library().shape_write_fitdat(os.fsencode(path), ndel, ndop, cd.as_dptr(f), float(cal), float(sdev)))


class VaryOptions(C.Structure):
    _fields_ = [("vary_delcor0", C.c_int), ("vary_radalb", C.c_int), ("vary_optalb", C.c_int),
                ("vary_dopscale", C.c_int), ("delcor0_free", C.POINTER(C.c_int)),
                ("dopscale_free", C.POINTER(C.c_int))]


class ObsOptions(C.Structure):
    _fields_ = [("perform_ltc", C.c_int), ("dd_gamma", C.c_double), ("speckle", C.c_int), ("big_endian", C.c_int)]


class ObsFile:
    """A SHAPE observation file read by shape_obs_read (delay-Doppler sets)."""

    def __init__(self, path):
        self.L = load_library()
        self.h = None
        h = C.c_void_p()
        _chk(self.L.shape_obs_read(os.fsencode(path), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.L.shape_obs_free(self.h)
            self.h = None

    __del__ = close

    def nsets(self):
        return _chk(self.L.shape_obs_nsets(self.h))

    def set_info(self, s):
        st, law, nf, ne = cd.DeldopSet(), C.c_int(), C.c_int(), C.c_size_t()
        ao, oo = np.zeros(3), np.zeros(3)
        _chk(self.L.shape_obs_set(self.h, s, C.byref(st), C.byref(law), C.byref(nf), cd.as_dptr(ao), cd.as_dptr(oo),
                                  C.byref(ne)))
        return {"set": st, "iradlaw": law.value, "nframes": nf.value, "angleoff": ao, "omegaoff": oo,
                "nelem": ne.value}

    def set_type(self, s):
        """0: delay-Doppler set, 1: Doppler set, 2: lightcurve set."""
        return _chk(self.L.shape_obs_set_type(self.h, s))

    def lghtcrv_info(self, s):
        law, nc, n = C.c_int(), C.c_int(), C.c_int()
        _chk(self.L.shape_obs_lghtcrv_info(self.h, s, C.byref(law), C.byref(nc), C.byref(n)))
        return {"ioptlaw": law.value, "ncalc": nc.value, "n": n.value}

    def lghtcrv(self, s, spin, pos_n, km_per_pixel, sun_appmag=-26.75, perform_ltc=1, law=None):
        """A lightcurve set: synth.LightcurveDataset ready for the engine."""
        from . import synth
        info = self.lghtcrv_info(s)
        nc, n = info["ncalc"], info["n"]
        st = cd.LghtcrvSet()
        if law is not None:
            st.law = law
        pts = (cd.LghtcrvPoint * nc)()
        x, t, obs, oov = np.zeros(nc), np.zeros(n), np.zeros(n), np.zeros(n)
        opt = ObsOptions(perform_ltc, 1.0, 0, 1)
        _chk(self.L.shape_obs_lghtcrv(self.h, s, C.byref(spin), int(pos_n), float(km_per_pixel), C.byref(opt),
                                      float(sun_appmag), C.byref(st), pts, cd.as_dptr(x), cd.as_dptr(t),
                                      cd.as_dptr(obs), cd.as_dptr(oov)))
        ds = synth.LightcurveDataset(st, list(pts), x, t, obs, oov)
        ds.bind()
        return ds

    def poset(self, s, spin, perform_ltc=1):
        """A plane-of-sky set's frames (list of cd.PosetFrame with the
        geometry filled), their image files and pixel-weighting flags."""
        law, nf = C.c_int(), C.c_int()
        _chk(self.L.shape_obs_poset_info(self.h, s, C.byref(law), C.byref(nf)))
        frames = (cd.PosetFrame * nf.value)()
        opt = ObsOptions(perform_ltc, 1.0, 0, 1)
        _chk(self.L.shape_obs_poset(self.h, s, C.byref(spin), C.byref(opt), frames))
        files = []
        for k in range(nf.value):
            buf = C.create_string_buffer(4096)
            w = C.c_int()
            _chk(self.L.shape_obs_poset_file(self.h, s, k, buf, 4096, C.byref(w)))
            files.append((buf.value.decode(), w.value))
        return list(frames), files, law.value

    def set_maskdir(self, path):
        """The .par file's mask directory: weighted frames' masks read from it."""
        _chk(self.L.shape_obs_set_maskdir(self.h, os.fsencode(str(path))))

    def doppler(self, s, spin, pos_n, km_per_pixel, nframes=None, ndop=None, perform_ltc=1, speckle=0,
                big_endian=1):
        """A Doppler set: (shape_doppler_set, frames, obs, 1/variance); each
        frame's spectrum is its mask window (the whole spectrum without one)."""
        info = self.set_info(s)
        nframes = info["nframes"]
        st = cd.DopplerSet()
        fr = (cd.DopplerFrame * nframes)()
        obs, oov = np.zeros(info["nelem"]), np.zeros(info["nelem"])
        opt = ObsOptions(perform_ltc, 1.0, speckle, big_endian)
        _chk(self.L.shape_obs_doppler(self.h, s, C.byref(spin), int(pos_n), float(km_per_pixel), C.byref(opt),
                                      C.byref(st), fr, cd.as_dptr(obs), cd.as_dptr(oov)))
        return st, list(fr), obs, oov

    def frames(self, s, spin, pos_n, km_per_pixel, perform_ltc=1, dd_gamma=1.0, speckle=0, big_endian=1):
        info = self.set_info(s)
        nf = info["nframes"]
        fr = (cd.DeldopFrame * nf)()
        obs, oov, sdev = np.zeros(info["nelem"]), np.zeros(info["nelem"]), np.zeros(nf)
        opt = ObsOptions(perform_ltc, dd_gamma, speckle, big_endian)
        _chk(self.L.shape_obs_frames(self.h, s, C.byref(spin), int(pos_n), float(km_per_pixel), C.byref(opt), fr,
                                     cd.as_dptr(obs), cd.as_dptr(oov), cd.as_dptr(sdev)))
        return list(fr), obs, oov, sdev

    def views(self, s):
        """(views per frame, index of the epoch view) of set s."""
        nv, v0 = C.c_int(), C.c_int()
        _chk(self.L.shape_obs_views(self.h, s, C.byref(nv), C.byref(v0)))
        return nv.value, v0.value

    def frame_views(self, s, spin, pos_n, km_per_pixel, perform_ltc=1, dd_gamma=1.0, speckle=0, big_endian=1):
        """A delay-Doppler set of any views per frame: (views per frame in
        rendering order, the epoch view last; obs, 1/variance, sdev)."""
        info = self.set_info(s)
        nf = info["nframes"]
        nv, _ = self.views(s)
        fr = (cd.DeldopFrame * (nf * nv))()
        obs, oov, sdev = np.zeros(info["nelem"]), np.zeros(info["nelem"]), np.zeros(nf)
        opt = ObsOptions(perform_ltc, dd_gamma, speckle, big_endian)
        _chk(self.L.shape_obs_frames_views(self.h, s, C.byref(spin), int(pos_n), float(km_per_pixel), C.byref(opt),
                                           fr, cd.as_dptr(obs), cd.as_dptr(oov), cd.as_dptr(sdev)))
        fl = list(fr)
        return [fl[f * nv:(f + 1) * nv] for f in range(nf)], obs, oov, sdev


class ModFile:
    """A SHAPE model file read by shape_mod_read (host code, no GPU)."""

    def __init__(self, path):
        self.L = load_library()
        self.h = None
        h = C.c_void_p()
        _chk(self.L.shape_mod_read(os.fsencode(path), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.L.shape_mod_free(self.h)
            self.h = None

    __del__ = close

    def model(self):
        """The shape as a synth.Model (copies of the arrays)."""
        from .synth import Model
        d = cd.ModelDesc()
        _chk(self.L.shape_mod_model(self.h, C.byref(d)))
        nv, nf = d.nv, d.nf
        arr = lambda p, n, dt: np.ctypeslib.as_array(p, shape=(n,)).astype(dt).copy()
        af_ptr = arr(d.af_ptr, nv + 1, np.int32)
        m = Model(arr(d.a, 3 * nv, np.float64).reshape(nv, 3), arr(d.u, 3 * nv, np.float64).reshape(nv, 3),
                  arr(d.r, nv, np.float64), arr(d.fv, 3 * nf, np.int32).reshape(nf, 3), af_ptr,
                  arr(d.af_idx, int(af_ptr[-1]), np.int32), np.array(d.scale[:]))
        if d.ncomp > 1:
            nc = d.ncomp
            m.comp_nv, m.comp_nf = arr(d.comp_nv, nc, np.int32), arr(d.comp_nf, nc, np.int32)
            m.comp_scale = arr(d.comp_scale, 3 * nc, np.float64).reshape(nc, 3)
            m.comp_rot = arr(d.comp_rot, 3 * nc, np.float64).reshape(nc, 3)
            m.comp_off = arr(d.comp_off, 3 * nc, np.float64).reshape(nc, 3)
        return m

    def radar_laws(self):
        n = _chk(self.L.shape_mod_radar_law(self.h, 0, None))
        out = []
        for i in range(n):
            law = cd.RadarLaw()
            _chk(self.L.shape_mod_radar_law(self.h, i, C.byref(law)))
            out.append(law)
        return out

    def optical_laws(self):
        n = _chk(self.L.shape_mod_optical_law(self.h, 0, None))
        out = []
        for i in range(n):
            law = cd.OpticalLaw()
            _chk(self.L.shape_mod_optical_law(self.h, i, C.byref(law)))
            out.append(law)
        return out

    def spin(self):
        s = cd.SpinState()
        _chk(self.L.shape_mod_spin(self.h, C.byref(s)))
        return s

    def write(self, path):
        _chk(self.L.shape_mod_write(self.h, os.fsencode(path)))

    def take_engine(self, engine):
        """The engine's current shape and spin parameters into this model."""
        _chk(self.L.shape_mod_take_engine(self.h, engine.h))

    def free_params(self):
        """[(kind, index), ...] in the reference's parameter-list order."""
        n = _chk(self.L.shape_mod_free_params(self.h, None, 0))
        arr = (FitParam * max(1, n))()
        _chk(self.L.shape_mod_free_params(self.h, arr, n))
        return [(arr[i].kind, arr[i].index) for i in range(n)]


def spin_state(pa=1, t0=0.0, angle=(0.0, 0.0, 0.0), omega=(0.0, 0.0, 0.0), omegadot=(0.0, 0.0, 0.0),
               impulses=(), lib=(0.0, 0.0, 0.0), inertia=(1.0, 1.0, 1.0)):
    """A shape_spin_state; impulses: (epoch, (wx, wy, wz)) pairs; inertia:
    principal moments (non-principal-axis states)."""
    s = cd.SpinState()
    s.pa, s.t0 = int(pa), float(t0)
    for j in range(3):
        s.angle[j], s.omega[j], s.omegadot[j] = angle[j], omega[j], omegadot[j]
    s.n_impulse = len(impulses)
    for k, (te, w) in enumerate(impulses[:cd.MAX_IMPULSES]):
        s.t_impulse[k] = te
        for j in range(3):
            s.impulse[k][j] = w[j]
    s.lib_amp, s.lib_freq, s.lib_phase = lib
    for j in range(3):
        s.inertia[j] = inertia[j]
    return s


def realize_spin(spin, t, orbspin=None, angleoff=(0.0, 0.0, 0.0), omegaoff=(0.0, 0.0, 0.0)):
    """shape_realize_spin: (ae [n,3,3] ecliptic -> body, total spin [n,3]
    ecliptic) of a principal-axis spin state at view epochs t."""
    L = load_library()
    t = np.ascontiguousarray(t, dtype=np.float64)
    n = t.size
    orb = np.zeros((n, 3)) if orbspin is None else np.ascontiguousarray(orbspin, dtype=np.float64).reshape(n, 3)
    ae, sp = np.zeros((n, 3, 3)), np.zeros((n, 3))
    ao, oo = np.array(angleoff, dtype=np.float64), np.array(omegaoff, dtype=np.float64)
    _chk(L.shape_realize_spin(C.byref(spin), cd.as_dptr(ao), cd.as_dptr(oo), n, cd.as_dptr(t), cd.as_dptr(orb),
                              cd.as_dptr(ae), cd.as_dptr(sp)))
    return ae, sp


def make_engine(model, params, deldops=(), lghtcrvs=(), device=0, dopplers=(), posets=()):
    """An engine with the sets added in the order deldops, dopplers, lightcurves, plane-of-sky sets."""
    e = Engine(device)
    e.set_model(model)
    e.set_params(params)
    for ds in deldops:
        e.add_deldop(ds)
    for ds in dopplers:
        e.add_doppler(ds)
    for ds in lghtcrvs:
        e.add_lghtcrv(ds)
    for ds in posets:
        e.add_poset(ds)
    e.finalize()
    return e


def engine_synthesizer(model, device=0):
    """A ``synthesize`` callable for synth.* that evaluates the true model
    with the engine's FP64 path (used to build observed images on a GPU)."""
    def deldop(ds, params):
        e = make_engine(model, params, deldops=[ds], device=device)
        e.evaluate(FORM_PLAIN_FP64)
        fits = [e.fit(k) for k in range(ds.nframes)]
        e.close()
        return fits

    def lghtcrv(ds, params):
        e = make_engine(model, params, lghtcrvs=[ds], device=device)
        e.evaluate(FORM_PLAIN_FP64)
        y = e.lghtcrv(0, ds)["y"]
        e.close()
        return y
    return deldop, lghtcrv


def engine_doppler_synthesizer(model, device=0):
    """A ``synthesize`` callable for synth.doppler_dataset (FP64 engine path)."""
    def doppler(ds, params):
        e = make_engine(model, params, dopplers=[ds], device=device)
        e.evaluate(FORM_PLAIN_FP64)
        fits = [e.fit(k) for k in range(ds.nframes)]
        e.close()
        return fits
    return doppler


class Server:
    """Continuous-batching evaluation server on one device (shape_server_*).

    Workloads are registered from configured engines; run() replays a trace of
    (workload, arrival time, scale factors) requests and returns per-request
    results and the trace's statistics."""

    def __init__(self, device=0, hbm_budget_bytes=8 << 30, max_slots=8):
        self.L = load_library()
        h = C.c_void_p()
        _chk(self.L.shape_server_create(device, hbm_budget_bytes, max_slots, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.L.shape_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_workload(self, engine, form=FORM_BATCHED_FP32):
        return _chk(self.L.shape_server_add_workload(self.h, engine.h, form))

    def workload_bytes(self, w):
        b = C.c_size_t()
        _chk(self.L.shape_server_workload_bytes(self.h, w, C.byref(b)))
        return b.value

    def run(self, requests):
        """requests: sequence of (workload, arrival_s, (s0, s1, s2)).
        Returns (list of result dicts, stats dict)."""
        n = len(requests)
        req = (Request * n)()
        for i, (w, t, sc) in enumerate(requests):
            req[i].workload = w
            req[i].arrival_s = t
            for j in range(3):
                req[i].scale[j] = sc[j]
        res = (RequestResult * n)()
        st = ServerStats()
        _chk(self.L.shape_server_run(self.h, req, n, res, C.byref(st)))
        out = [{k: getattr(r, k) for k, _ in RequestResult._fields_} for r in res]
        return out, {k: getattr(st, k) for k, _ in ServerStats._fields_}

    # online use: requests submitted as they arrive, results collected later
    def start(self):
        _chk(self.L.shape_server_start(self.h))

    def submit(self, workload, scale=(1.0, 1.0, 1.0)):
        """Queues one request; returns its ticket."""
        t = C.c_longlong()
        sc = np.ascontiguousarray(scale, dtype=np.float64)
        _chk(self.L.shape_server_submit(self.h, workload, cd.as_dptr(sc), C.byref(t)))
        return t.value

    def poll(self, ticket):
        """The result dict of a finished request, or None while it runs."""
        r = RequestResult()
        if _chk(self.L.shape_server_poll(self.h, ticket, C.byref(r))) == 0:
            return None
        return {k: getattr(r, k) for k, _ in RequestResult._fields_}

    def wait(self, ticket, timeout_s=60.0):
        r = RequestResult()
        _chk(self.L.shape_server_wait(self.h, ticket, float(timeout_s), C.byref(r)))
        return {k: getattr(r, k) for k, _ in RequestResult._fields_}

    def stats(self):
        st = ServerStats()
        _chk(self.L.shape_server_stats_get(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def stop(self):
        _chk(self.L.shape_server_stop(self.h))


PARAM_OBJECTIVE = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_int),
                              C.POINTER(C.c_int))


def bestfit_host(objective, values, params, term_prec=1e-4, term_maxiter=0, trace_max=0):
    """shape_bestfit_host: the bestfit iteration on a host objective.
    objective(values) -> (objective value, posbnd, badradar); values: start
    values of the free parameters (updated in place)."""
    L = load_library()
    L.shape_bestfit_host.argtypes = [PARAM_OBJECTIVE, C.c_void_p, cd.dptr, C.POINTER(FitParam), C.c_int,
                                     C.POINTER(FitOptions), C.POINTER(FitResult), cd.dptr, C.c_int]
    n = len(params)

    def cb(vals, user, posbnd, badradar):
        v, pb, br = objective(np.ctypeslib.as_array(vals, shape=(n,)))
        posbnd[0], badradar[0] = int(pb), int(br)
        return v
    fn = PARAM_OBJECTIVE(cb)
    arr = (FitParam * n)(*[FitParam(*t) for t in params])
    opt = FitOptions(0, term_prec, term_maxiter)
    res = FitResult()
    vals = np.ascontiguousarray(values, dtype=np.float64)
    tr = np.zeros(2 * max(1, trace_max))
    _chk(L.shape_bestfit_host(fn, None, cd.as_dptr(vals), arr, n, C.byref(opt), C.byref(res),
                              cd.as_dptr(tr) if trace_max else None, trace_max))
    values[:] = vals
    return {k: getattr(res, k) for k, _ in FitResult._fields_}


def register_workloads(server, work, params, form, device=0):
    """Registers every (category, model, deldop datasets, lightcurve
    datasets) entry of `work` with the server in one form; returns the
    workload indices."""
    ids = []
    for _, model, dds, lcs in work:
        e = Engine(device)
        e.set_model(model)
        e.set_params(params)
        for ds in dds:
            e.add_deldop(ds)
        for ds in lcs:
            e.add_lghtcrv(ds)
        ids.append(server.add_workload(e, form))
        e.close()
    return ids


def poisson_trace(nreq, rate_per_s, nworkloads, seed=0, scale_jitter=0.05):
    """Seeded Poisson arrivals: exponential gaps of mean 1/rate, workloads
    drawn uniformly, scale factors 1 +- scale_jitter."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, nreq))
    t -= t[0]
    w = rng.integers(0, nworkloads, nreq)
    sc = 1.0 + scale_jitter * rng.uniform(-1, 1, (nreq, 3))
    return [(int(w[i]), float(t[i]), tuple(float(x) for x in sc[i])) for i in range(nreq)]
