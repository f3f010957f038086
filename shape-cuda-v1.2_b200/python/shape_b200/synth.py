"""Seeded synthetic SHAPE inputs with the shapes and sizes of the benchmark
configurations (the reference ships no example .mod/.obs files).

Models are single-component VERTEX models (x = scale*(u*r + a)); datasets are
delay-Doppler frames (one view each) and lightcurves, described with the plain
structs of include/shape_types.h. Observed images are produced by a caller-
supplied ``synthesize`` callable that evaluates the TRUE model (the engine's
FP64 path on a GPU, or the CPU oracle in tests), then noise is added.

Seeds: 42 for shape deviations, 7 for phases and sizes, 1234 for noise.
"""
from dataclasses import dataclass, field
import math

import numpy as np

from . import ctypes_defs as cd

KM2US = 6.67128190396304
KM2HZFACT = 7.72139109254982e-5
DEG = math.pi / 180.0


# --------------------------------------------------------------------- models

@dataclass
class Model:
    a: np.ndarray          # [nv,3]
    u: np.ndarray          # [nv,3]
    r: np.ndarray          # [nv]
    fv: np.ndarray         # [nf,3] int32
    af_ptr: np.ndarray     # [nv+1] int32
    af_idx: np.ndarray     # int32
    scale: np.ndarray = field(default_factory=lambda: np.ones(3))
    name: str = ""
    # several components (comp_nv / comp_nf vertices and facets each, back to
    # back; comp_scale replaces scale; comp_rot Euler angles, comp_off
    # translations): None for one component
    comp_nv: np.ndarray = None
    comp_nf: np.ndarray = None
    comp_scale: np.ndarray = None
    comp_rot: np.ndarray = None
    comp_off: np.ndarray = None

    @property
    def ncomp(self):
        return 1 if self.comp_nv is None else len(self.comp_nv)

    @property
    def nv(self):
        return self.a.shape[0]

    @property
    def nf(self):
        return self.fv.shape[0]

    def copy(self):
        cp = lambda v: None if v is None else v.copy()
        return Model(self.a.copy(), self.u.copy(), self.r.copy(), self.fv.copy(),
                     self.af_ptr.copy(), self.af_idx.copy(), self.scale.copy(), self.name,
                     cp(self.comp_nv), cp(self.comp_nf), cp(self.comp_scale), cp(self.comp_rot), cp(self.comp_off))

    def desc(self):
        """ctypes shape_model_desc pointing into this model's arrays."""
        for k in ("a", "u", "r"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.float64))
        for k in ("fv", "af_ptr", "af_idx"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.int32))
        d = cd.ModelDesc()
        d.nv, d.nf = self.nv, self.nf
        d.a, d.u, d.r = cd.as_dptr(self.a), cd.as_dptr(self.u), cd.as_dptr(self.r)
        for j in range(3):
            d.scale[j] = float(self.scale[j])
        d.fv, d.af_ptr, d.af_idx = cd.as_iptr(self.fv), cd.as_iptr(self.af_ptr), cd.as_iptr(self.af_idx)
        if self.comp_nv is not None:
            self.comp_nv = np.ascontiguousarray(self.comp_nv, dtype=np.int32)
            self.comp_nf = np.ascontiguousarray(self.comp_nf, dtype=np.int32)
            for k in ("comp_scale", "comp_rot", "comp_off"):
                setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.float64))
            d.ncomp = len(self.comp_nv)
            d.comp_nv, d.comp_nf = cd.as_iptr(self.comp_nv), cd.as_iptr(self.comp_nf)
            d.comp_scale, d.comp_rot = cd.as_dptr(self.comp_scale), cd.as_dptr(self.comp_rot)
            d.comp_off = cd.as_dptr(self.comp_off)
        return d


def _orient_outward(x, fv):
    """Make every facet right-handed with its normal pointing away from the origin."""
    p0, p1, p2 = x[fv[:, 0]], x[fv[:, 1]], x[fv[:, 2]]
    nrm = np.cross(p1 - p0, p2 - p1)
    cen = (p0 + p1 + p2) / 3.0
    flip = np.einsum("ij,ij->i", nrm, cen) < 0
    fv = fv.copy()
    fv[flip, 1], fv[flip, 2] = fv[flip, 2].copy(), fv[flip, 1].copy()
    return fv


def _attached(nv, fv):
    """CSR lists of the facets attached to each vertex, in increasing facet order."""
    counts = np.zeros(nv, dtype=np.int64)
    for k in range(3):
        np.add.at(counts, fv[:, k], 1)
    ptr = np.zeros(nv + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    pairs = np.stack([fv.reshape(-1), np.repeat(np.arange(fv.shape[0]), 3)], axis=1)
    order = np.lexsort((pairs[:, 1], pairs[:, 0]))
    idx = pairs[order, 1]
    return ptr.astype(np.int32), idx.astype(np.int32)


def ring_sphere(nrings, nper):
    """Unit directions and facets of a latitude-ring tessellation:
    nrings rings of nper vertices plus 2 poles, 2*nper*nrings facets."""
    dirs = [np.array([0.0, 0.0, 1.0])]
    for k in range(nrings):
        th = math.pi * (k + 1) / (nrings + 1)
        off = 0.5 * (k % 2)
        for m in range(nper):
            ph = 2 * math.pi * (m + off) / nper
            dirs.append(np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)]))
    dirs.append(np.array([0.0, 0.0, -1.0]))
    dirs = np.array(dirs)
    nv = dirs.shape[0]
    ring = lambda k, m: 1 + k * nper + (m % nper)
    faces = []
    for m in range(nper):
        faces.append((0, ring(0, m), ring(0, m + 1)))
    for k in range(nrings - 1):
        for m in range(nper):
            if k % 2 == 0:
                faces.append((ring(k, m), ring(k + 1, m), ring(k, m + 1)))
                faces.append((ring(k, m + 1), ring(k + 1, m), ring(k + 1, m + 1)))
            else:
                faces.append((ring(k, m), ring(k + 1, m), ring(k + 1, m + 1)))
                faces.append((ring(k, m), ring(k + 1, m + 1), ring(k, m + 1)))
    last = nv - 1
    for m in range(nper):
        faces.append((last, ring(nrings - 1, m + 1), ring(nrings - 1, m)))
    return dirs, np.array(faces, dtype=np.int32)


def octa_sphere(levels):
    """Unit directions and facets of an octahedron subdivided `levels` times
    (V = 4**levels * 4 + 2, F = 8 * 4**levels)."""
    verts = [np.array(v, dtype=np.float64) for v in
             [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]]
    faces = [(4, 0, 2), (4, 2, 1), (4, 1, 3), (4, 3, 0), (5, 2, 0), (5, 1, 2), (5, 3, 1), (5, 0, 3)]
    for _ in range(levels):
        cache = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                p = verts[i] + verts[j]
                verts.append(p / np.linalg.norm(p))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for (a, b, c) in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int32)


def _real_sph_harm_basis(dirs, lmax):
    """Real spherical-harmonic-like basis (unnormalised Legendre x cos/sin)."""
    ct = dirs[:, 2]
    ph = np.arctan2(dirs[:, 1], dirs[:, 0])
    st = np.sqrt(np.maximum(0.0, 1 - ct * ct))
    cols = []
    for l in range(1, lmax + 1):
        for m in range(0, l + 1):
            # associated Legendre P_l^m by recurrence
            pmm = np.ones_like(ct)
            for k in range(1, m + 1):
                pmm = pmm * (-(2 * k - 1)) * st
            if l == m:
                plm = pmm
            else:
                pm1 = ct * (2 * m + 1) * pmm
                if l == m + 1:
                    plm = pm1
                else:
                    pa, pb = pmm, pm1
                    for ll in range(m + 2, l + 1):
                        pc = (ct * (2 * ll - 1) * pb - (ll + m - 1) * pa) / (ll - m)
                        pa, pb = pb, pc
                    plm = pb
            cols.append(plm * np.cos(m * ph))
            if m > 0:
                cols.append(plm * np.sin(m * ph))
    B = np.stack(cols, axis=1)
    return B / np.maximum(np.sqrt((B * B).mean(axis=0)), 1e-300)


def make_model(dirs, fv, radius, base=None, name=""):
    nv = dirs.shape[0]
    if base is None:
        a = np.zeros((nv, 3))
        u = dirs.copy()
        r = np.asarray(radius, dtype=np.float64).copy()
    else:
        a = base.copy()
        u = dirs.copy()
        r = np.zeros(nv)
    xr = a + u * r[:, None]
    fv = _orient_outward(xr, fv)
    ptr, idx = _attached(nv, fv)
    return Model(a, u, r, fv, ptr, idx, np.ones(3), name)


def ellipsoid_model(semi=(1.0, 0.8, 0.6), nrings=23, nper=50):
    """Config-1 model: triaxial ellipsoid, 23 rings x 50 + 2 poles =
    1152 vertices / 2300 facets, as a VERTEX model with a on the surface,
    u radial and r = 0."""
    dirs, fv = ring_sphere(nrings, nper)
    base = dirs * np.asarray(semi)[None, :]
    u = base / np.linalg.norm(base, axis=1)[:, None]
    return make_model(u, fv, None, base=base, name="ellipsoid-%d" % fv.shape[0])


def two_component_model(rot=(0.3, 0.5, -0.2), off=(0.6, -0.1, 0.05), radius=0.35):
    """A contact-binary-like two-component VERTEX model: the config-1
    ellipsoid (1152 vertices) and a smaller sphere (602 vertices) that it
    partly hides, rotated by Euler angles rot and translated by off (km),
    scale factors per component."""
    m1 = ellipsoid_model()
    dirs, fv2 = ring_sphere(15, 40)
    base2 = radius * dirs
    m2 = make_model(dirs, fv2, None, base=base2, name="sphere")
    nv1 = m1.nv
    a = np.concatenate([m1.a, m2.a])
    u = np.concatenate([m1.u, m2.u])
    r = np.concatenate([m1.r, m2.r])
    fv = np.concatenate([m1.fv, m2.fv + nv1]).astype(np.int32)
    af_ptr = np.concatenate([m1.af_ptr[:-1], m2.af_ptr + m1.af_ptr[-1]]).astype(np.int32)
    af_idx = np.concatenate([m1.af_idx, m2.af_idx + m1.nf]).astype(np.int32)
    m = Model(a, u, r, fv, af_ptr, af_idx, np.ones(3), "two-component")
    m.comp_nv = np.array([m1.nv, m2.nv], dtype=np.int32)
    m.comp_nf = np.array([m1.nf, m2.nf], dtype=np.int32)
    m.comp_scale = np.array([[1.0, 1.0, 1.0], [1.05, 0.95, 1.0]])
    m.comp_rot = np.array([[0.0, 0.0, 0.0], list(rot)])
    m.comp_off = np.array([[0.0, 0.0, 0.0], list(off)])
    return m


def harmonic_model(nrings=40, nper=100, lmax=8, amp=0.05, seed=42):
    """Config-2/3 model: 4002 vertices / 8000 facets, unit sphere perturbed by
    random real spherical harmonics up to degree 8 with 5% RMS amplitude."""
    dirs, fv = ring_sphere(nrings, nper)
    rng = np.random.default_rng(seed)
    B = _real_sph_harm_basis(dirs, lmax)
    dev = B @ rng.standard_normal(B.shape[1])
    dev *= amp / np.sqrt((dev * dev).mean())
    return make_model(dirs, fv, 1.0 + dev, name="harmonic-%d" % fv.shape[0])


def noisy_octa_model(levels=6, sigma=0.03, seed=42):
    """Config-4 model: 16386 vertices / 32768 facets, unit radii with 3%
    Gaussian noise."""
    dirs, fv = octa_sphere(levels)
    rng = np.random.default_rng(seed)
    return make_model(dirs, fv, 1.0 + sigma * rng.standard_normal(dirs.shape[0]),
                      name="octa-%d" % fv.shape[0])


# ------------------------------------------------------------------- geometry

def unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


def ecl_dir(lon_deg, lat_deg):
    lo, la = lon_deg * DEG, lat_deg * DEG
    return np.array([math.cos(la) * math.cos(lo), math.cos(la) * math.sin(lo), math.sin(la)])


def body_matrix(pole, phase):
    """ecliptic -> body rotation (rows = body axes in ecliptic coords) for a
    principal-axis rotator with spin axis `pole` at rotation phase `phase`."""
    zb = unit(pole)
    x0 = np.cross([0.0, 0.0, 1.0], zb)
    if np.linalg.norm(x0) < 1e-12:
        x0 = np.array([1.0, 0.0, 0.0])
    x0 = unit(x0)
    y0 = np.cross(zb, x0)
    xb = math.cos(phase) * x0 + math.sin(phase) * y0
    yb = -math.sin(phase) * x0 + math.cos(phase) * y0
    return np.stack([xb, yb, zb])


def observer_matrix(to_obs):
    """ecliptic -> observer rotation whose z axis points to the observer."""
    zo = unit(to_obs)
    north = np.array([0.0, 0.0, 1.0]) - zo[2] * zo
    if np.linalg.norm(north) < 1e-12:
        north = np.array([0.0, 1.0, 0.0])
    yo = unit(north)
    xo = np.cross(yo, zo)
    return np.stack([xo, yo, zo])


def rotate_about(v, axis, ang):
    k = unit(axis)
    v = np.asarray(v, dtype=np.float64)
    return v * math.cos(ang) + np.cross(k, v) * math.sin(ang) + k * np.dot(k, v) * (1 - math.cos(ang))


# ------------------------------------------------------------------- datasets

@dataclass
class DeldopDataset:
    set: "cd.DeldopSet"
    frames: list             # list of cd.DeldopFrame
    obs: np.ndarray          # concatenated [sum ndel*ndop]
    oneovervar: np.ndarray
    offsets: np.ndarray      # [nframes+1] element offsets into obs
    # smearing: per frame, its views in rendering order (the epoch view,
    # frames[f], last); None for one view per frame
    views: list = None
    v0: int = 0              # the epoch view's index among the reference's views

    @property
    def nframes(self):
        return len(self.frames)

    @property
    def nviews(self):
        return len(self.views[0]) if self.views else 1

    def frame_array(self):
        arr = (cd.DeldopFrame * len(self.frames))(*self.frames)
        return arr

    def view_array(self):
        """Every frame's views back to back (frame-major, rendering order)."""
        flat = [v for fv in self.views for v in fv]
        return (cd.DeldopFrame * len(flat))(*flat)

    def frame_obs(self, f):
        return self.obs[self.offsets[f]:self.offsets[f + 1]]


@dataclass
class DopplerDataset:
    set: "cd.DopplerSet"
    frames: list             # list of cd.DopplerFrame
    obs: np.ndarray          # concatenated [sum ndop]
    oneovervar: np.ndarray
    offsets: np.ndarray      # [nframes+1] element offsets into obs

    @property
    def nframes(self):
        return len(self.frames)

    def frame_array(self):
        return (cd.DopplerFrame * len(self.frames))(*self.frames)

    def frame_obs(self, f):
        return self.obs[self.offsets[f]:self.offsets[f + 1]]


@dataclass
class LightcurveDataset:
    set: "cd.LghtcrvSet"
    points: list             # list of cd.LghtcrvPoint
    x: np.ndarray
    t: np.ndarray
    obs: np.ndarray
    oneovervar: np.ndarray

    def bind(self):
        self.set.x, self.set.t = cd.as_dptr(self.x), cd.as_dptr(self.t)
        self.set.obs, self.set.oneovervar = cd.as_dptr(self.obs), cd.as_dptr(self.oneovervar)
        return self.set

    def point_array(self):
        return (cd.LghtcrvPoint * len(self.points))(*self.points)


def eval_params(pos_smooth=1, nsinc2=1, sinc2width=7, mask_tol=0.0, mincosine_seen=0.0, mark_seen=1):
    p = cd.EvalParams()
    p.pos_smooth, p.nsinc2, p.sinc2width = pos_smooth, nsinc2, sinc2width
    p.mask_tol, p.mincosine_seen, p.mark_seen = mask_tol, mincosine_seen, mark_seen
    return p


def radar_cosine(R=0.1, C=1.0):
    law = cd.RadarLaw()
    law.type, law.diff_R, law.diff_C = 1, R, C
    law.qs_R, law.qs_C, law.qs_cos_cutoff = 0.0, 0.0, 0.0
    return law


def _frame(pos_n, kmpp, ae, oe, spin, ndel, ndop, delcom, dopcom):
    fr = cd.DeldopFrame()
    fr.pos_n, fr.km_per_pixel = pos_n, kmpp
    cd.fill9(fr.ae, ae)
    cd.fill9(fr.oe, oe)
    for j in range(3):
        fr.spin[j] = float(spin[j])
    fr.deloff = fr.dopoff = 0.0
    fr.ndel, fr.ndop = ndel, ndop
    fr.delcom_vig, fr.dopcom_vig, fr.dopDC_vig = delcom, dopcom, dopcom
    fr.weight = 1.0
    fr.dof = float(ndel * ndop)
    fr.cal_floating, fr.cal = 1, 1.0
    return fr


def _finish_deldop(dset, frames, synthesize, amp, sdev, seed, params):
    sizes = [f.ndel * f.ndop for f in frames]
    offsets = np.zeros(len(frames) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offsets[1:])
    obs = np.zeros(int(offsets[-1]))
    oov = np.full(int(offsets[-1]), 1.0 / (sdev * sdev))
    ds = DeldopDataset(dset, frames, obs, oov, offsets)
    if synthesize is not None:
        fits = synthesize(ds, params)
        rng = np.random.default_rng(seed)
        for f in range(len(frames)):
            ft = np.asarray(fits[f], dtype=np.float64)
            peak = ft.max() if ft.size and ft.max() > 0 else 1.0
            ds.obs[offsets[f]:offsets[f + 1]] = amp * ft / peak + sdev * rng.standard_normal(ft.size)
    return ds


def config1_dataset(synthesize=None, params=None, pos_n=75):
    """Config 1: one 100x100 delay-Doppler frame, POS 151x151 at 15 m/px,
    period 6 h, pole (30, 60) deg, cos^2 law (COSINELAW_DIFF, C=1, R=0.1),
    LONG_ORIG spb=1 stride=1, Ftx 2380 MHz, 0.1 usec x 0.1 Hz pixels."""
    params = params or eval_params()
    pole = ecl_dir(30.0, 60.0)
    omega = 2 * math.pi / 0.25
    to_earth = ecl_dir(0.0, 10.0)
    ae = body_matrix(pole, 0.7)
    oe = observer_matrix(to_earth)
    dset = cd.DeldopSet()
    dset.del_per_pixel, dset.dop_per_pixel = 0.1, 0.1
    dset.Ftx, dset.dopscale = 2380.0, 1.0
    dset.codemethod, dset.spb, dset.stride, dset.dopfftlen = 1, 1, 1, 64
    dset.law = radar_cosine()
    fr = _frame(pos_n, 2.25 / 150.0, ae, oe, omega * pole, 100, 100, 70.0, 50.5)
    return _finish_deldop(dset, [fr], synthesize, 20.0, 1.0, 1234, params)


def batched_dataset(nframes=64, pos_range=(101, 301), ndel_range=(64, 256),
                    ndop_range=(64, 512), synthesize=None, params=None, seed=7,
                    radius=1.05, codemethod=1, spb=1, stride=1, law=None, dopfftlen=64):
    """Config 2 (and, with other sizes, config 4): frames at rotation phases
    uniform in [0, 2pi), odd POS sides, delay/Doppler sizes uniform in the
    given ranges, resolutions scaled so the target spans ~80% of each frame."""
    params = params or eval_params()
    rng = np.random.default_rng(seed)
    pole = ecl_dir(30.0, 60.0)
    omega = 2 * math.pi / 0.25
    to_earth = ecl_dir(0.0, 10.0)
    oe = observer_matrix(to_earth)
    w_obs = oe @ (omega * pole)
    w_proj = math.hypot(w_obs[0], w_obs[1])
    Ftx = 2380.0
    dset = cd.DeldopSet()
    dset.Ftx, dset.dopscale = Ftx, 1.0
    dset.codemethod, dset.spb, dset.stride, dset.dopfftlen = codemethod, spb, stride, dopfftlen
    dset.law = law if law is not None else radar_cosine()
    frames = []
    # one set-level resolution: taken from the median frame size, then each
    # frame's POS scale adapts to its own pixel count
    ndels = rng.integers(ndel_range[0], ndel_range[1] + 1, nframes)
    ndops = rng.integers(ndop_range[0], ndop_range[1] + 1, nframes)
    sides = rng.integers(pos_range[0], pos_range[1] + 1, nframes) | 1
    phases = rng.uniform(0.0, 2 * math.pi, nframes)
    dset.del_per_pixel = KM2US * radius / (0.75 * float(ndel_range[0]))
    dset.dop_per_pixel = 2 * KM2HZFACT * Ftx * w_proj * radius / (0.7 * float(ndop_range[0]))
    for f in range(nframes):
        n = int(sides[f]) // 2
        kmpp = 2 * radius / (0.8 * sides[f])
        ae = body_matrix(pole, float(phases[f]))
        ndel, ndop = int(ndels[f]), int(ndops[f])
        delcom = 0.5 * ndel + 0.5 * (KM2US * radius / dset.del_per_pixel)
        frames.append(_frame(n, kmpp, ae, oe, omega * pole, ndel, ndop, delcom, 0.5 * ndop + 0.5))
    return _finish_deldop(dset, frames, synthesize, 20.0, 1.0, 1234, params)


def smeared_dataset(nframes=4, nviews=3, v0=1, view_interval=0.004, pos_n=75, synthesize=None,
                    params=None, seed=11):
    """Delay-Doppler frames rendered from nviews views each (smearing): view k
    of the reference's numbering sits at t0 + (k - v0) * view_interval days
    (src/shape/read_dat.c:868-873), so its body rotates by omega times that;
    each view carries its own small delay / Doppler correction. The views are
    listed in rendering order, v0+1 .. v0+nviews modulo nviews, ending with
    the epoch view."""
    params = params or eval_params()
    rng = np.random.default_rng(seed)
    pole = ecl_dir(30.0, 60.0)
    omega = 2 * math.pi / 0.25
    to_earth = ecl_dir(0.0, 10.0)
    oe = observer_matrix(to_earth)
    dset = cd.DeldopSet()
    dset.del_per_pixel, dset.dop_per_pixel = 0.1, 0.1
    dset.Ftx, dset.dopscale = 2380.0, 1.0
    dset.codemethod, dset.spb, dset.stride, dset.dopfftlen = 1, 1, 1, 64
    dset.law = radar_cosine()
    frames, views = [], []
    for f in range(nframes):
        phase0 = 0.7 + 2 * math.pi * f / nframes
        fv = [None] * nviews
        for k in range(nviews):
            fr = _frame(pos_n, 2.25 / 150.0, body_matrix(pole, phase0 + omega * (k - v0) * view_interval),
                        oe, omega * pole, 100, 100, 70.0, 50.5)
            fr.deloff, fr.dopoff = rng.uniform(-0.3, 0.3, 2)
            fv[k] = fr
        order = [(v0 + 1 + j) % nviews for j in range(nviews)]
        views.append([fv[k] for k in order])
        frames.append(fv[v0])
    ds = _finish_deldop(dset, frames, synthesize, 20.0, 1.0, 1234 + nviews, params)
    ds.views, ds.v0 = views, v0
    return ds


def config2_dataset(synthesize=None, params=None):
    return batched_dataset(64, (101, 301), (64, 256), (64, 512), synthesize, params, seed=7)


def config4_dataset(synthesize=None, params=None):
    """Config 4: 16 frames, POS pos_pixels=512 (effective 511x511, n=255),
    256x256 delay-Doppler."""
    return batched_dataset(16, (511, 511), (256, 256), (256, 256), synthesize, params, seed=7)


def doppler_dataset(nframes=8, pos_range=(101, 301), ndop_range=(64, 256), synthesize=None,
                    params=None, seed=13, radius=1.05, law=None, span=0.7, sdev=1.0):
    """Doppler-only frames (spectra) at rotation phases uniform in [0, 2pi):
    odd POS sides and spectrum lengths uniform in the given ranges, one
    set-level resolution chosen so the limb-to-limb bandwidth spans `span` of
    the shortest spectrum (span > 1 pushes the model past the spectrum edges
    and into the overflow spectrum)."""
    params = params or eval_params()
    rng = np.random.default_rng(seed)
    pole = ecl_dir(30.0, 60.0)
    omega = 2 * math.pi / 0.25
    to_earth = ecl_dir(0.0, 10.0)
    oe = observer_matrix(to_earth)
    w_obs = oe @ (omega * pole)
    w_proj = math.hypot(w_obs[0], w_obs[1])
    Ftx = 2380.0
    dset = cd.DopplerSet()
    dset.Ftx, dset.dopscale = Ftx, 1.0
    dset.law = law if law is not None else radar_cosine()
    ndops = rng.integers(ndop_range[0], ndop_range[1] + 1, nframes)
    sides = rng.integers(pos_range[0], pos_range[1] + 1, nframes) | 1
    phases = rng.uniform(0.0, 2 * math.pi, nframes)
    dset.dop_per_bin = 2 * KM2HZFACT * Ftx * w_proj * radius / (span * float(ndop_range[0]))
    frames = []
    for f in range(nframes):
        fr = cd.DopplerFrame()
        fr.pos_n = int(sides[f]) // 2
        fr.km_per_pixel = 2 * radius / (0.8 * sides[f])
        cd.fill9(fr.ae, body_matrix(pole, float(phases[f])))
        cd.fill9(fr.oe, oe)
        for j in range(3):
            fr.spin[j] = float(omega * pole[j])
        fr.dopoff = 0.0
        fr.ndop = int(ndops[f])
        fr.dopcom_vig = 0.5 * fr.ndop + 0.5
        fr.weight = 1.0
        fr.dof = float(fr.ndop)
        fr.cal_floating, fr.cal = 1, 1.0
        fr.sdev = sdev
        frames.append(fr)
    sizes = [fr.ndop for fr in frames]
    offsets = np.zeros(nframes + 1, dtype=np.int64)
    np.cumsum(sizes, out=offsets[1:])
    obs = np.zeros(int(offsets[-1]))
    oov = np.full(int(offsets[-1]), 1.0 / (sdev * sdev))
    ds = DopplerDataset(dset, frames, obs, oov, offsets)
    if synthesize is not None:
        fits = synthesize(ds, params)
        nrng = np.random.default_rng(seed + 1000)
        for f in range(nframes):
            ft = np.asarray(fits[f], dtype=np.float64)
            peak = ft.max() if ft.size and ft.max() > 0 else 1.0
            ds.obs[offsets[f]:offsets[f + 1]] = 20.0 * ft / peak + sdev * nrng.standard_normal(ft.size)
    return ds


def lightcurve_dataset(npoints=200, pos_range=(129, 257), synthesize=None, params=None,
                       seed=7, set_index=0, radius=1.05, law_type=11, obs_between=False):
    """Config 3: one lightcurve of `npoints` points, solar phase uniform in
    5-60 deg, odd POS sides uniform in pos_range, Kaasalainen law with
    wt=0.3 (Lommel-Seeliger 0.7 + Lambert 0.3), A0=0, k=0; calc epochs equal
    observation epochs; 1% Gaussian noise.

    obs_between: the npoints epochs are the calculated ones only, and the
    npoints - 1 observation epochs lie strictly between consecutive calc
    epochs (at 20-80 % of each gap), so every fit value is the natural
    spline of the calculated brightnesses evaluated off its knots
    (src/shape/calc_fits.c:1923-1933); the observed values are the
    synthesized brightnesses interpolated linearly to those epochs, with the
    same 1% noise."""
    params = params or eval_params()
    rng = np.random.default_rng(seed + 101 * set_index)
    pole = ecl_dir(30.0, 60.0)
    to_earth = ecl_dir(20.0 * set_index, 5.0 + 3.0 * set_index)
    oe = observer_matrix(to_earth)
    alpha = float(rng.uniform(5.0, 60.0)) * DEG
    axis = np.cross(to_earth, [0.0, 0.0, 1.0])
    to_sun = rotate_about(to_earth, axis, alpha)
    se = observer_matrix(to_sun)
    t = np.sort(rng.uniform(0.0, 0.5, npoints)) + 2458000.0 + 10.0 * set_index
    sides = rng.integers(pos_range[0], pos_range[1] + 1, npoints) | 1
    pts = []
    for i in range(npoints):
        p = cd.LghtcrvPoint()
        p.pos_n = int(sides[i]) // 2
        p.km_per_pixel = 2 * radius / (0.8 * sides[i])
        phase = 2 * math.pi * (t[i] - t[0]) / 0.25
        cd.fill9(p.ae, body_matrix(pole, phase))
        cd.fill9(p.oe, oe)
        cd.fill9(p.se, se)
        p.solar_phase = alpha
        pts.append(p)
    x = t.copy()
    if obs_between:
        frac = np.random.default_rng(seed + 7 + 101 * set_index).uniform(0.2, 0.8, npoints - 1)
        t = x[:-1] + frac * (x[1:] - x[:-1])
    nobs = len(t)
    ls = cd.LghtcrvSet()
    ls.ncalc, ls.n = npoints, nobs
    ls.weight, ls.dof = 1.0, float(nobs)
    ls.cal_floating, ls.cal = 1, 1.0
    law = cd.OpticalLaw()
    law.type, law.R, law.wt, law.A0, law.D, law.k = law_type, 1.0, 0.3, 0.0, 0.1, 0.0
    ls.law = law
    obs = np.ones(nobs)
    ds = LightcurveDataset(ls, pts, x, t.copy(), obs, np.ones(nobs))
    if synthesize is not None:
        y = np.asarray(synthesize(ds, params), dtype=np.float64)
        if obs_between:
            y = np.interp(t, x, y)
        nrng = np.random.default_rng(1234 + set_index)
        ds.obs = y * (1.0 + 0.01 * nrng.standard_normal(nobs))
        ds.oneovervar = 1.0 / (0.01 * ds.obs) ** 2
    ds.bind()
    return ds


class PosetDataset:
    """A plane-of-sky set: frames (dicts of shape_poset_frame's fields; ae,
    oe, se as 3x3), the optical law, the resampling mode and rebinning, and
    the frames' observed images and 1/variance back to back (ncol x nrow,
    row index contiguous)."""

    def __init__(self, frames, law, resample, rebin, obs, oneovervar):
        self.frames, self.law, self.resample, self.rebin = frames, law, resample, rebin
        self.obs, self.oneovervar = obs, oneovervar
        sizes = [f["ncol"] * f["nrow"] for f in frames]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)

    @property
    def nframes(self):
        return len(self.frames)

    def bind(self):
        st = cd.PosetSet()
        st.law, st.resample, st.rebin = self.law, int(self.resample), int(self.rebin)
        arr = (cd.PosetFrame * len(self.frames))()
        for k, f in enumerate(self.frames):
            c = arr[k]
            for key, val in f.items():
                if key in ("ae", "oe", "se"):
                    cd.fill9(getattr(c, key), val)
                else:
                    setattr(c, key, val)
        return st, arr, np.ascontiguousarray(self.obs, dtype=np.float64), \
            np.ascontiguousarray(self.oneovervar, dtype=np.float64)


def poset_dataset(nframes=2, synthesize=None, params=None, pos_n=60, ncol=44, nrow=38, fit_scale=1.9,
                  resample=2, rebin=False, northangle=0.35, offsets=(1.3, -0.7), radius=1.0, seed=5,
                  law_type=3, northangle_step=0.2):
    """A plane-of-sky set of the config-1 body: sky renderings of (2 pos_n + 1)^2
    pixels spanning the body, resampled onto ncol x nrow fit images whose
    pixels are fit_scale rendering pixels wide, turned by the north angle
    and shifted by the COM offsets (fit-grid pixels); frame k's north angle
    is northangle + k northangle_step. Observed images: A *
    fit / max(fit) + N(0, 1) from synthesize(ds, params) (a list of fit
    images), or zeros."""
    rng = np.random.default_rng(seed)
    pole = ecl_dir(30.0, 60.0)
    frames = []
    for k in range(nframes):
        to_earth = ecl_dir(15.0 + 40.0 * k, 10.0 - 5.0 * k)
        alpha = float(rng.uniform(10.0, 50.0)) * DEG
        axis = np.cross(to_earth, [0.0, 0.0, 1.0])
        to_sun = rotate_about(to_earth, axis, alpha)
        kmpp = 2.2 * radius / (2 * pos_n + 1)
        frames.append({
            "pos_n": pos_n, "km_per_pixel": kmpp,
            "ae": body_matrix(pole, 0.9 * k), "oe": observer_matrix(to_earth), "se": observer_matrix(to_sun),
            "solar_phase": alpha, "ncol": ncol, "nrow": nrow, "fit_km_per_pixel": fit_scale * kmpp,
            "colcom_vig": (ncol + 1) / 2.0 + 0.25 * k, "rowcom_vig": (nrow + 1) / 2.0 - 0.4 * k,
            "xoff": float(offsets[0]), "yoff": float(offsets[1]), "northangle": northangle + northangle_step * k,
            "weight": 1.0, "dof": float(ncol * nrow),
        })
    law = cd.OpticalLaw()
    law.type, law.R, law.wt, law.A0, law.D, law.k = law_type, 1.0, 0.3, 0.0, 0.1, 0.0
    total = sum(f["ncol"] * f["nrow"] for f in frames)
    ds = PosetDataset(frames, law, resample, rebin, np.zeros(total), np.ones(total))
    if synthesize is not None:
        fits = synthesize(ds, params or eval_params())
        nrng = np.random.default_rng(1234 + seed)
        for k, fit in enumerate(fits):
            a, b = ds.offsets[k], ds.offsets[k + 1]
            f = np.asarray(fit, dtype=np.float64).ravel()
            ds.obs[a:b] = 20.0 * f / max(f.max(), 1e-300) + nrng.standard_normal(b - a)
    return ds


def config3_datasets(synthesize=None, params=None, npoints=200):
    return [lightcurve_dataset(npoints, (129, 257), synthesize, params, set_index=k) for k in range(4)]


# ------------------------------------------------------------- serving mix

def frame_prefix(ds, k):
    """The first k frames of a delay-Doppler dataset (observations shared)."""
    off = ds.offsets[:k + 1].copy()
    return DeldopDataset(ds.set, ds.frames[:k], ds.obs[:off[-1]], ds.oneovervar[:off[-1]], off)


def config1_frames(nframes=4, synthesize=None, params=None, pos_n=75):
    """Config-1 geometry (ellipsoid, 151x151 POS, 100x100 delay-Doppler) at
    nframes rotation phases 0.7 + 2*pi*j/nframes."""
    params = params or eval_params()
    one = config1_dataset(None, params, pos_n)
    pole = ecl_dir(30.0, 60.0)
    frames = []
    for j in range(nframes):
        fr = cd.DeldopFrame.from_buffer_copy(one.frames[0])
        cd.fill9(fr.ae, body_matrix(pole, 0.7 + 2 * math.pi * j / nframes))
        frames.append(fr)
    return _finish_deldop(one.set, frames, synthesize, 20.0, 1.0, 1234, params)


def serving_mix(synthesize_dd, synthesize_lc, params=None):
    """Workloads of the serving mix: the config-1 model with 1-4 frames,
    the config-2 model with 8-64 frames, the config-3 lightcurve sets (4 x
    200 points) and the config-4 model with 1-16 frames; one workload per
    frame count. Returns (categories, workloads) where workloads[i] =
    (category, model, deldop datasets, lightcurve datasets) and
    categories[c] lists the workload indices of category c (a request picks a
    category uniformly, then a workload of it uniformly)."""
    params = params or eval_params()
    m1, m2, m4 = ellipsoid_model(), harmonic_model(), noisy_octa_model()
    d1 = config1_frames(4, synthesize_dd(m1), params)
    d2 = config2_dataset(synthesize_dd(m2), params)
    d4 = config4_dataset(synthesize_dd(m4), params)
    lc = config3_datasets(synthesize_lc(m2), params)
    work, cats = [], [[], [], [], []]
    for k in range(1, 5):
        cats[0].append(len(work))
        work.append(("c1", m1, [frame_prefix(d1, k)], []))
    for k in range(8, 65):
        cats[1].append(len(work))
        work.append(("c2", m2, [frame_prefix(d2, k)], []))
    cats[2].append(len(work))
    work.append(("c3", m2, [], lc))
    for k in range(1, 17):
        cats[3].append(len(work))
        work.append(("c4", m4, [frame_prefix(d4, k)], []))
    return cats, work


def serving_trace(cats, nreq, rate_per_s, seed=0, scale_jitter=0.02):
    """Seeded Poisson request stream over the serving mix: exponential gaps
    of mean 1/rate, a category uniformly, then a workload of it uniformly,
    scale factors 1 +- scale_jitter."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, nreq))
    t -= t[0]
    out = []
    for i in range(nreq):
        c = cats[int(rng.integers(0, len(cats)))]
        w = c[int(rng.integers(0, len(c)))]
        sc = 1.0 + scale_jitter * rng.uniform(-1, 1, 3)
        out.append((w, float(t[i]), tuple(float(x) for x in sc)))
    return out
