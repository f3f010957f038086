// One plane-of-sky view per call, on images the caller keeps in host memory:
// the device forms of the reference's posvis, pos2deldop, posmask and
// apply_photo (src/shape/posvis.c:84-364, src/shape/pos2deldop.c:176-581,
// src/shape/posmask.c:58-174, src/shape/apply_photo.c:78-309) behind the
// C ABI of include/shape_b200.h (shape_posvis, shape_pos2deldop,
// shape_posmask, shape_apply_photo, shape_posclr).
//
// They serve callers that drive the plane of sky themselves (the write,
// view and map actions, multi-component and binary-system code): each call
// uploads what it reads, runs the engine's kernels on one view and copies
// back what it writes. FP64 throughout, compiled without FMA contraction:
// posvis uses the engine's transform, binning and FP64 tile raster in the
// raster's accumulate mode, so facet, depth and cos(e) maps are bit-exact
// with the reference's; pos2deldop evaluates each lit pixel's footprint
// with the raster's pos2deldop functions (fit to the reference's sum order
// within rounding).
//
// Each device has one context (stream, growable device buffers), guarded by
// a mutex: calls on one device run one at a time.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "engine_impl.h"
#include "kernels.h"
#include "posmask_dev.cuh"
#include "raster_impl.cuh"
#include "shape_b200.h"

namespace shape {
namespace posview {

constexpr int MAX_DEVICES = 64;

struct Buf {
    void *p = nullptr;
    size_t n = 0;
};

struct Ctx {
    bool ready = false;
    cudaStream_t s = nullptr;
    Buf vx, vn, fn, fvi, vt, geom, state, bin_count, bin_ids, work, z, ca, cb, f, won, laws, fit, zi, fi;
    int cap = 256;
};

static std::mutex g_mu;
static Ctx g_ctx[MAX_DEVICES];

#define PV_CK(call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return report_error(e_ == cudaErrorMemoryAllocation ? SHAPE_E_NOMEM : SHAPE_E_CUDA,       \
                                std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

static int grow(Buf &b, size_t bytes)
{
    if (bytes <= b.n) return SHAPE_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
    size_t want = bytes < 4096 ? 4096 : bytes + bytes / 4;
    PV_CK(cudaMalloc(&b.p, want));
    b.n = want;
    return SHAPE_OK;
}

// The device context of `device`, made current.
static int context(int device, Ctx **out)
{
    if (device < 0 || device >= MAX_DEVICES) return report_error(SHAPE_E_ARG, "pos view: bad device");
    PV_CK(cudaSetDevice(device));
    Ctx &c = g_ctx[device];
    if (!c.ready) {
        PV_CK(configure_raster_f64());
        PV_CK(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        c.ready = true;
    }
    *out = &c;
    return SHAPE_OK;
}

// Makes the call's device current and gives the caller's back afterwards.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

static size_t npix(const shape_pos_view *v) { return (size_t)(2 * v->n + 1) * (size_t)(2 * v->n + 1); }

static int check_view(const shape_pos_view *v, const char *who)
{
    if (!v || v->n < 0 || v->n > 32767 || !(v->km_per_pixel > 0.0))
        return report_error(SHAPE_E_ARG, std::string(who) + ": invalid plane-of-sky view");
    return SHAPE_OK;
}

// ------------------------------------------------------------------ posvis

// posbnd_logfactor from the view's extremes (src/shape/posvis.c:301-307):
// the won pixels and the facets wholly outside the frame.
static double host_logfactor(int n, const FrameState &st)
{
    double oimin = dkey_inv(st.ofr_ov[0]), oimax = dkey_inv(st.ofr_ov[1]);
    double ojmin = dkey_inv(st.ofr_ov[2]), ojmax = dkey_inv(st.ofr_ov[3]);
    if (st.cov_i[0] != INT_MAX) {
        oimin = std::min(oimin, (double)st.cov_i[0]);
        oimax = std::max(oimax, (double)st.cov_i[1]);
        ojmin = std::min(ojmin, (double)st.cov_j[0]);
        ojmax = std::max(ojmax, (double)st.cov_j[1]);
    }
    double xfactor = (std::max(oimax, (double)n) - std::min(oimin, (double)-n) + 1) / (2 * n + 1);
    double yfactor = (std::max(ojmax, (double)n) - std::min(ojmin, (double)-n) + 1) / (2 * n + 1);
    return log(xfactor * yfactor);
}

static int posvis_impl(int device, const shape_pos_view *view, shape_pos_images *img, int nv, const double *x,
                       const double *vn, int nf, const int *fv, const double *fn, const double orbit_offset[3],
                       int smooth, int src, int body, int comp)
{
    if (int rc = check_view(view, "posvis")) return rc;
    if (!img || nv < 3 || nf < 1 || !x || !fv || !fn || (smooth && !vn))
        return report_error(SHAPE_E_ARG, "posvis: invalid model arguments");
    for (int k = 0; k < 3 * nf; k++)
        if (fv[k] < 0 || fv[k] >= nv) return report_error(SHAPE_E_ARG, "posvis: facet vertex index out of range");
    double *Z = src ? img->zill : img->z;
    double *CA = src ? img->cosill : img->cose;
    double *CB = (!src && view->bistatic) ? img->cosi : nullptr;
    int *F = src ? img->fill : img->f;
    int *BOD = src ? img->bodyill : img->body;
    int *CMP = src ? img->compill : img->comp;
    int *xlim = src ? img->xlim2 : img->xlim;
    int *ylim = src ? img->ylim2 : img->ylim;
    if (!Z || !CA || !F || !BOD || !CMP || (!src && view->bistatic && !CB))
        return report_error(SHAPE_E_ARG, "posvis: missing plane-of-sky image");
    DeviceGuard dg;
    Ctx *c;
    if (int rc = context(device, &c)) return rc;
    cudaStream_t s = c->s;
    const int n = view->n, side = 2 * n + 1;
    const size_t P = npix(view);
    const int tiles_x = (side + TILE_W - 1) / TILE_W, ntiles = tiles_x * tiles_x;

    // the view: observer (or sun) <- body, the sun direction for a bistatic
    // observer view, and the orbit offset (src/shape/posvis.c:101-131, 159-166)
    FrameGeom g;
    memset(&g, 0, sizeof g);
    mul_bt(g.oa, src ? view->se : view->oe, view->ae);
    if (!src && view->bistatic) {
        double us[3] = {0.0, 0.0, 1.0};
        mtv(us, view->se, us);
        mv(us, view->oe, us);
        g.usrc[0] = us[0]; g.usrc[1] = us[1]; g.usrc[2] = us[2];
    }
    if (orbit_offset)
        for (int k = 0; k < 3; k++) g.off[k] = orbit_offset[k];
    g.kmpp = view->km_per_pixel;
    g.n = n;
    g.side = side;
    g.tiles_x = tiles_x;
    g.kind = src ? VIEW_LC_SUN : (view->bistatic ? VIEW_LC_OBS : VIEW_POS);
    g.wscale = 1.0;
    g.smooth = smooth ? 1 : 0;

    // model arrays in the engine's layout
    std::vector<double4> hx(nv), hvn(nv), hfn(nf);
    std::vector<int4> hfv(nf);
    for (int i = 0; i < nv; i++) {
        hx[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.0);
        hvn[i] = vn ? make_double4(vn[3 * i], vn[3 * i + 1], vn[3 * i + 2], 0.0) : make_double4(0, 0, 0, 0);
    }
    for (int f = 0; f < nf; f++) {
        hfn[f] = make_double4(fn[3 * f], fn[3 * f + 1], fn[3 * f + 2], 0.0);
        hfv[f] = make_int4(fv[3 * f], fv[3 * f + 1], fv[3 * f + 2], 0);
    }
    std::vector<int2> work(ntiles);
    for (int t = 0; t < ntiles; t++) work[t] = make_int2(0, t);
    int rc = grow(c->vx, sizeof(double4) * nv);
    if (!rc) rc = grow(c->vn, sizeof(double4) * nv);
    if (!rc) rc = grow(c->vt, sizeof(double4) * nv);
    if (!rc) rc = grow(c->fn, sizeof(double4) * nf);
    if (!rc) rc = grow(c->fvi, sizeof(int4) * nf);
    if (!rc) rc = grow(c->geom, sizeof(FrameGeom));
    if (!rc) rc = grow(c->state, sizeof(FrameState));
    if (!rc) rc = grow(c->bin_count, sizeof(int) * ntiles);
    if (!rc) rc = grow(c->work, sizeof(int2) * ntiles);
    if (!rc) rc = grow(c->z, sizeof(double) * P);
    if (!rc) rc = grow(c->ca, sizeof(double) * P);
    if (!rc) rc = grow(c->cb, sizeof(double) * P);
    if (!rc) rc = grow(c->f, sizeof(int) * P);
    if (!rc) rc = grow(c->won, P);
    if (rc) return rc;
    PV_CK(cudaMemcpyAsync(c->vx.p, hx.data(), sizeof(double4) * nv, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->vn.p, hvn.data(), sizeof(double4) * nv, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->fn.p, hfn.data(), sizeof(double4) * nf, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->fvi.p, hfv.data(), sizeof(int4) * nf, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->geom.p, &g, sizeof g, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->work.p, work.data(), sizeof(int2) * ntiles, cudaMemcpyHostToDevice, s));
    // the images' current contents: each pixel starts from them
    PV_CK(cudaMemcpyAsync(c->z.p, Z, sizeof(double) * P, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->ca.p, CA, sizeof(double) * P, cudaMemcpyHostToDevice, s));
    if (CB) PV_CK(cudaMemcpyAsync(c->cb.p, CB, sizeof(double) * P, cudaMemcpyHostToDevice, s));
    else PV_CK(cudaMemsetAsync(c->cb.p, 0, sizeof(double) * P, s));
    PV_CK(cudaMemcpyAsync(c->f.p, F, sizeof(int) * P, cudaMemcpyHostToDevice, s));

    ModelDev md;
    memset(&md, 0, sizeof md);
    md.nv = nv;
    md.nf = nf;
    md.vx = static_cast<double4 *>(c->vx.p);
    md.vn = static_cast<double4 *>(c->vn.p);
    md.fn = static_cast<double4 *>(c->fn.p);
    md.fvi = static_cast<int4 *>(c->fvi.p);
    const FrameGeom *dgeom = static_cast<const FrameGeom *>(c->geom.p);
    FrameState *dst = static_cast<FrameState *>(c->state.p);
    int *dcount = static_cast<int *>(c->bin_count.p);
    // bins sized from the previous call's fullest tile; a tile that still
    // overflows takes the raster's ordered full-scan path (same results)
    for (int pass = 0; pass < 2; pass++) {
        if (int r2 = grow(c->bin_ids, sizeof(int2) * (size_t)ntiles * c->cap)) return r2;
        launch_reset_state(dst, 1, dcount, ntiles, s);
        launch_xform_f64(dgeom, 1, md.vx, nv, static_cast<double4 *>(c->vt.p), s);
        launch_bin_f64(dgeom, 0, 1, md, static_cast<double4 *>(c->vt.p), dst, dcount,
                       static_cast<int2 *>(c->bin_ids.p), c->cap, s);
        std::vector<int> counts(ntiles);
        PV_CK(cudaMemcpyAsync(counts.data(), dcount, sizeof(int) * ntiles, cudaMemcpyDeviceToHost, s));
        PV_CK(cudaStreamSynchronize(s));
        int mx = 0;
        for (int v : counts) mx = std::max(mx, v);
        if (mx <= c->cap || pass == 1) break;
        while (c->cap < mx && c->cap < 8192) c->cap *= 2;
    }
    RasterArgs ra;
    memset(&ra, 0, sizeof ra);
    ra.geoms = dgeom;
    ra.work = static_cast<const int2 *>(c->work.p);
    ra.nwork = ntiles;
    ra.vt = c->vt.p;
    ra.fvi = md.fvi;
    ra.vn = md.vn;
    ra.fn = md.fn;
    ra.nf = nf;
    ra.bin_count = dcount;
    ra.bin_ids = static_cast<const int2 *>(c->bin_ids.p);
    ra.cap = c->cap;
    ra.states = dst;
    ra.pos_z = c->z.p;
    ra.pos_cose = c->ca.p;
    ra.pos_cosi = c->cb.p;
    ra.pos_f = static_cast<int *>(c->f.p);
    ra.keep_pos = 1;
    ra.accumulate = 1;
    ra.won = static_cast<unsigned char *>(c->won.p);
    launch_raster_f64(ra, s);
    PV_CK(cudaGetLastError());
    std::vector<unsigned char> won(P);
    FrameState st;
    PV_CK(cudaMemcpyAsync(Z, c->z.p, sizeof(double) * P, cudaMemcpyDeviceToHost, s));
    PV_CK(cudaMemcpyAsync(CA, c->ca.p, sizeof(double) * P, cudaMemcpyDeviceToHost, s));
    if (CB) PV_CK(cudaMemcpyAsync(CB, c->cb.p, sizeof(double) * P, cudaMemcpyDeviceToHost, s));
    PV_CK(cudaMemcpyAsync(F, c->f.p, sizeof(int) * P, cudaMemcpyDeviceToHost, s));
    PV_CK(cudaMemcpyAsync(won.data(), c->won.p, P, cudaMemcpyDeviceToHost, s));
    PV_CK(cudaMemcpyAsync(&st, dst, sizeof st, cudaMemcpyDeviceToHost, s));
    PV_CK(cudaStreamSynchronize(s));
    for (size_t p = 0; p < P; p++)
        if (won[p]) { BOD[p] = body; CMP[p] = comp; }
    // POSrect (src/shape/posvis.c:322-364): the won pixels and the facets
    // wholly outside the frame move the limits outward only
    if (st.cov_i[0] != INT_MAX) {
        xlim[0] = std::min(xlim[0], st.cov_i[0]); xlim[1] = std::max(xlim[1], st.cov_i[1]);
        ylim[0] = std::min(ylim[0], st.cov_j[0]); ylim[1] = std::max(ylim[1], st.cov_j[1]);
    }
    if (st.ofr_i[0] != INT_MAX) {
        xlim[0] = std::min(xlim[0], st.ofr_i[0]); xlim[1] = std::max(xlim[1], st.ofr_i[1]);
        ylim[0] = std::min(ylim[0], st.ofr_j[0]); ylim[1] = std::max(ylim[1], st.ofr_j[1]);
    }
    img->posbnd_logfactor = st.outbnd ? host_logfactor(n, st) : 0.0;
    return st.outbnd ? 1 : 0;
}

// -------------------------------------------------------------- pos2deldop

// The constants a lit pixel's footprint needs, plus the orbit offsets of
// pos2deldop's Doppler position (src/shape/pos2deldop.c:327).
struct P2dArgs {
    RasterArgs ra;               // laws (the one radar law), nothing else
    const FrameGeom *g;
    const double *z, *cose;
    const int *bodymap;
    int body;
    int n, side;
    int x0, y0, nx, ny;          // the limits' rectangle (pos->xlim, ylim)
    double xoff, yoff;
    double *fit;                 // ndel x ndop, added to
    FrameState *st;
};

// One thread per pixel of the limits' rectangle: a lit pixel of the body
// (cos(e) > 0, depth set) adds its footprint to the fit image (in-frame
// footprints only) and moves the frame's bin and position limits
// (src/shape/pos2deldop.c:305-496).
__global__ void k_pos2deldop(P2dArgs a)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)a.nx * a.ny) return;
    const int xi = a.x0 + (int)(k / a.ny), yj = a.y0 + (int)(k % a.ny);
    const long long p = (long long)(xi + a.n) * a.side + (yj + a.n);
    const double cose = a.cose[p], z = a.z[p];
    if (!(cose > 0.0 && a.bodymap[p] == a.body && z != -1e20)) return;
    const FrameGeom &g = *a.g;
    const DDC<double> kc = load_ddc<double>(g);
    PixPos pp;
    PixDD<double> d = pixel_dd_setup<double>(g, kc, xi, yj, z, pp);
    if (a.xoff != 0.0 || a.yoff != 0.0) {
        // Doppler position with the binary-orbit offsets (x - xoff, y - yoff)
        d.dopPOS = kc.ax * ((double)xi - a.xoff) + kc.ay * ((double)yj - a.yoff) + kc.dopshift;
        d.idop_min = (int)floor(d.dopPOS - kc.dopdiff_max + 1 - kc.half_w);
        d.idop_max = (int)floor(d.dopPOS + kc.dopdiff_max + kc.half_w);
        d.codefactor = ((g.codemethod == SHAPE_CODE_SHORT) ? sinc2<double>((d.dopPOS - kc.dopDC_vig) / kc.dopfftlen)
                                                           : 1.0) * g.wscale;
        pp.dop = d.dopPOS;
        d.ok = (d.idel_min >= 1) && (d.idel_max <= g.ndel) && (d.idop_min >= 1) && (d.idop_max <= g.ndop) &&
               (d.idel_max - d.idel_min + 1 <= SHAPE_MAXBINS);
    }
    FrameState &S = *a.st;
    atomicMin(&S.idellim[0], d.idel_min);
    atomicMax(&S.idellim[1], d.idel_max);
    atomicMin(&S.idoplim[0], d.idop_min);
    atomicMax(&S.idoplim[1], d.idop_max);
    atomicMin(&S.dellim[0], dkey(pp.del));
    atomicMax(&S.dellim[1], dkey(pp.del));
    atomicMin(&S.doplim[0], dkey(pp.dop));
    atomicMax(&S.doplim[1], dkey(pp.dop));
    S.any_lit = 1;
    if (d.ok) pixel_dd_scatter<double>(a.ra, g, kc, cose, d, a.fit, 1, 1, g.ndop);
}

static int pos2deldop_impl(int device, const shape_pos_view *view, const shape_pos_images *img,
                           const shape_eval_params *par, const shape_deldop_set *set, const shape_deldop_frame *frame,
                           double orbit_xoff, double orbit_yoff, double orbit_dopoff, int body, double *fit,
                           shape_deldop_result *res, double *km2Hz)
{
    if (int rc = check_view(view, "pos2deldop")) return rc;
    if (!img || !img->z || !img->cose || !img->body || !par || !set || !frame || !fit || !res)
        return report_error(SHAPE_E_ARG, "pos2deldop: null argument");
    if (frame->ndel < 1 || frame->ndop < 1 || set->spb < 1 || set->stride < 1 || set->spb / set->stride < 1 ||
        par->nsinc2 < 1)
        return report_error(SHAPE_E_ARG, "pos2deldop: invalid frame or set");
    if (set->law.type < SHAPE_RADLAW_COSINE_DIFF || set->law.type > SHAPE_RADLAW_COSINE_COSINE)
        return report_error(SHAPE_E_UNSUPPORTED, "pos2deldop: radar scattering law not supported");
    DeviceGuard dg;
    Ctx *c;
    if (int rc = context(device, &c)) return rc;
    cudaStream_t s = c->s;
    const int n = view->n, side = 2 * n + 1;
    const size_t P = npix(view), D = (size_t)frame->ndel * frame->ndop;

    // the frame's constants (src/shape/pos2deldop.c:201-275); the view's
    // km_per_pixel is the POS frame's
    FrameGeom g;
    memset(&g, 0, sizeof g);
    g.kind = VIEW_RADAR;
    g.wscale = 1.0;
    g.n = n;
    g.side = side;
    g.kmpp = view->km_per_pixel;
    g.ndel = frame->ndel;
    g.ndop = frame->ndop;
    radar_set_consts(g, *set, *par, 0, 0);
    shape_deldop_frame F = *frame;
    F.km_per_pixel = view->km_per_pixel;
    FrameHost h;
    memset(&h, 0, sizeof h);
    double dop_extra;
    radar_view_geom(g, h, dop_extra, F, *set);
    g.dopshift = F.dopcom_vig + F.dopoff + orbit_dopoff;
    if (km2Hz) *km2Hz = sqrt(g.ax * g.ax + g.ay * g.ay) * set->dop_per_pixel / view->km_per_pixel;
    RadarLawDev law{set->law.type, set->law.diff_R, set->law.diff_C, set->law.qs_R, set->law.qs_C,
                    set->law.qs_cos_cutoff, 2 * set->law.diff_C - 1 == 1.0, 2 * set->law.qs_C - 1 == 1.0};

    const int x0 = std::max(img->xlim[0], -n), x1 = std::min(img->xlim[1], n);
    const int y0 = std::max(img->ylim[0], -n), y1 = std::min(img->ylim[1], n);
    FrameState st0;
    memset(&st0, 0, sizeof st0);
    st0.idellim[0] = frame->ndel + 999999; st0.idellim[1] = -999999;
    st0.idoplim[0] = frame->ndop + 999999; st0.idoplim[1] = -999999;
    st0.dellim[0] = dkey(SHAPE_HUGENUMBER); st0.dellim[1] = dkey(-SHAPE_HUGENUMBER);
    st0.doplim[0] = dkey(SHAPE_HUGENUMBER); st0.doplim[1] = dkey(-SHAPE_HUGENUMBER);
    int rc = grow(c->geom, sizeof(FrameGeom));
    if (!rc) rc = grow(c->state, sizeof(FrameState));
    if (!rc) rc = grow(c->laws, sizeof(RadarLawDev));
    if (!rc) rc = grow(c->z, sizeof(double) * P);
    if (!rc) rc = grow(c->ca, sizeof(double) * P);
    if (!rc) rc = grow(c->f, sizeof(int) * P);
    if (!rc) rc = grow(c->fit, sizeof(double) * D);
    if (rc) return rc;
    PV_CK(cudaMemcpyAsync(c->geom.p, &g, sizeof g, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->state.p, &st0, sizeof st0, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->laws.p, &law, sizeof law, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->z.p, img->z, sizeof(double) * P, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->ca.p, img->cose, sizeof(double) * P, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->f.p, img->body, sizeof(int) * P, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->fit.p, fit, sizeof(double) * D, cudaMemcpyHostToDevice, s));
    if (x1 >= x0 && y1 >= y0) {
        P2dArgs a;
        memset(&a, 0, sizeof a);
        a.ra.laws = static_cast<const RadarLawDev *>(c->laws.p);
        a.g = static_cast<const FrameGeom *>(c->geom.p);
        a.z = static_cast<const double *>(c->z.p);
        a.cose = static_cast<const double *>(c->ca.p);
        a.bodymap = static_cast<const int *>(c->f.p);
        a.body = body;
        a.n = n;
        a.side = side;
        a.x0 = x0; a.y0 = y0; a.nx = x1 - x0 + 1; a.ny = y1 - y0 + 1;
        a.xoff = orbit_xoff;
        a.yoff = orbit_yoff;
        a.fit = static_cast<double *>(c->fit.p);
        a.st = static_cast<FrameState *>(c->state.p);
        const long long cnt = (long long)a.nx * a.ny;
        k_pos2deldop<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(a);
        PV_CK(cudaGetLastError());
    }
    FrameState st;
    PV_CK(cudaMemcpyAsync(fit, c->fit.p, sizeof(double) * D, cudaMemcpyDeviceToHost, s));
    PV_CK(cudaMemcpyAsync(&st, c->state.p, sizeof st, cudaMemcpyDeviceToHost, s));
    PV_CK(cudaStreamSynchronize(s));
    res->idellim[0] = st.idellim[0]; res->idellim[1] = st.idellim[1];
    res->idoplim[0] = st.idoplim[0]; res->idoplim[1] = st.idoplim[1];
    // delay and Doppler limits in usec and Hz, the Doppler ones widened by
    // the pixel's extent (src/shape/pos2deldop.c:503-510)
    res->dellim[0] = (dkey_inv(st.dellim[0]) - g.delshift) * set->del_per_pixel;
    res->dellim[1] = (dkey_inv(st.dellim[1]) - g.delshift) * set->del_per_pixel;
    res->doplim[0] = (dkey_inv(st.doplim[0]) - g.dopshift) * set->dop_per_pixel - dop_extra;
    res->doplim[1] = (dkey_inv(st.doplim[1]) - g.dopshift) * set->dop_per_pixel + dop_extra;
    res->badradar = h.badradar;
    res->badradar_logfactor = h.badradar_logfactor;
    return h.badradar;
}

// ----------------------------------------------------------------- posmask

struct MaskArgs {
    double so[9];                // sun <- observer: se oe^T
    double ppkm, kmpp, tol;
    int n, side;
    const double *z, *zill;
    const int *f, *comp, *body, *fill, *compill, *bodyill;
    double *cose;
};

// posmask per observer pixel (src/shape/posmask.c:58-174): a pixel whose
// point is farther from the sun than the sun view's surface there (by more
// than tol), where the sun view sees another facet, component or body, is
// in shadow and its cos(e) becomes 0.
__global__ void k_posmask(MaskArgs a)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)a.side * a.side) return;
    if (a.cose[p] == 0.0) return;
    const int n = a.n, side = a.side;
    const int i = (int)(p / side) - n, j = (int)(p % side) - n;
    const double xin[3] = {i * a.kmpp, j * a.kmpp, a.z[p]};
    double x[3];
    for (int r = 0; r < 3; r++) {
        x[r] = 0.0;
        x[r] += a.so[3 * r + 0] * xin[0];
        x[r] += a.so[3 * r + 1] * xin[1];
        x[r] += a.so[3 * r + 2] * xin[2];
    }
    const double i0 = x[0] * a.ppkm, j0 = x[1] * a.ppkm;
    const int im = iround_(i0), jm = iround_(j0);
    if (!(fabs(i0) < n && fabs(j0) < n)) return;
    const long long q = (long long)(im + n) * side + (jm + n);
    if (!(a.zill[q] > -0.99 * SHAPE_HUGENUMBER)) return;
    if (a.f[p] == a.fill[q] && a.comp[p] == a.compill[q] && a.body[p] == a.bodyill[q]) return;
    if (posmask_zill(a.zill, n, side, i0, j0, im, jm) - x[2] > a.tol) a.cose[p] = 0.0;
}

static int posmask_impl(int device, const shape_pos_view *view, shape_pos_images *img, double tol)
{
    if (int rc = check_view(view, "posmask")) return rc;
    if (!img || !img->z || !img->zill || !img->cose || !img->f || !img->fill || !img->comp || !img->compill ||
        !img->body || !img->bodyill)
        return report_error(SHAPE_E_ARG, "posmask: missing plane-of-sky image");
    DeviceGuard dg;
    Ctx *c;
    if (int rc = context(device, &c)) return rc;
    cudaStream_t s = c->s;
    const size_t P = npix(view);
    MaskArgs a;
    memset(&a, 0, sizeof a);
    mul_bt(a.so, view->se, view->oe);
    a.ppkm = 1 / view->km_per_pixel;
    a.kmpp = view->km_per_pixel;
    a.tol = tol;
    a.n = view->n;
    a.side = 2 * view->n + 1;
    // one device buffer for the six facet / component / body maps
    int rc = grow(c->z, sizeof(double) * P);
    if (!rc) rc = grow(c->zi, sizeof(double) * P);
    if (!rc) rc = grow(c->ca, sizeof(double) * P);
    if (!rc) rc = grow(c->fi, sizeof(int) * 6 * P);
    if (rc) return rc;
    int *m = static_cast<int *>(c->fi.p);
    const int *src[6] = {img->f, img->comp, img->body, img->fill, img->compill, img->bodyill};
    for (int k = 0; k < 6; k++)
        PV_CK(cudaMemcpyAsync(m + k * P, src[k], sizeof(int) * P, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->z.p, img->z, sizeof(double) * P, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->zi.p, img->zill, sizeof(double) * P, cudaMemcpyHostToDevice, s));
    PV_CK(cudaMemcpyAsync(c->ca.p, img->cose, sizeof(double) * P, cudaMemcpyHostToDevice, s));
    a.z = static_cast<const double *>(c->z.p);
    a.zill = static_cast<const double *>(c->zi.p);
    a.cose = static_cast<double *>(c->ca.p);
    a.f = m; a.comp = m + P; a.body = m + 2 * P; a.fill = m + 3 * P; a.compill = m + 4 * P; a.bodyill = m + 5 * P;
    k_posmask<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(a);
    PV_CK(cudaGetLastError());
    PV_CK(cudaMemcpyAsync(img->cose, c->ca.p, sizeof(double) * P, cudaMemcpyDeviceToHost, s));
    PV_CK(cudaStreamSynchronize(s));
    return SHAPE_OK;
}

// ------------------------------------------------------------- apply_photo

struct PhotoArgs {
    int law;                     // SHAPE_OPTLAW_*
    double scale, s_ls, s_l, intensity;
    int n, side, x0, y0, nx, ny, body;
    const double *cose, *cosi;
    const int *bodymap;
    double *b;
};

// Brightness of every lit pixel of the body in the limits' rectangle
// (src/shape/apply_photo.c:85-133, 226-248), one thread per pixel. The
// total is then added on the host pixel by pixel in (i, j) order, the
// reference's order, so it is the reference's sum.
__global__ void k_apply_photo(PhotoArgs a)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)a.nx * a.ny) return;
    const int xi = a.x0 + (int)(k / a.ny), yj = a.y0 + (int)(k % a.ny);
    const long long p = (long long)(xi + a.n) * a.side + (yj + a.n);
    const double ce = a.cose[p], ci = a.cosi[p];
    if (ce > 0.0 && ci > 0.0 && a.bodymap[p] == a.body) {
        double b;
        if (a.law == SHAPE_OPTLAW_LAMBERT) b = a.intensity * a.scale * ci;
        else if (a.law == SHAPE_OPTLAW_LOMMEL) b = a.intensity * a.scale * ci / (ci + ce);
        else b = a.intensity * ci * (a.s_ls / (ci + ce) + a.s_l);
        a.b[p] = b;
    }
}

static int apply_photo_impl(int device, const shape_optical_law *law, double phase, double intensityfactor,
                            const shape_pos_view *view, shape_pos_images *img, int body, double *sum)
{
    if (int rc = check_view(view, "apply_photo")) return rc;
    if (!law || !img || !img->cose || !img->cosi || !img->body || !img->b || !sum)
        return report_error(SHAPE_E_ARG, "apply_photo: null argument");
    PhotoArgs a;
    memset(&a, 0, sizeof a);
    a.law = law->type;
    switch (law->type) {
    case SHAPE_OPTLAW_LAMBERT: a.scale = law->R / SHAPE_PIE; break;
    case SHAPE_OPTLAW_LOMMEL: a.scale = law->R / (4 * SHAPE_PIE); break;
    case SHAPE_OPTLAW_KAASALAINEN: {
        const double phasefunc = law->A0 * exp(-phase / law->D) + law->k * phase + 1;
        a.s_ls = (1 - law->wt) * phasefunc * law->R / (4 * SHAPE_PIE);
        a.s_l = law->wt * phasefunc * law->R / SHAPE_PIE;
        break;
    }
    default:
        return report_error(SHAPE_E_UNSUPPORTED, "apply_photo: optical scattering law not supported");
    }
    a.intensity = intensityfactor;
    const int n = view->n;
    const int x0 = std::max(img->xlim[0], -n), x1 = std::min(img->xlim[1], n);
    const int y0 = std::max(img->ylim[0], -n), y1 = std::min(img->ylim[1], n);
    double total = 0.0;
    if (x1 >= x0 && y1 >= y0) {
        DeviceGuard dg;
        Ctx *c;
        if (int rc = context(device, &c)) return rc;
        cudaStream_t s = c->s;
        const size_t P = npix(view);
        int rc = grow(c->z, sizeof(double) * P);
        if (!rc) rc = grow(c->ca, sizeof(double) * P);
        if (!rc) rc = grow(c->cb, sizeof(double) * P);
        if (!rc) rc = grow(c->f, sizeof(int) * P);
        if (rc) return rc;
        PV_CK(cudaMemcpyAsync(c->ca.p, img->cose, sizeof(double) * P, cudaMemcpyHostToDevice, s));
        PV_CK(cudaMemcpyAsync(c->cb.p, img->cosi, sizeof(double) * P, cudaMemcpyHostToDevice, s));
        PV_CK(cudaMemcpyAsync(c->f.p, img->body, sizeof(int) * P, cudaMemcpyHostToDevice, s));
        PV_CK(cudaMemcpyAsync(c->z.p, img->b, sizeof(double) * P, cudaMemcpyHostToDevice, s));
        a.n = n;
        a.side = 2 * n + 1;
        a.x0 = x0; a.y0 = y0; a.nx = x1 - x0 + 1; a.ny = y1 - y0 + 1;
        a.body = body;
        a.cose = static_cast<const double *>(c->ca.p);
        a.cosi = static_cast<const double *>(c->cb.p);
        a.bodymap = static_cast<const int *>(c->f.p);
        a.b = static_cast<double *>(c->z.p);
        const long long cnt = (long long)a.nx * a.ny;
        k_apply_photo<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(a);
        PV_CK(cudaGetLastError());
        PV_CK(cudaMemcpyAsync(img->b, c->z.p, sizeof(double) * P, cudaMemcpyDeviceToHost, s));
        PV_CK(cudaStreamSynchronize(s));
        // the reference's running sum, pixel by pixel in (i, j) order
        for (int r = 0; r < a.nx; r++) {
            const int xi = x0 + r;
            for (int cc = 0; cc < a.ny; cc++) {
                const size_t p = (size_t)(xi + n) * (2 * n + 1) + (size_t)(y0 + cc + n);
                if (img->cose[p] > 0.0 && img->cosi[p] > 0.0 && img->body[p] == body) total += img->b[p];
            }
        }
    }
    *sum = (total == 0.0) ? 1.0e-40 : total;     // TINY, src/shape/apply_photo.c:76, 305-306
    return SHAPE_OK;
}

}  // namespace posview
}  // namespace shape

using namespace shape::posview;

extern "C" {

int shape_posvis(int device, const shape_pos_view *view, shape_pos_images *img, int nv, const double *x,
                 const double *vn, int nf, const int *fv, const double *fn, const double orbit_offset[3],
                 int smooth, int src, int body, int comp)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return posvis_impl(device, view, img, nv, x, vn, nf, fv, fn, orbit_offset, smooth, src, body, comp);
}

int shape_pos2deldop(int device, const shape_pos_view *view, const shape_pos_images *img,
                     const shape_eval_params *par, const shape_deldop_set *set, const shape_deldop_frame *frame,
                     double orbit_xoff, double orbit_yoff, double orbit_dopoff, int body, double *fit,
                     shape_deldop_result *res, double *km2Hz)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return pos2deldop_impl(device, view, img, par, set, frame, orbit_xoff, orbit_yoff, orbit_dopoff, body, fit, res,
                           km2Hz);
}

int shape_posmask(int device, const shape_pos_view *view, shape_pos_images *img, double tol)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return posmask_impl(device, view, img, tol);
}

int shape_apply_photo(int device, const shape_optical_law *law, double phase, double intensityfactor,
                      const shape_pos_view *view, shape_pos_images *img, int body, double *sum)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return apply_photo_impl(device, law, phase, intensityfactor, view, img, body, sum);
}

int shape_posclr(const shape_pos_view *view, shape_pos_images *img)
{
    if (int rc = check_view(view, "posclr")) return rc;
    if (!img) return shape::report_error(SHAPE_E_ARG, "posclr: null argument");
    const size_t P = npix(view);
    const int n = view->n;
    // src/shape/posclr.c:24-67
    for (size_t p = 0; p < P; p++) {
        if (img->b) img->b[p] = 0.0;
        if (img->cose) img->cose[p] = 0.0;
        if (img->cosi) img->cosi[p] = 0.0;
        if (img->z) img->z[p] = -SHAPE_HUGENUMBER;
        if (img->body) img->body[p] = -1;
        if (img->comp) img->comp[p] = -1;
        if (img->f) img->f[p] = -1;
    }
    img->xlim[0] = img->ylim[0] = n;
    img->xlim[1] = img->ylim[1] = -n;
    if (view->bistatic) {
        for (size_t p = 0; p < P; p++) {
            if (img->cosill) img->cosill[p] = 0.0;
            if (img->zill) img->zill[p] = -SHAPE_HUGENUMBER;
            if (img->bodyill) img->bodyill[p] = -1;
            if (img->compill) img->compill[p] = -1;
            if (img->fill) img->fill[p] = -1;
        }
        img->xlim2[0] = img->ylim2[0] = n;
        img->xlim2[1] = img->ylim2[1] = -n;
    }
    return SHAPE_OK;
}

}  // extern "C"
