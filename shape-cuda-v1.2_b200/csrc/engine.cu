// Host side of the SHAPE B200 engine and its C ABI (include/shape_b200.h).
//
// Per-frame constants of posvis / pos2deldop / posmask / apply_photo are
// computed here in FP64 with the reference's operation order (this file is
// compiled with -ffp-contract=off for the host compiler), uploaded once, and
// reused by every evaluation. An evaluation copies the free model parameters
// (vertex deviations and scale factors) host->device, runs the kernel
// sequence on the engine stream and copies the summary device->host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "engine_impl.h"
#include "spin_impl.cuh"
#include "kernels.h"
#include "shape_b200.h"

namespace shape {

static thread_local std::string g_err;

static int set_err(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

// Shared with other translation units of the library (noalloc.cu).
int report_error(int code, const std::string &msg) { return set_err(code, msg); }

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return set_err(e_ == cudaErrorMemoryAllocation ? SHAPE_E_NOMEM : SHAPE_E_CUDA, \
                           std::string(#call) + ": " + cudaGetErrorString(e_));            \
    } while (0)

static int radar_law_index(EngineImpl &E, const shape_radar_law &L)
{
    if (L.type < SHAPE_RADLAW_COSINE_DIFF || L.type > SHAPE_RADLAW_COSINE_COSINE) return -1;
    RadarLawDev d{L.type, L.diff_R, L.diff_C, L.qs_R, L.qs_C, L.qs_cos_cutoff,
                  2 * L.diff_C - 1 == 1.0, 2 * L.qs_C - 1 == 1.0};
    E.laws.push_back(d);
    return (int)E.laws.size() - 1;
}

// Set-level constants of pos2deldop for a radar view
// (src/shape/pos2deldop.c:201-240): the code method's delay response
// extents, the delay scale, the sinc^2 sampling and the law index. A Doppler
// frame is a single row: delPOS = z*0 + 1 = 1 exactly, so its delay response
// tri2(0) is 1 and its weights are pos2doppler's.
void radar_set_consts(FrameGeom &g, const shape_deldop_set &S, const shape_eval_params &P, int law, int doppler)
{
    g.codemethod = S.codemethod;
    g.spb = S.spb;
    g.stride = S.stride;
    g.spb_over_stride = S.spb / S.stride;
    g.one_over_spb = 1.0 / S.spb;
    g.spb_sq = S.spb * S.spb;
    if (S.codemethod != SHAPE_CODE_LONG_ORIG) {
        g.const1 = (3 * S.spb - 1) / (2.0 * S.stride);
        g.const2 = (S.spb - 1) / (2.0 * S.stride);
    } else {
        g.const1 = (double)g.spb_over_stride;
        g.const2 = 0.0;
    }
    g.delfact = doppler ? 0.0 : -SHAPE_KM2US / S.del_per_pixel;
    g.nsinc2 = P.nsinc2;
    g.nsinc2_sq = P.nsinc2 * P.nsinc2;
    g.sinc2width = P.sinc2width;
    g.dopfftlen = S.dopfftlen;
    g.law = law;
}

int EngineImpl::finalize()
{
    if (!have_model) return set_err(SHAPE_E_STATE, "finalize: no model set");
    if (dd.empty() && lc.empty() && ps.empty()) return set_err(SHAPE_E_STATE, "finalize: no datasets");
    mem.release();
    invalidate_graphs();
    for (int f = 0; f < 3; f++) tuned[f] = 0;
    d_work_sorted = nullptr;
    d_sides = nullptr; d_msum_part = d_msum = nullptr;
    d_side_v2 = nullptr; d_comp_facets = nullptr; d_act_v = d_act_f = nullptr; d_surf_err = nullptr;
    cap = fixed_cap > 0 ? fixed_cap : 512;
    geoms.clear(); fh.clear(); work.clear(); view_work0.clear(); view_nwork.clear();
    chi2_items.clear(); frame_view.clear(); dop_extra.clear(); set_delpp.clear(); set_doppp.clear();
    lcpts.clear(); lc_items.clear(); pt_items.clear(); lcdev.clear(); dop_frames.clear();

    const int nframes = (int)frames.size();
    const int npts = (int)points.size();
    nviews = 2 * npts + 2 * nps_frames;      // lightcurve points and plane-of-sky frames: two views each
    for (int fi = 0; fi < nframes; fi++) nviews += fviews[fi].empty() ? 1 : (int)fviews[fi].size();
    int tile_base = 0;
    long long pos_base = 0;
    auto add_view = [&](FrameGeom &g, int n, double kmpp) {
        g.n = n;
        g.side = 2 * n + 1;
        g.kmpp = kmpp;
        g.tiles_x = (g.side + TILE_W - 1) / TILE_W;
        g.tile_base = tile_base;
        g.vt_base = (int)geoms.size() * nv;
        g.pos_base = pos_base;
        view_work0.push_back((int)work.size());
        view_nwork.push_back(g.tiles_x * g.tiles_x);
        for (int t = 0; t < g.tiles_x * g.tiles_x; t++) work.push_back(make_int2((int)geoms.size(), t));
        tile_base += g.tiles_x * g.tiles_x;
        pos_base += (long long)g.side * g.side;
        view_float_consts(g);
        geoms.push_back(g);
    };

    // delay-Doppler frames: constants of pos2deldop (src/shape/pos2deldop.c:201-275)
    laws.clear();
    for (size_t s = 0; s < dd.size(); s++) {
        const shape_deldop_set &S = dd[s].set;
        set_delpp.push_back(S.del_per_pixel);
        set_doppp.push_back(S.dop_per_pixel);
        int law = radar_law_index(*this, S.law);
        if (law < 0) return set_err(SHAPE_E_UNSUPPORTED, "radar scattering law not supported");
        if (S.spb < 1 || S.stride < 1 || S.spb / S.stride < 1)
            return set_err(SHAPE_E_ARG, "deldop set: spb/stride must be >= 1");
        for (int k = 0; k < dd[s].nframes; k++) {
            int fi = dd[s].frame0 + k;
            const shape_deldop_frame &F = frames[fi];
            FrameGeom g;
            memset(&g, 0, sizeof g);
            g.kind = VIEW_RADAR;
            g.smooth = params.pos_smooth;
            g.ndel = F.ndel;
            g.ndop = F.ndop;
            g.fit_base = frame_off[fi];
            radar_set_consts(g, S, params, law, dd[s].doppler);
            g.frame_index = fi;
            g.dop1d = dd[s].doppler;
            if (g.dop1d) g.ovf_base = (long long)dop_frames.size() * DOP_MAXOVERFLOW;
            FrameHost h;
            memset(&h, 0, sizeof h);
            h.weight = F.weight;
            h.dof = F.dof;
            h.cal_in = F.cal;
            h.cal_floating = F.cal_floating;
            // a smeared frame's views in the reference's order, its epoch
            // view last (src/shape/calc_fits.c:489-490): each rasterized
            // into the same fit image at 1/views of its cross-section; the
            // frame's limits, posbnd and seen marks are the epoch view's
            const std::vector<shape_deldop_frame> &V = fviews[fi];
            const int nview = V.empty() ? 1 : (int)V.size();
            h.nviews = nview;
            for (int k2 = 0; k2 + 1 < nview; k2++) {
                FrameGeom gv = g;
                FrameHost hv = h;
                double dxv;
                radar_view_geom(gv, hv, dxv, V[k2], S);
                gv.wscale = 1.0 / nview;
                gv.no_seen = 1;
                if (hv.badradar) {
                    h.badradar_any = 1;
                    h.badradar_lfsum += hv.badradar_logfactor;
                }
                add_view(gv, F.pos_n, F.km_per_pixel);
            }
            double dx;
            radar_view_geom(g, h, dx, F, S);
            g.wscale = 1.0 / nview;
            if (h.badradar) {
                h.badradar_any = 1;
                h.badradar_lfsum += h.badradar_logfactor;
            }
            dop_extra.push_back(dx);
            h.view = (int)geoms.size();
            h.set = (int)s;
            h.dop_index = g.dop1d ? (int)dop_frames.size() : -1;
            h.sdev = frame_sdev[fi];
            if (g.dop1d) dop_frames.push_back(fi);
            frame_view.push_back(h.view);
            h.item0 = (int)chi2_items.size();
            int D = F.ndel * F.ndop, chunk = CHI2_ITEM;
            for (int st = 0; st < D; st += chunk)
                chi2_items.push_back(Chi2Item{fi, st, std::min(chunk, D - st)});
            h.nitems = (int)chi2_items.size() - h.item0;
            fh.push_back(h);
            add_view(g, F.pos_n, F.km_per_pixel);
        }
    }
    {
        // the fused chi-square / summary kernel needs every frame to own an
        // item and its staging buffer to hold a frame's partials and the
        // per-frame terms
        int max_items = 0;
        bool every = true;
        for (const FrameHost &h : fh) { max_items = std::max(max_items, h.nitems); every = every && h.nitems > 0; }
        fused_chi2 = every && !chi2_items.empty() && chi2_summary_fits((int)fh.size(), max_items);
        fused_smem = fused_chi2 ? chi2_summary_smem((int)fh.size(), max_items) : 0;
    }
    // lightcurve points: two views each (src/shape/calc_fits.c:1634-1716);
    // a plane-of-sky frame is rendered the same way (calc_poset,
    // src/shape/calc_fits.c:1205-1266) and keeps its brightness image
    const int LC_CHUNK = 4096;
    auto add_point = [&](const shape_lghtcrv_point &P, const shape_optical_law &law, int set, long long b_base) {
        LcPointDev pd;
        memset(&pd, 0, sizeof pd);
        FrameGeom go, gs;
        memset(&go, 0, sizeof go);
        memset(&gs, 0, sizeof gs);
        go.wscale = gs.wscale = 1.0;
        lc_view_geom(go, gs, pd, P);
        go.kind = VIEW_LC_OBS;
        go.smooth = params.pos_smooth;
        go.frame_index = (int)lcpts.size();
        pd.obs_view = (int)geoms.size();
        add_view(go, P.pos_n, P.km_per_pixel);
        gs.kind = VIEW_LC_SUN;
        gs.smooth = 0;
        gs.frame_index = (int)lcpts.size();
        pd.sun_view = (int)geoms.size();
        add_view(gs, P.pos_n, P.km_per_pixel);
        pd.set = set;
        pd.law_type = law.type;
        pd.intensityfactor = pow(P.km_per_pixel / SHAPE_AU, 2.0);
        if (law.type == SHAPE_OPTLAW_LAMBERT) {
            pd.scale = law.R / SHAPE_PIE;
        } else if (law.type == SHAPE_OPTLAW_LOMMEL) {
            pd.scale = law.R / (4 * SHAPE_PIE);
        } else {
            double phasefunc = law.A0 * exp(-P.solar_phase / law.D) + law.k * P.solar_phase + 1;
            pd.s_ls = (1 - law.wt) * phasefunc * law.R / (4 * SHAPE_PIE);
            pd.s_l = law.wt * phasefunc * law.R / SHAPE_PIE;
        }
        pd.mask_tol = params.mask_tol;
        pd.pixels_per_km = 1 / P.km_per_pixel;
        pd.b_base = b_base;
        int side = 2 * P.pos_n + 1;
        long long np = (long long)side * side;
        pt_items.push_back((int)lc_items.size());
        int cnt = 0;
        for (long long p0 = 0; p0 < np; p0 += LC_CHUNK, cnt++)
            lc_items.push_back(make_int2((int)lcpts.size(), (int)p0));
        pt_items.push_back(cnt);
        lcpts.push_back(pd);
    };
    for (size_t s = 0; s < lc.size(); s++) {
        const shape_lghtcrv_set &S = lc[s].set;
        if (S.law.type != SHAPE_OPTLAW_LAMBERT && S.law.type != SHAPE_OPTLAW_LOMMEL &&
            S.law.type != SHAPE_OPTLAW_KAASALAINEN)
            return set_err(SHAPE_E_UNSUPPORTED, "optical scattering law not supported");
        LcSetDev L;
        memset(&L, 0, sizeof L);
        L.npts = lc[s].npts;
        L.n = S.n;
        L.pt0 = lc[s].pt0;
        L.item0 = (int)lc_items.size();
        L.weight = S.weight;
        L.dof = S.dof;
        L.cal_in = S.cal;
        L.cal_floating = S.cal_floating;
        for (int k = 0; k < lc[s].npts; k++) add_point(points[lc[s].pt0 + k], S.law, (int)s, -1);
        L.nitems = (int)lc_items.size() - L.item0;
        lcdev.push_back(L);
    }
    // plane-of-sky frames after every lightcurve point: their views'
    // points (ps_points), brightness images and resampling descriptors
    ps_points.clear();
    psf.clear();
    ps_img_elems = ps_b_elems = 0;
    for (size_t s = 0; s < ps.size(); s++) {
        const PosetHost &H = ps[s];
        for (size_t k = 0; k < H.frames.size(); k++) {
            const shape_poset_frame &Fr = H.frames[k];
            shape_lghtcrv_point P;
            memset(&P, 0, sizeof P);
            P.pos_n = Fr.pos_n;
            P.km_per_pixel = Fr.km_per_pixel;
            memcpy(P.ae, Fr.ae, sizeof P.ae);
            memcpy(P.oe, Fr.oe, sizeof P.oe);
            memcpy(P.se, Fr.se, sizeof P.se);
            P.solar_phase = Fr.solar_phase;
            ps_points.push_back(P);
            PosetFrameDev d;
            memset(&d, 0, sizeof d);
            d.point = (int)lcpts.size();
            d.ncol = Fr.ncol;
            d.nrow = Fr.nrow;
            d.img_base = ps_img_elems;
            // the resampling grid of calc_poset (src/shape/calc_fits.c:1278-1291)
            const double xcom_fit = (Fr.colcom_vig - (Fr.ncol + 1) / 2.0) + Fr.xoff;
            const double ycom_fit = (Fr.rowcom_vig - (Fr.nrow + 1) / 2.0) + Fr.yoff;
            const double fact = Fr.fit_km_per_pixel / Fr.km_per_pixel;
            d.x0 = -xcom_fit * fact;
            d.y0 = -ycom_fit * fact;
            d.xwidth = fact * (Fr.ncol - 1);
            d.ywidth = fact * (Fr.nrow - 1);
            const double angle = -Fr.northangle;
            d.cosang = cos(angle);
            d.sinang = sin(angle);
            d.mode = H.set.resample;
            d.rebin = H.set.rebin ? 1 : 0;
            d.weight = Fr.weight;
            d.dof = Fr.dof;
            psf.push_back(d);
            add_point(P, H.set.law, -1, ps_b_elems);
            const long long side = 2 * (long long)Fr.pos_n + 1;
            ps_b_elems += side * side;
            ps_img_elems += (long long)Fr.ncol * Fr.nrow;
        }
    }
    if (laws.empty()) laws.push_back(RadarLawDev{SHAPE_RADLAW_COSINE_DIFF, 0.0, 0.0, 0.0, 0.0, 0.0, 0, 0});
    ntiles = tile_base;
    pos_elems = pos_base;
    fit_elems = obs.size();

    // ---- device allocations
    int rc;
#define AL(p, n) if ((rc = mem.alloc(&(p), (n))) != SHAPE_OK) return rc
    AL(d_a, (size_t)3 * nv); AL(d_u, (size_t)3 * nv); AL(d_r, (size_t)npar());
    d_scale = d_r + nv;
    AL(d_fv, (size_t)3 * nf); AL(d_afp, (size_t)nv + 1); AL(d_afi, af_idx.size());
    AL(md.vx, (size_t)nv); AL(md.vn, (size_t)nv); AL(md.fn, (size_t)nf); AL(md.area, (size_t)nf);
    AL(md.fvi, (size_t)nf);
    AL(d_geoms, (size_t)nviews); AL(d_states, (size_t)nviews); AL(d_laws, laws.size());
    AL(d_work, work.size());
    AL(d_vt64, (size_t)nviews * nv);
    AL(d_bin_count, (size_t)ntiles); AL(d_bin_ids, (size_t)ntiles * cap);
    AL(d_obs, (size_t)fit_elems); AL(d_oov, (size_t)fit_elems);
    // the FP32 raster adds rows of its footprints with aligned 16-byte
    // vector reductions that may reach up to 8 elements past a row's last
    // bin (adding zero); the padding keeps the last frame's in the array
    AL(d_fit64, (size_t)fit_elems); AL(d_fit32, (size_t)fit_elems + FIT32_PAD);
    {
        double *pz, *pc, *pi;
        AL(pz, (size_t)pos_elems); AL(pc, (size_t)pos_elems); AL(pi, (size_t)pos_elems);
        d_pos_z = pz; d_pos_cose = pc; d_pos_cosi = pi;
    }
    AL(d_pos_f, (size_t)pos_elems);
    AL(d_seen, (size_t)nf);
    AL(d_chi2_items, chi2_items.size()); AL(d_frame_view, frame_view.size());
    AL(d_partials, chi2_items.size() * 6);
    AL(d_o2pre, chi2_items.size() * 2);
    AL(d_chi2_counters, fh.size() + 1);
    AL(d_fh, fh.size()); AL(d_results, fh.size());
    AL(d_set_delpp, set_delpp.size()); AL(d_set_doppp, set_doppp.size()); AL(d_dop_extra, dop_extra.size());
    AL(d_lcpts, lcpts.size()); AL(d_lc_items, lc_items.size()); AL(d_pt_items, pt_items.size());
    AL(d_lc_partials, lc_items.size());
    AL(d_lcsets, lcdev.size()); AL(d_lc_out, 4 * lcdev.size());
    AL(d_lc_dof, lcdev.size()); AL(d_lc_npts, lcdev.size());
    AL(d_setrecs, setrecs.size());
    AL(d_psf, psf.size()); AL(d_ps_res, psf.size());
    AL(d_ps_obs, (size_t)ps_img_elems); AL(d_ps_oov, (size_t)ps_img_elems); AL(d_ps_fit, (size_t)ps_img_elems);
    AL(d_ps_b, (size_t)ps_b_elems);
    if (!dop_frames.empty()) {
        AL(d_ovf, dop_frames.size() * DOP_MAXOVERFLOW);
        AL(d_ovf_out, dop_frames.size() * DOP_OVF_TERMS);
        AL(d_dop_frames, dop_frames.size());
    }
    size_t lc_tot_pts = points.size(), lc_tot_n = 0;
    for (auto &L : lc) lc_tot_n += L.set.n;
    AL(d_lc_x, lc_tot_pts); AL(d_lc_y, lc_tot_pts); AL(d_lc_y2, lc_tot_pts);
    AL(d_lc_t, lc_tot_n); AL(d_lc_obs, lc_tot_n); AL(d_lc_oov, lc_tot_n);
    AL(d_lc_fit, lc_tot_n + lc_tot_pts);
#undef AL
    if (!h_params) CK(cudaMallocHost((void **)&h_params, sizeof(double) * (size_t)npar()));
    else {
        cudaFreeHost(h_params);
        CK(cudaMallocHost((void **)&h_params, sizeof(double) * (size_t)npar()));
    }
    if (!h_summary) {
        CK(cudaHostAlloc((void **)&h_summary, sizeof(shape_eval_summary), cudaHostAllocMapped));
        CK(cudaHostGetDevicePointer((void **)&d_summary_map, h_summary, 0));
    }

    // ---- uploads (once)
    cudaStream_t s = stream;
    CK(cudaMemcpyAsync(d_a, a.data(), sizeof(double) * 3 * nv, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_u, u.data(), sizeof(double) * 3 * nv, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_fv, fv.data(), sizeof(int) * 3 * nf, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_afp, af_ptr.data(), sizeof(int) * (nv + 1), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_afi, af_idx.data(), sizeof(int) * std::max<size_t>(1, af_idx.size()),
                       cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_geoms, geoms.data(), sizeof(FrameGeom) * nviews, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_laws, laws.data(), sizeof(RadarLawDev) * std::max<size_t>(1, laws.size()),
                       cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_work, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice, s));
    if (fit_elems) {
        CK(cudaMemcpyAsync(d_obs, obs.data(), sizeof(double) * fit_elems, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_oov, oov.data(), sizeof(double) * fit_elems, cudaMemcpyHostToDevice, s));
    }
    if (!chi2_items.empty()) {
        CK(cudaMemcpyAsync(d_chi2_items, chi2_items.data(), sizeof(Chi2Item) * chi2_items.size(),
                           cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_frame_view, frame_view.data(), sizeof(int) * frame_view.size(),
                           cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_fh, fh.data(), sizeof(FrameHost) * fh.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_set_delpp, set_delpp.data(), sizeof(double) * set_delpp.size(),
                           cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_set_doppp, set_doppp.data(), sizeof(double) * set_doppp.size(),
                           cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_dop_extra, dop_extra.data(), sizeof(double) * dop_extra.size(),
                           cudaMemcpyHostToDevice, s));
    }
    if (!chi2_items.empty()) {
        // o2 = sum obs^2/var of each item depends on the data only: summed
        // once here by the evaluation's own kernel and order, then kept
        CK(cudaMemsetAsync(d_fit64, 0, sizeof(double) * fit_elems, s));
        Chi2Args c0;
        memset(&c0, 0, sizeof c0);
        c0.items = d_chi2_items; c0.nitems = (int)chi2_items.size();
        c0.obs = d_obs; c0.oov = d_oov; c0.fit = d_fit64;
        c0.geoms = d_geoms; c0.frame_view = d_frame_view; c0.partials = d_partials;
        c0.o2pre = nullptr;
        launch_chi2_partials(c0, 0, s);
        CK(cudaMemcpy2DAsync(d_o2pre, 2 * sizeof(double), d_partials, 6 * sizeof(double), 2 * sizeof(double),
                             chi2_items.size(), cudaMemcpyDeviceToDevice, s));
    }
    if (!lcpts.empty()) {
        CK(cudaMemcpyAsync(d_lcpts, lcpts.data(), sizeof(LcPointDev) * lcpts.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_lc_items, lc_items.data(), sizeof(int2) * lc_items.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_pt_items, pt_items.data(), sizeof(int) * pt_items.size(), cudaMemcpyHostToDevice, s));
        size_t px = 0, pn = 0;
        std::vector<double> lcdof, lcnp;
        for (size_t k = 0; k < lc.size(); k++) {
            LcSetDev &L = lcdev[k];
            L.x = d_lc_x + px; L.y = d_lc_y + px; L.y2 = d_lc_y2 + px;
            L.t = d_lc_t + pn; L.obs = d_lc_obs + pn; L.oov = d_lc_oov + pn;
            L.fit = d_lc_fit + pn + px;   // n outputs followed by npts scratch
            CK(cudaMemcpyAsync(d_lc_x + px, lc[k].x.data(), sizeof(double) * L.npts, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(d_lc_t + pn, lc[k].t.data(), sizeof(double) * L.n, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(d_lc_obs + pn, lc[k].obs.data(), sizeof(double) * L.n, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(d_lc_oov + pn, lc[k].oov.data(), sizeof(double) * L.n, cudaMemcpyHostToDevice, s));
            px += L.npts;
            pn += L.n;
            lcdof.push_back(L.dof);
            lcnp.push_back((double)L.npts);
        }
        CK(cudaMemcpyAsync(d_lcsets, lcdev.data(), sizeof(LcSetDev) * lcdev.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_lc_dof, lcdof.data(), sizeof(double) * lcdof.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_lc_npts, lcnp.data(), sizeof(double) * lcnp.size(), cudaMemcpyHostToDevice, s));
    }
    CK(cudaMemcpyAsync(d_setrecs, setrecs.data(), sizeof(SetRec) * setrecs.size(), cudaMemcpyHostToDevice, s));
    if (!psf.empty()) {
        CK(cudaMemcpyAsync(d_psf, psf.data(), sizeof(PosetFrameDev) * psf.size(), cudaMemcpyHostToDevice, s));
        for (const PosetHost &H : ps) {
            const long long b = psf[H.frame0].img_base;
            CK(cudaMemcpyAsync(d_ps_obs + b, H.obs.data(), sizeof(double) * H.obs.size(), cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(d_ps_oov + b, H.oov.data(), sizeof(double) * H.oov.size(), cudaMemcpyHostToDevice, s));
        }
    }
    if (!dop_frames.empty())
        CK(cudaMemcpyAsync(d_dop_frames, dop_frames.data(), sizeof(int) * dop_frames.size(),
                           cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(d_seen, 0, nf, s));
    CK(cudaStreamSynchronize(s));

    if (!stream2) {
        CK(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&stream3, cudaStreamNonBlocking));
        for (auto &e : evf) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    CK(configure_raster_f64());
    CK(configure_raster_f32());
    CK(configure_lc_finalize());
    CK(configure_summary());
    md.nv = nv; md.nf = nf;
    md.a = d_a; md.u = d_u; md.r = d_r; md.scale = d_scale;
    md.vcomp = nullptr;
    md.cxf = nullptr;
    if (ncomp > 1) {
        if ((rc = mem.alloc(&d_vcomp, (size_t)nv)) != SHAPE_OK) return rc;
        if ((rc = mem.alloc(&d_cxf, cxf.size())) != SHAPE_OK) return rc;
        CK(cudaMemcpyAsync(d_vcomp, vcomp.data(), sizeof(int) * (size_t)nv, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_cxf, cxf.data(), sizeof(double) * cxf.size(), cudaMemcpyHostToDevice, stream));
        md.vcomp = d_vcomp;
        md.cxf = d_cxf;
    }
    md.fv = d_fv; md.af_ptr = d_afp; md.af_idx = d_afi;
    rc = tune_bins();
    if (rc) return rc;
    rc = setup_spin_device();
    if (rc) return rc;
    finalized = true;
    return SHAPE_OK;
}

// A new view for radar frame fi (spin, pole and delay-correction trials):
// its constants are recomputed as finalize computes them and the changed
// elements copied to the device on the engine stream, ahead of the next
// evaluation. Every kernel reads them through the device arrays, so the
// captured graphs stay valid.
int EngineImpl::set_frame_view(int fi, const double ae[9], const double oe[9], const double spin[3],
                               double deloff, double dopoff)
{
    if (fi < 0 || fi >= (int)frames.size()) return set_err(SHAPE_E_ARG, "set_frame_view: frame out of range");
    if (!fviews[fi].empty())
        return set_err(SHAPE_E_UNSUPPORTED, "set_frame_view: the frame has several views (smearing)");
    if (spin_device) return set_err(SHAPE_E_STATE, "set_frame_view: views are realized on the device from the spin model");
    shape_deldop_frame &F = frames[fi];
    memcpy(F.ae, ae, sizeof F.ae);
    memcpy(F.oe, oe, sizeof F.oe);
    memcpy(F.spin, spin, sizeof F.spin);
    size_t s = 0;
    while (!(fi >= dd[s].frame0 && fi < dd[s].frame0 + dd[s].nframes)) s++;
    F.deloff = dd[s].doppler ? 0.0 : deloff;
    F.dopoff = dopoff;
    if (!finalized) return SHAPE_OK;
    FrameHost &h = fh[fi];
    FrameGeom &g = geoms[h.view];
    radar_view_geom(g, h, dop_extra[fi], F, dd[s].set);
    view_float_consts(g);
    cudaStream_t st = stream;
    CK(cudaMemcpyAsync(d_geoms + h.view, &g, sizeof g, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_fh + fi, &h, sizeof h, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_dop_extra + fi, &dop_extra[fi], sizeof(double), cudaMemcpyHostToDevice, st));
    return SHAPE_OK;
}

// A new view for lightcurve point pt (same contract as set_frame_view).
int EngineImpl::set_point_view(int pt, const double ae[9], const double oe[9], const double se[9])
{
    if (pt < 0 || pt >= (int)points.size()) return set_err(SHAPE_E_ARG, "set_point_view: point out of range");
    if (spin_device) return set_err(SHAPE_E_STATE, "set_point_view: views are realized on the device from the spin model");
    shape_lghtcrv_point &P = points[pt];
    memcpy(P.ae, ae, sizeof P.ae);
    memcpy(P.oe, oe, sizeof P.oe);
    memcpy(P.se, se, sizeof P.se);
    if (!finalized) return SHAPE_OK;
    LcPointDev &pd = lcpts[pt];
    FrameGeom &go = geoms[pd.obs_view], &gs = geoms[pd.sun_view];
    lc_view_geom(go, gs, pd, P);
    view_float_consts(go);
    view_float_consts(gs);
    cudaStream_t st = stream;
    CK(cudaMemcpyAsync(d_geoms + pd.obs_view, &go, sizeof go, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_geoms + pd.sun_view, &gs, sizeof gs, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_lcpts + pt, &pd, sizeof pd, cudaMemcpyHostToDevice, st));
    return SHAPE_OK;
}

int EngineImpl::set_spin_model(const shape_spin_state &sp, const double *ao, const double *oo, const double *t,
                               const double *orb)
{
    if (!t && !frames.empty()) return set_err(SHAPE_E_ARG, "set_spin_model: frame epochs needed");
    const size_t nsets = setrecs.size(), nfr = frames.size();
    spin_st = sp;
    spin_angleoff.assign(ao ? ao : nullptr, ao ? ao + 3 * nsets : nullptr);
    spin_omegaoff.assign(oo ? oo : nullptr, oo ? oo + 3 * nsets : nullptr);
    spin_angleoff.resize(3 * nsets, 0.0);
    spin_omegaoff.resize(3 * nsets, 0.0);
    frame_t.assign(t ? t : nullptr, t ? t + nfr : nullptr);
    frame_orbspin.assign(orb ? orb : nullptr, orb ? orb + 3 * nfr : nullptr);
    frame_orbspin.resize(3 * nfr, 0.0);
    have_spin = true;
    int rc = realize_views();
    if (rc == SHAPE_OK && finalized && spin_device) rc = setup_spin_device();
    return rc;
}

// The field of the spin model that a spin parameter names, or null.
double *EngineImpl::spin_param(int kind, int index)
{
    if (!have_spin || index < 0) return nullptr;
    const int nsets = (int)(spin_angleoff.size() / 3);
    switch (kind) {
    case SHAPE_PAR_SPIN_ANGLE: return index < 3 ? &spin_st.angle[index] : nullptr;
    case SHAPE_PAR_SPIN_OMEGA: return index < 3 ? &spin_st.omega[index] : nullptr;
    case SHAPE_PAR_SPIN_INERTIA: return index < 3 ? &spin_st.inertia[index] : nullptr;
    case SHAPE_PAR_SPIN_OMEGADOT: return index < 3 ? &spin_st.omegadot[index] : nullptr;
    case SHAPE_PAR_SPIN_IMPULSE:
        return index < 3 * spin_st.n_impulse ? &spin_st.impulse[index / 3][index % 3] : nullptr;
    case SHAPE_PAR_SPIN_LIB:
        return index == 0 ? &spin_st.lib_amp : index == 1 ? &spin_st.lib_freq : index == 2 ? &spin_st.lib_phase
                                                                                           : nullptr;
    case SHAPE_PAR_ANGLEOFF: return index < 3 * nsets ? &spin_angleoff[index] : nullptr;
    case SHAPE_PAR_OMEGAOFF: return index < 3 * nsets ? &spin_omegaoff[index] : nullptr;
    default: return nullptr;
    }
}

// Realizes every view's ae (and a radar frame's spin vector) from the spin
// model, dataset by dataset, then refreshes the view constants.
int EngineImpl::realize_views()
{
    if (!ps.empty()) return set_err(SHAPE_E_UNSUPPORTED, "spin model: plane-of-sky sets take their views as given");
    if (spin_angleoff.size() != 3 * setrecs.size() || frame_t.size() != frames.size())
        return set_err(SHAPE_E_STATE, "spin model: datasets were added after set_spin_model");
    for (const auto &V : fviews)
        if (!V.empty()) return set_err(SHAPE_E_UNSUPPORTED, "spin model: a frame has several views (smearing)");
    std::vector<double> ae, sp, zero;
    for (size_t r = 0; r < setrecs.size(); r++) {
        const double *ao = &spin_angleoff[3 * r], *oo = &spin_omegaoff[3 * r];
        if (setrecs[r].type == 0) {
            const int f0 = setrecs[r].first, n = setrecs[r].count;
            ae.resize(9 * (size_t)n);
            sp.resize(3 * (size_t)n);
            int rc = shape_realize_spin(&spin_st, ao, oo, n, &frame_t[f0], &frame_orbspin[3 * (size_t)f0],
                                        ae.data(), sp.data());
            if (rc) return rc;
            for (int k = 0; k < n; k++) {
                memcpy(frames[f0 + k].ae, &ae[9 * (size_t)k], 9 * sizeof(double));
                memcpy(frames[f0 + k].spin, &sp[3 * (size_t)k], 3 * sizeof(double));
            }
        } else {
            const LcSetHost &L = lc[setrecs[r].first];
            ae.resize(9 * (size_t)L.npts);
            sp.resize(3 * (size_t)L.npts);
            zero.assign(3 * (size_t)L.npts, 0.0);
            int rc = shape_realize_spin(&spin_st, ao, oo, L.npts, L.x.data(), zero.data(), ae.data(), sp.data());
            if (rc) return rc;
            for (int k = 0; k < L.npts; k++) memcpy(points[L.pt0 + k].ae, &ae[9 * (size_t)k], 9 * sizeof(double));
        }
    }
    return refresh_views();
}

// Spin realization inside the evaluation: one source per radar frame and
// lightcurve point (its epoch, dataset record and orbital spin), device
// copies of the frames, points and delay-Doppler sets it rebuilds views
// from, and the pinned spin state and offsets the graph copies in.
int EngineImpl::setup_spin_device()
{
    n_spin_src = 0;
    if (!spin_device) return SHAPE_OK;
    if (!have_spin) return set_err(SHAPE_E_STATE, "device spin realization: no spin model");
    if (!ps.empty())
        return set_err(SHAPE_E_UNSUPPORTED, "device spin realization: plane-of-sky sets take their views as given");
    if (!spin_st.pa)
        return set_err(SHAPE_E_UNSUPPORTED, "device spin realization: principal-axis rotators only");
    for (const auto &V : fviews)
        if (!V.empty()) return set_err(SHAPE_E_UNSUPPORTED, "device spin realization: a frame has several views");
    std::vector<SpinViewSrc> src;
    for (size_t r = 0; r < setrecs.size(); r++) {
        if (setrecs[r].type == 0) {
            int ds = 0;
            while (ds < (int)dd.size() && dd[ds].frame0 != setrecs[r].first) ds++;
            for (int k = 0; k < setrecs[r].count; k++) {
                const int fi = setrecs[r].first + k;
                SpinViewSrc v{0, fi, (int)r, ds, frame_t[fi], {0.0, 0.0, 0.0}};
                for (int j = 0; j < 3; j++) v.orb[j] = frame_orbspin[3 * (size_t)fi + j];
                src.push_back(v);
            }
        } else {
            const LcSetHost &L = lc[setrecs[r].first];
            for (int k = 0; k < L.npts; k++) src.push_back(SpinViewSrc{1, L.pt0 + k, (int)r, 0, L.x[k], {0.0, 0.0, 0.0}});
        }
    }
    std::vector<shape_deldop_set> sets;
    for (const DdSetHost &D : dd) sets.push_back(D.set);
    const size_t nrec = setrecs.size();
    int rc;
    for (void *p : {(void *)d_spin_src, (void *)d_spin, (void *)d_spin_off, (void *)d_frames_dev,
                    (void *)d_ddsets, (void *)d_points_dev})
        if (p) mem.release_one(p);
    d_spin_src = nullptr; d_spin = nullptr; d_spin_off = nullptr;
    d_frames_dev = nullptr; d_ddsets = nullptr; d_points_dev = nullptr;
    if ((rc = mem.alloc(&d_spin_src, std::max<size_t>(1, src.size()))) != SHAPE_OK) return rc;
    if ((rc = mem.alloc(&d_spin, 1)) != SHAPE_OK) return rc;
    if ((rc = mem.alloc(&d_spin_off, 6 * std::max<size_t>(1, nrec))) != SHAPE_OK) return rc;
    if ((rc = mem.alloc(&d_frames_dev, std::max<size_t>(1, frames.size()))) != SHAPE_OK) return rc;
    if ((rc = mem.alloc(&d_ddsets, std::max<size_t>(1, sets.size()))) != SHAPE_OK) return rc;
    if ((rc = mem.alloc(&d_points_dev, std::max<size_t>(1, points.size()))) != SHAPE_OK) return rc;
    if (h_spin_off) cudaFreeHost(h_spin_off);
    h_spin_off = nullptr;
    if (!h_spin) CK(cudaMallocHost((void **)&h_spin, sizeof(shape_spin_state)));
    CK(cudaMallocHost((void **)&h_spin_off, sizeof(double) * 6 * std::max<size_t>(1, nrec)));
    cudaStream_t st = stream;
    if (!src.empty())
        CK(cudaMemcpyAsync(d_spin_src, src.data(), sizeof(SpinViewSrc) * src.size(), cudaMemcpyHostToDevice, st));
    if (!frames.empty())
        CK(cudaMemcpyAsync(d_frames_dev, frames.data(), sizeof(shape_deldop_frame) * frames.size(),
                           cudaMemcpyHostToDevice, st));
    if (!sets.empty())
        CK(cudaMemcpyAsync(d_ddsets, sets.data(), sizeof(shape_deldop_set) * sets.size(), cudaMemcpyHostToDevice, st));
    if (!points.empty())
        CK(cudaMemcpyAsync(d_points_dev, points.data(), sizeof(shape_lghtcrv_point) * points.size(),
                           cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    n_spin_src = (int)src.size();
    invalidate_graphs();
    return SHAPE_OK;
}

// The spin state and offsets of the next evaluation, into pinned memory.
void EngineImpl::fill_spin()
{
    if (!spin_device || !h_spin) return;
    *h_spin = spin_st;
    for (size_t r = 0; r < setrecs.size(); r++)
        for (int j = 0; j < 3; j++) {
            h_spin_off[6 * r + j] = spin_angleoff[3 * r + j];
            h_spin_off[6 * r + 3 + j] = spin_omegaoff[3 * r + j];
        }
}

// First step of an evaluation in device spin mode: the state copy and the
// view realization (before the transform reads the views).
int EngineImpl::enqueue_spin()
{
    if (!spin_device || n_spin_src == 0) return SHAPE_OK;
    cudaStream_t st = stream;
    CK(cudaMemcpyAsync(d_spin, h_spin, sizeof(shape_spin_state), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_spin_off, h_spin_off, sizeof(double) * 6 * std::max<size_t>(1, setrecs.size()),
                       cudaMemcpyHostToDevice, st));
    SpinRealizeArgs a;
    a.n = n_spin_src;
    a.src = d_spin_src; a.spin = d_spin; a.off = d_spin_off;
    a.frames = d_frames_dev; a.ddsets = d_ddsets; a.points = d_points_dev;
    a.geoms = d_geoms; a.fh = d_fh; a.dop_extra = d_dop_extra; a.lcpts = d_lcpts;
    launch_realize_views(a, st);
    return SHAPE_OK;
}

// After finalize: every view's constants recomputed from frames / points and
// the arrays copied to the device on the engine stream (set_frame_view does
// the same for one frame).
int EngineImpl::refresh_views()
{
    if (!finalized) return SHAPE_OK;
    for (size_t s = 0; s < dd.size(); s++)
        for (int k = 0; k < dd[s].nframes; k++) {
            const int fi = dd[s].frame0 + k;
            FrameHost &h = fh[fi];
            radar_view_geom(geoms[h.view], h, dop_extra[fi], frames[fi], dd[s].set);
            view_float_consts(geoms[h.view]);
        }
    for (size_t pt = 0; pt < lcpts.size(); pt++) {
        LcPointDev &pd = lcpts[pt];
        const shape_lghtcrv_point &P = pt < points.size() ? points[pt] : ps_points[pt - points.size()];
        lc_view_geom(geoms[pd.obs_view], geoms[pd.sun_view], pd, P);
        view_float_consts(geoms[pd.obs_view]);
        view_float_consts(geoms[pd.sun_view]);
    }
    cudaStream_t st = stream;
    CK(cudaMemcpyAsync(d_geoms, geoms.data(), sizeof(FrameGeom) * geoms.size(), cudaMemcpyHostToDevice, st));
    if (!fh.empty()) {
        CK(cudaMemcpyAsync(d_fh, fh.data(), sizeof(FrameHost) * fh.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_dop_extra, dop_extra.data(), sizeof(double) * dop_extra.size(),
                           cudaMemcpyHostToDevice, st));
    }
    if (!lcpts.empty())
        CK(cudaMemcpyAsync(d_lcpts, lcpts.data(), sizeof(LcPointDev) * lcpts.size(), cudaMemcpyHostToDevice, st));
    return SHAPE_OK;
}

// ---- penalties (src/shape/penalties.c:121-1236)

static bool pen_needs_spin(int t)
{
    return t == SHAPE_PEN_INERTIADEV || t == SHAPE_PEN_NONPA || t == SHAPE_PEN_IMPULSE;
}

int EngineImpl::set_penalties(int n, const int *type, const double *weight)
{
    if (n < 0 || (n > 0 && (!type || !weight))) return set_err(SHAPE_E_ARG, "set_penalties: invalid argument");
    for (int i = 0; i < n; i++) {
        switch (type[i]) {
        case SHAPE_PEN_NONSMOOTH: case SHAPE_PEN_CONCAVITY: case SHAPE_PEN_RDEV: case SHAPE_PEN_VOLUME:
        case SHAPE_PEN_COMDEV: case SHAPE_PEN_INERTIADEV: case SHAPE_PEN_INERTIADEV_UNI: case SHAPE_PEN_PA3TILT:
        case SHAPE_PEN_NONPA: case SHAPE_PEN_NONPA_UNI: case SHAPE_PEN_EULEROFFS: case SHAPE_PEN_FLATTENING:
        case SHAPE_PEN_MAXRDEV: case SHAPE_PEN_IMPULSE:
            break;
        default:
            return set_err(SHAPE_E_UNSUPPORTED, "set_penalties: penalty type not supported");
        }
    }
    pen_type.assign(type, type + n);
    pen_weight.assign(weight, weight + n);
    pen_base.assign((size_t)n, 0.0);
    return SHAPE_OK;
}

// Before an evaluation with penalties: the spin model where a penalty needs
// it, the edges of the closed triangulated surface (each with its two
// facets) and the device buffers of the model sums, built on first use.
int EngineImpl::prepare_penalties()
{
    for (int t : pen_type)
        if (pen_needs_spin(t) && !have_spin)
            return set_err(SHAPE_E_STATE, "penalties: inertiadev, nonpa and impulse need the spin model");
    if (!d_sides) {
        struct Half { long long key; int f, j; };
        std::vector<Half> hs;
        hs.reserve(3 * (size_t)nf);
        for (int f = 0; f < nf; f++)
            for (int j = 0; j < 3; j++) {
                const long long a = fv[3 * f + j], b = fv[3 * f + (j + 1) % 3];
                hs.push_back(Half{std::min(a, b) * (long long)nv + std::max(a, b), f, j});
            }
        std::sort(hs.begin(), hs.end(), [](const Half &x, const Half &y) {
            return x.key != y.key ? x.key < y.key : x.f < y.f;
        });
        std::vector<int4> sides;
        std::vector<int> side_v2;
        for (size_t k = 0; k < hs.size(); k += 2) {
            if (k + 1 >= hs.size() || hs[k + 1].key != hs[k].key || (k + 2 < hs.size() && hs[k + 2].key == hs[k].key))
                return set_err(SHAPE_E_ARG, "penalties: the model is not a closed surface (an edge without two facets)");
            const Half &h1 = hs[k];
            sides.push_back(make_int4(fv[3 * h1.f + h1.j], fv[3 * h1.f + (h1.j + 2) % 3], h1.f, hs[k + 1].f));
            side_v2.push_back(fv[3 * h1.f + (h1.j + 1) % 3]);
        }
        nsides = (int)sides.size();
        int rc;
        if (ncomp > 1) {
            // check_surface's inputs and flags: each component's facet range
            // (components listed back to back), the edges' other ends
            std::vector<int2> cf((size_t)ncomp, make_int2(0, 0));
            for (int f = 0; f < nf; f++) {
                const int c = vcomp[fv[3 * f]];
                if (cf[c].y == 0) cf[c].x = f;
                cf[c].y++;
            }
            if ((rc = mem.alloc(&d_comp_facets, cf.size())) != SHAPE_OK) return rc;
            if ((rc = mem.alloc(&d_side_v2, side_v2.size())) != SHAPE_OK) return rc;
            if ((rc = mem.alloc(&d_act_v, (size_t)nv)) != SHAPE_OK) return rc;
            if ((rc = mem.alloc(&d_act_f, (size_t)nf)) != SHAPE_OK) return rc;
            if ((rc = mem.alloc(&d_surf_err, 1)) != SHAPE_OK) return rc;
            CK(cudaMemcpyAsync(d_comp_facets, cf.data(), sizeof(int2) * cf.size(), cudaMemcpyHostToDevice, stream));
            CK(cudaMemcpyAsync(d_side_v2, side_v2.data(), sizeof(int) * side_v2.size(), cudaMemcpyHostToDevice,
                               stream));
        }
        if ((rc = mem.alloc(&d_sides, sides.size())) != SHAPE_OK) return rc;
        if ((rc = mem.alloc(&d_msum_part, (size_t)model_sums_blocks() * MSUM_N)) != SHAPE_OK) return rc;
        if ((rc = mem.alloc(&d_msum, (size_t)MSUM_N)) != SHAPE_OK) return rc;
        if (!h_msum) CK(cudaMallocHost((void **)&h_msum, sizeof(double) * MSUM_N));
        CK(cudaMemcpyAsync(d_sides, sides.data(), sizeof(int4) * sides.size(), cudaMemcpyHostToDevice, stream));
    }
    return SHAPE_OK;
}

// The two model-sum launches and the copy of the sums to pinned memory, on
// the engine stream after the evaluation.
int EngineImpl::enqueue_model_sums()
{
    ModelSumArgs a;
    memset(&a, 0, sizeof a);
    a.m = md;
    a.sides = d_sides;
    a.nsides = nsides;
    a.ncomp = ncomp;
    a.part = d_msum_part;
    a.out = d_msum;
    if (ncomp > 1) {
        a.side_v2 = d_side_v2;
        a.comp_facets = d_comp_facets;
        a.act_v = d_act_v;
        a.act_f = d_act_f;
        a.surf_err = d_surf_err;
        CK(cudaMemsetAsync(d_surf_err, 0, sizeof(int), stream));
        launch_check_surface(a, stream);
    }
    launch_model_sums(a, stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_msum, d_msum, sizeof(double) * MSUM_N, cudaMemcpyDeviceToHost, stream));
    return SHAPE_OK;
}

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (Jacobi's method; each rotation through the smaller angle, |tan| <= 1), so
// every eigenvalue stays at the diagonal position it converges from: d =
// eigenvalues, columns of V = eigenvectors (principal axes in body
// coordinates). Converges quadratically; 50 sweeps bound it.
static void jacobi3(const double A[3][3], double d[3], double V[3][3])
{
    double a[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) { a[i][j] = A[i][j]; V[i][j] = (i == j) ? 1.0 : 0.0; }
    for (int sweep = 0; sweep < 50; sweep++) {
        if (a[0][1] == 0.0 && a[0][2] == 0.0 && a[1][2] == 0.0) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                const double apq = a[p][q];
                if (apq == 0.0) continue;
                if (std::fabs(apq) <= 1e-18 * std::fabs(a[p][p]) && std::fabs(apq) <= 1e-18 * std::fabs(a[q][q])) {
                    a[p][q] = a[q][p] = 0.0;        // below the diagonals' rounding
                    continue;
                }
                const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                double t = 1.0 / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                if (theta < 0.0) t = -t;
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; k++) {        // columns p, q of A J
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) {        // rows p, q of J^T (A J)
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                a[p][q] = a[q][p] = 0.0;
                for (int k = 0; k < 3; k++) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 3; i++) d[i] = a[i][i];
}

// The penalty sum of the objective from the model sums (each penalty's
// value as src/shape/penalties.c:149-1220 defines it; weight >= 0 gives
// |weight| * value, a negative weight |weight| / max(value, 1e-10)).
double EngineImpl::penalty_sum(const double *ms)
{
    const double PIE = 3.141592653589793, R2D = 57.29577951308232;
    const double V = ms[MSUM_VOLUME];
    const double com[3] = {ms[MSUM_COM] / V, ms[MSUM_COM + 1] / V, ms[MSUM_COM + 2] / V};
    const double I[3][3] = {{ms[MSUM_IXX], ms[MSUM_IXY], ms[MSUM_IXZ]},
                            {ms[MSUM_IXY], ms[MSUM_IYY], ms[MSUM_IYZ]},
                            {ms[MSUM_IXZ], ms[MSUM_IYZ], ms[MSUM_IZZ]}};
    const double r_eff = pow(3 * V / (4 * PIE), 1.0 / 3.0);
    bool got_pa = false;
    double pm[3] = {0, 0, 0}, ap[3][3];
    auto principal = [&]() { if (!got_pa) { jacobi3(I, pm, ap); got_pa = true; } };
    auto inertia_dev = [&](const double *p) {
        double a = 0.0, b = 0.0, adotb = 0.0;
        for (int j = 0; j < 3; j++) {
            a += p[j] * p[j];
            adotb += p[j] * I[j][j];
            for (int k = 0; k < 3; k++) b += I[j][k] * I[j][k];
        }
        return 1 - adotb / sqrt(a * b);
    };
    auto nonpa = [](const double *p) {
        const double pen = std::max(p[0] / p[2] - 1, p[1] / p[2] - 1) + 0.01;
        return pen < 0.0 ? 0.0 : pen;
    };
    double sum = 0.0;
    for (size_t i = 0; i < pen_type.size(); i++) {
        double pen = 0.0;
        switch (pen_type[i]) {
        case SHAPE_PEN_NONSMOOTH: pen = ms[MSUM_NONSMOOTH] / ms[MSUM_NSIDES]; break;
        case SHAPE_PEN_CONCAVITY: pen = ms[MSUM_CONCAVITY] / ms[MSUM_NSIDES]; break;
        case SHAPE_PEN_RDEV: pen = ms[MSUM_RDEV] / (r_eff * r_eff) / ms[MSUM_NVERT]; break;
        case SHAPE_PEN_MAXRDEV: pen = ms[MSUM_RDEV_MAX] / (r_eff * r_eff); break;
        case SHAPE_PEN_VOLUME: pen = V; break;
        case SHAPE_PEN_COMDEV:
            for (int k = 0; k < 3; k++) pen += com[k] * com[k];
            pen /= (r_eff * r_eff);
            break;
        case SHAPE_PEN_INERTIADEV: pen = inertia_dev(spin_st.inertia); break;
        case SHAPE_PEN_INERTIADEV_UNI: principal(); pen = inertia_dev(pm); break;
        case SHAPE_PEN_PA3TILT: principal(); pen = std::max(0.0, 1 - ap[2][2] * ap[2][2]); break;
        case SHAPE_PEN_NONPA: pen = nonpa(spin_st.inertia); break;
        case SHAPE_PEN_NONPA_UNI: principal(); pen = nonpa(pm); break;
        case SHAPE_PEN_EULEROFFS: {
            int ntot = 0;
            for (size_t k = 0; k < setrecs.size(); k++)
                for (int j = 0; j < 3; j++) {
                    const double ao = have_spin ? spin_angleoff[3 * k + j] : 0.0;
                    const double oo = have_spin ? spin_omegaoff[3 * k + j] : 0.0;
                    pen += ao * ao;
                    pen += oo * oo;
                    ntot += 2;
                }
            pen *= R2D * R2D / ntot;
            break;
        }
        case SHAPE_PEN_FLATTENING: {
            principal();
            const double b_over_c =
                sqrt(std::min(-pm[0] + pm[1] + pm[2], pm[0] - pm[1] + pm[2]) / (pm[0] + pm[1] - pm[2]));
            if (b_over_c > 1.0) {
                const double x = b_over_c - 1;
                pen = x * x * x * x;
            }
            break;
        }
        case SHAPE_PEN_IMPULSE:
            for (int n = 0; n < spin_st.n_impulse; n++)
                for (int j = 0; j < 3; j++) pen += spin_st.impulse[n][j] * spin_st.impulse[n][j];
            pen *= R2D * R2D / (3 * spin_st.n_impulse);
            break;
        }
        pen_base[i] = pen_weight[i] >= 0.0 ? pen : 1.0 / std::max(pen, 1.0e-10);
        sum += fabs(pen_weight[i]) * pen_base[i];
    }
    return sum;
}

// Bin autotuning from a dry-run binning of the model as loaded: the bin
// capacity becomes the next power of two above 1.25x the fullest tile (so a
// fit's small model changes do not overflow into the full-scan path), and
// the batched raster visits tiles in decreasing facet count, so the heavy
// tiles start first instead of forming a tail.
int EngineImpl::tune_bins()
{
    cudaStream_t s = stream;
    fill_params(h_params);
    CK(cudaMemcpyAsync(d_r, h_params, sizeof(double) * npar(), cudaMemcpyHostToDevice, s));
    launch_realize(md, s);
    launch_reset_state(d_states, nviews, d_bin_count, ntiles, s);
    launch_xform_f64(d_geoms, nviews, md.vx, nv, d_vt64, s);
    launch_bin_f64(d_geoms, 0, nviews, md, d_vt64, d_states, d_bin_count, d_bin_ids, cap, s);
    std::vector<int> counts(ntiles);
    CK(cudaMemcpyAsync(counts.data(), d_bin_count, sizeof(int) * ntiles, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    int mx = 0, nonempty = 0;
    for (int c : counts) { mx = std::max(mx, c); nonempty += (c > 0); }
    tuned_max_count = mx;
    tuned_nonempty = nonempty;
    int want = 64;
    while (want < (int)(1.25 * mx) + 16 && want < 8192) want *= 2;
    if (fixed_cap > 0) want = fixed_cap;
    if (want != cap) {
        mem.release_one(d_bin_ids);
        cap = want;
        int rc = mem.alloc(&d_bin_ids, (size_t)ntiles * cap);
        if (rc) return rc;
    }
    // work order for the batched forms: decreasing count, stable
    std::vector<int> order(work.size());
    for (size_t k = 0; k < work.size(); k++) order[k] = (int)k;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        int cx = counts[geoms[work[x].x].tile_base + work[x].y];
        int cy = counts[geoms[work[y].x].tile_base + work[y].y];
        return cx > cy;
    });
    // radar tiles first, lightcurve-view tiles after them, each part in
    // decreasing count: the batched FP32 form rasters the two parts with
    // different kernels
    std::stable_partition(order.begin(), order.end(),
                          [&](int x) { return geoms[work[x].x].kind == VIEW_RADAR; });
    std::vector<int2> sorted(work.size());
    work_radar = nonempty_radar = nonempty_lc = 0;
    for (size_t k = 0; k < work.size(); k++) {
        sorted[k] = work[order[k]];
        const bool radar = geoms[sorted[k].x].kind == VIEW_RADAR;
        const bool busy = counts[geoms[sorted[k].x].tile_base + sorted[k].y] > 0;
        work_radar += radar;
        nonempty_radar += radar && busy;
        nonempty_lc += !radar && busy;
    }
    if (!d_work_sorted) {
        int rc = mem.alloc(&d_work_sorted, work.size());
        if (rc) return rc;
    }
    CK(cudaMemcpyAsync(d_work_sorted, sorted.data(), sizeof(int2) * sorted.size(), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return SHAPE_OK;
}

// Enqueue one evaluation (without the H2D of parameters / D2H of the summary).
// marks (optional, batched forms only): events recorded after each stage
// 0 realize, 1 reset, 2 transform, 3 bin, 4 raster, 5 chi2, 6 lightcurve
// photometry, 7 finalize + summary.
int EngineImpl::enqueue(int form, cudaEvent_t *marks)
{
    cudaStream_t s = stream;
    const bool f32 = (form == SHAPE_FORM_BATCHED_FP32);
    auto mark = [&](int k) { if (marks) cudaEventRecord(marks[k], s); };
    // a launch rejected by the runtime (configuration, resources) is
    // reported with the stage it belongs to
    auto launched = [&](const char *stage) -> int {
        const cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) return SHAPE_OK;
        return set_err(SHAPE_E_CUDA, std::string(stage) + ": " + cudaGetErrorString(e));
    };
    // The batched forms run two side branches beside the view transform
    // (which realizes its vertices on the fly): the state reset and image
    // clears (stream2), and realize with the facet and vertex normals
    // (stream3); binning waits for the facet normals and the reset, the
    // raster for the vertex normals. The plain form and stage timing run
    // them in line.
    const bool fork = (form != SHAPE_FORM_PLAIN_FP64) && !marks;
    cudaStream_t sr = fork ? stream2 : s;
    if (int rc = enqueue_spin()) return rc;
    if (fork) {
        CK(cudaEventRecord(evf[0], s));
        CK(cudaStreamWaitEvent(stream2, evf[0], 0));
        CK(cudaStreamWaitEvent(stream3, evf[0], 0));
        launch_realize_vf(md, stream3);
        CK(cudaEventRecord(evf[1], stream3));        // vertices, facet normals and areas
        launch_realize_vn(md, stream3);
        CK(cudaEventRecord(evf[3], stream3));        // vertex normals
    } else {
        launch_realize(md, s);
    }
    mark(0);
    if (int rc_ = launched("realize")) return rc_;
    launch_reset_state(d_states, nviews, d_bin_count, ntiles, sr);
    if (fit_elems) {
        if (f32) CK(cudaMemsetAsync(d_fit32, 0, sizeof(float) * fit_elems, sr));
        // the FP32 form sums Doppler spectra in FP64 (then rounds them once)
        if (!f32 || !dop_frames.empty()) CK(cudaMemsetAsync(d_fit64, 0, sizeof(double) * fit_elems, sr));
    }
    CK(cudaMemsetAsync(d_seen, 0, nf, sr));
    if (!dop_frames.empty())
        CK(cudaMemsetAsync(d_ovf, 0, sizeof(double) * dop_frames.size() * DOP_MAXOVERFLOW, sr));
    const bool fused = fused_chi2 && form != SHAPE_FORM_PLAIN_FP64;
    if (fused) CK(cudaMemsetAsync(d_chi2_counters, 0, sizeof(int) * (fh.size() + 1), sr));
    if (fork) CK(cudaEventRecord(evf[2], stream2));   // reset and clears done
    mark(1);
    if (int rc_ = launched("state reset")) return rc_;

    RasterArgs ra;
    memset(&ra, 0, sizeof ra);
    ra.geoms = d_geoms;
    ra.vt = d_vt64;         // both forms stage from the FP64 view-frame vertices
    ra.fvi = md.fvi;
    ra.vn = md.vn;
    ra.fn = md.fn;
    ra.nf = nf;
    ra.bin_count = d_bin_count;
    ra.bin_ids = d_bin_ids;
    ra.cap = cap;
    ra.states = d_states;
    ra.laws = d_laws;
    ra.fit = f32 ? (void *)d_fit32 : (void *)d_fit64;
    ra.fit64 = d_fit64;
    ra.pos_z = d_pos_z; ra.pos_cose = d_pos_cose; ra.pos_cosi = d_pos_cosi; ra.pos_f = d_pos_f;
    ra.seen = d_seen;
    ra.mincosine_seen = params.mincosine_seen;
    ra.mark_seen = params.mark_seen;
    ra.keep_pos = keep_pos;
    ra.ovf = d_ovf;

    Chi2Args ca;
    ca.obs = d_obs; ca.oov = d_oov;
    ca.fit = ra.fit;
    ca.geoms = d_geoms;
    ca.frame_view = d_frame_view;
    ca.partials = d_partials;
    ca.o2pre = d_o2pre;

    LcArgs la;
    memset(&la, 0, sizeof la);
    la.pts = d_lcpts; la.geoms = d_geoms; la.states = d_states;
    la.chunk = 4096;
    la.z = static_cast<const double *>(d_pos_z); la.cose = d_pos_cose; la.cosi = d_pos_cosi;
    la.zill = static_cast<const double *>(d_pos_z);
    la.f = d_pos_f; la.fill = d_pos_f;
    la.partials = d_lc_partials;
    la.bimg = d_ps_b;
    la.seen = d_seen;
    la.mincosine_seen = params.mincosine_seen;
    la.mark_seen = params.mark_seen;

    if (form == SHAPE_FORM_PLAIN_FP64) {
        // One view at a time, in dataset order, as calc_fits walks frames.
        for (int v = 0; v < nviews; v++) {
            launch_xform_f64(d_geoms + v, 1, md.vx, nv, d_vt64, s);
            launch_bin_f64(d_geoms, v, 1, md, d_vt64, d_states, d_bin_count, d_bin_ids, cap, s);
            RasterArgs rv = ra;
            rv.work = d_work + view_work0[v];
            rv.nwork = view_nwork[v];
            launch_raster_f64(rv, s);
            const FrameGeom &g = geoms[v];
            if (g.kind == VIEW_RADAR && fh[g.frame_index].view == v) {
                const FrameHost &h = fh[g.frame_index];
                Chi2Args cv = ca;
                cv.items = d_chi2_items + h.item0;
                cv.nitems = h.nitems;
                cv.partials = d_partials + (size_t)h.item0 * 6;
                cv.o2pre = d_o2pre + (size_t)h.item0 * 2;
                launch_chi2_partials(cv, 0, s);
            } else if (g.kind == VIEW_LC_SUN) {
                int pt = g.frame_index;
                LcArgs lv = la;
                lv.items = d_lc_items + pt_items[2 * pt];
                lv.nitems = pt_items[2 * pt + 1];
                lv.partials = d_lc_partials + pt_items[2 * pt];
                launch_lc_photo(lv, 0, s);
            }
            if (int rc_ = launched(g.kind == VIEW_RADAR ? "radar view chain" : "lightcurve view chain")) return rc_;
        }
    } else {
        // graph-captured chain: each kernel after the first is a programmatic
        // dependent launch of the one before it (stage timing keeps plain
        // launches so its events separate the stages)
        const bool pdl = fork;
        if (fork) launch_xform_realize_f64(d_geoms, nviews, md, d_vt64, s);
        else launch_xform_f64(d_geoms, nviews, md.vx, nv, d_vt64, s);
        mark(2);
        if (int rc_ = launched("view transform")) return rc_;
        if (fork) {
            CK(cudaStreamWaitEvent(s, evf[1], 0));
            CK(cudaStreamWaitEvent(s, evf[2], 0));
        }
        launch_bin_f64(d_geoms, 0, nviews, md, d_vt64, d_states, d_bin_count, d_bin_ids, cap, s, pdl);
        if (fork) CK(cudaStreamWaitEvent(s, evf[3], 0));
        mark(3);
        if (int rc_ = launched("binning")) return rc_;
        // one CTA per tile, heaviest tiles first (empty tiles sort last and
        // exit at once); the block scheduler balances the rest
        // one CTA per tile that was non-empty when the bins were tuned (they
        // lead each part of the sorted list); the grid-stride loop visits the
        // tiles after them, empty then, so those cost no CTA launches of
        // their own. The FP32 form rasters lightcurve views with its exact
        // variant, in a second launch.
        ra.work = d_work_sorted;
        ra.pdl = pdl ? 1 : 0;
        ra.variant = raster_variant[form];
        if (f32) {
            RasterArgs rr = ra, rl = ra;
            rr.nwork = work_radar;
            rr.exact = fp32_exact;
            rr.grid = raster_grid(form, nonempty_radar, rr, true);
            rl.work = d_work_sorted + work_radar;
            rl.nwork = (int)work.size() - work_radar;
            rl.exact = 1;
            rl.variant = 0;       // lightcurve views: the tile-per-CTA kernel
            rl.lc_views = 1;
            rl.grid = raster_grid(form, nonempty_lc, rl, true);
            launch_raster_f32(rr, s);
            launch_raster_f32(rl, s);
            launch_dop_fit_f32(d_dop_frames, (int)dop_frames.size(), d_fh, d_geoms, d_fit64, d_fit32, s);
        } else {
            ra.nwork = (int)work.size();
            ra.grid = raster_grid(form, tuned_nonempty, ra, false);
            launch_raster_f64(ra, s);
        }
        mark(4);
        if (int rc_ = launched("raster")) return rc_;
        ca.items = d_chi2_items;
        ca.nitems = (int)chi2_items.size();
        // fused: the chi-square partials run with the summary, last
        if (!chi2_items.empty() && !fused) launch_chi2_partials(ca, f32 ? 1 : 0, s);
        mark(5);
        if (int rc_ = launched("chi-square partials")) return rc_;
        if (!lc_items.empty()) {
            la.items = d_lc_items;
            la.nitems = (int)lc_items.size();
            // lightcurve views hold FP64 cosines in both forms
            launch_lc_photo(la, 0, s);
        }
        mark(6);
        if (int rc_ = launched("lightcurve photometry")) return rc_;
    }
    FinalizeArgs fa;
    memset(&fa, 0, sizeof fa);
    fa.nframes = (int)fh.size();
    fa.fh = d_fh; fa.geoms = d_geoms; fa.states = d_states; fa.partials = d_partials;
    fa.results = d_results; fa.set_delpp = d_set_delpp; fa.set_doppp = d_set_doppp;
    fa.dop_extra = d_dop_extra;
    fa.ovf_out = d_ovf_out;
    if (!dop_frames.empty()) {
        DopOvfArgs oa;
        oa.n = (int)dop_frames.size();
        oa.frames = d_dop_frames; oa.fh = d_fh; oa.geoms = d_geoms; oa.states = d_states;
        oa.ovf = d_ovf; oa.out = d_ovf_out;
        launch_doppler_overflow(oa, s);
        if (int rc_ = launched("Doppler overflow")) return rc_;
    }
    if (!psf.empty()) {
        PosetArgs pa;
        pa.nframes = (int)psf.size();
        pa.frames = d_psf; pa.pts = d_lcpts; pa.geoms = d_geoms; pa.states = d_states;
        pa.bimg = d_ps_b; pa.obs = d_ps_obs; pa.oov = d_ps_oov; pa.fit = d_ps_fit; pa.res = d_ps_res;
        launch_poset_frames(pa, s);
        if (int rc_ = launched("plane-of-sky frames")) return rc_;
    }
    if (!lcdev.empty()) {
        LcFinalizeArgs lf;
        lf.nsets = (int)lcdev.size();
        lf.sets = d_lcsets; lf.pts = d_lcpts; lf.geoms = d_geoms; lf.states = d_states;
        lf.pt_items = d_pt_items; lf.partials = d_lc_partials; lf.set_out = d_lc_out;
        size_t sm = 1;
        for (const LcSetDev &L : lcdev) {
            size_t b = lc_finalize_smem(L.npts, L.n);
            sm = (b == 0 || sm == 0) ? 0 : std::max(sm, b);
        }
        lf.smem_per_set = sm;
        launch_lc_finalize(lf, s);
        if (int rc_ = launched("lightcurve finalize")) return rc_;
    }
    SummaryArgs sa;
    memset(&sa, 0, sizeof sa);
    sa.nsets = (int)setrecs.size();
    sa.sets = d_setrecs; sa.fh = d_fh; sa.results = d_results;
    sa.lc_out = d_lc_out; sa.lc_dof = d_lc_dof; sa.lc_npts = d_lc_npts;
    sa.ps_res = d_ps_res; sa.ps_frames = d_psf; sa.dof_poset = dof_poset;
    sa.dof = dof; sa.dof_radar = dof_deldop + dof_doppler; sa.bad_objfactor = bad_objfactor;
    sa.nitems = (int)chi2_items.size();
    // the bad-diameter factor depends only on host-side scale factors and is
    // applied by evaluate(), so captured graphs stay valid when it changes
    sa.baddiam = 0;
    sa.baddiam_logfactor = 0.0;
    // the summary kernel writes the pinned host summary directly (mapped
    // memory), so an evaluation needs no device-to-host copy after it
    sa.out = d_summary_map;
    if (fused) launch_chi2_summary(ca, fa, sa, d_chi2_counters, f32 ? 1 : 0, s, fork, fused_smem);
    else launch_summary(fa, sa, s);
    mark(7);
    CK(cudaGetLastError());
    return SHAPE_OK;
}

// Kernel launches enqueue() makes for one evaluation in this form (memsets
// and copies excluded).
int EngineImpl::kernels_per_eval(int form) const
{
    int n = 2 + 1;                       // realize (vertices + facets, vertex normals), state reset
    n += (spin_device && n_spin_src > 0) ? 1 : 0;   // view realization from the spin state
    if (form == SHAPE_FORM_PLAIN_FP64) {
        for (int v = 0; v < nviews; v++)
            n += 3 + ((geoms[v].kind == VIEW_RADAR && fh[geoms[v].frame_index].view == v) ||
                              geoms[v].kind == VIEW_LC_SUN ? 1 : 0);
    } else {
        n += 3;                          // transform, bin, raster
        if (form == SHAPE_FORM_BATCHED_FP32 && work_radar > 0 && work_radar < (int)work.size())
            n += 1;                      // FP32: radar and lightcurve views in two launches
        if (form == SHAPE_FORM_BATCHED_FP32 && !dop_frames.empty())
            n += 1;                      // FP32: Doppler spectra rounded from their FP64 sums
        n += (chi2_items.empty() || fused_chi2) ? 0 : 1;   // fused: counted with the summary
        n += lc_items.empty() ? 0 : 1;
    }
    n += lcdev.empty() ? 0 : 1;          // lightcurve finalize
    n += psf.empty() ? 0 : 1;            // plane-of-sky frames
    n += dop_frames.empty() ? 0 : 1;     // Doppler overflow spectra
    n += pen_type.empty() ? 0 : (ncomp > 1 ? 3 : 2);   // model sums (and check_surface) for the penalties
    return n + 1;                        // finalize + summary (with the chi-square partials when fused)
}

int EngineImpl::evaluate(int form, shape_eval_summary *out)
{
    int rc = launch(form);
    if (rc) return rc;
    return finish(out);
}

// Enqueues one evaluation on the engine stream and returns without waiting:
// parameters host->device, the kernel sequence (a graph replay for the
// batched forms), the summary device->host, then event ev1.
int EngineImpl::launch(int form)
{
    if (!finalized) return set_err(SHAPE_E_STATE, "evaluate before finalize");
    if (form < 0 || form > 2) return set_err(SHAPE_E_ARG, "unknown form");
    cudaStream_t s = stream;
    fill_params(h_params);
    fill_spin();
    std::vector<double> sc(3 * (size_t)ncomp);
    effective_scale(sc.data(), &pending_baddiam, &pending_bdl);
    if (!pen_type.empty()) {
        int rc = prepare_penalties();
        if (rc) return rc;
    }
    if (form == SHAPE_FORM_PLAIN_FP64) {
        CK(cudaEventRecord(ev0, s));
        CK(cudaMemcpyAsync(d_r, h_params, sizeof(double) * npar(), cudaMemcpyHostToDevice, s));
        int rc = enqueue(form);
        if (rc) return rc;
        if (!pen_type.empty() && (rc = enqueue_model_sums()) != SHAPE_OK) return rc;
        CK(cudaEventRecord(ev1, s));
    } else {
        if (gexec[form] && graph_keep_pos[form] != keep_pos) {
            cudaGraphExecDestroy(gexec[form]);
            gexec[form] = nullptr;
        }
        if (!gexec[form]) {
            if (!tuned[form]) {
                if (tune_mode < 0) {
                    int rc = autotune(form);
                    if (rc) return rc;
                } else {
                    raster_variant[form] = (form == SHAPE_FORM_BATCHED_FP64 && !lcpts.empty()) ? 0 : tune_mode;
                    raster_persistent[form] = 0;
                    tuned[form] = 1;
                }
            }
            // baddiam factors are baked into the summary launch: graphs are
            // rebuilt if the flag changes (rare: a scale factor <= 0.01).
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            cudaMemcpyAsync(d_r, h_params, sizeof(double) * npar(), cudaMemcpyHostToDevice, s);
            int rc = enqueue(form);
            cudaError_t ce = cudaStreamEndCapture(s, &graph);
            if (rc) { if (ce == cudaSuccess) cudaGraphDestroy(graph); return rc; }
            CK(ce);
            CK(cudaGraphInstantiate(&gexec[form], graph, 0));
            cudaGraphDestroy(graph);
            graph_keep_pos[form] = keep_pos;
        }
        CK(cudaEventRecord(ev0, s));
        CK(cudaGraphLaunch(gexec[form], s));
        if (!pen_type.empty()) {
            int rc = enqueue_model_sums();
            if (rc) return rc;
        }
        CK(cudaEventRecord(ev1, s));
    }
    last_form = form;
    return SHAPE_OK;
}

// The raster grid of a batched launch: one CTA per tile that was non-empty
// at bin tuning, or (persistent) the kernel's resident CTAs on every SM,
// each striding over the sorted tiles.
int EngineImpl::raster_grid(int form, int nonempty, const RasterArgs &a, bool f32) const
{
    if (!raster_persistent[form] || nonempty <= 0) return nonempty;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
        return nonempty;
    const int occ = f32 ? raster_occupancy_f32(a) : raster_occupancy_f64(a);
    if (occ <= 0) return nonempty;
    return std::min(nonempty, occ * sms);
}

namespace {
// Raster choices by size class, shared by the engines of the process (the
// server's clones of one dataset tune once).
struct TuneKey {
    int device, form, exact, nviews, nf, nonempty, maxcount;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(device, form, exact, nviews, nf, nonempty, maxcount) <
               std::tie(o.device, o.form, o.exact, o.nviews, o.nf, o.nonempty, o.maxcount);
    }
};
struct TuneChoice {
    int variant, persistent;
    double ms[4];
};
std::mutex tune_mu;
std::map<TuneKey, TuneChoice> tune_cache;

// The tuning file (SHAPE_B200_TUNING_CACHE names it; none by default): one
// JSON object per line and size class, keyed by the GPU's name and SM count
// so that a file carried to another machine of the same kind is reused and
// one of another kind is ignored. Read once per device, rewritten whenever
// a new size class is tuned.
std::string gpu_tag(int device)
{
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, device) != cudaSuccess) return std::string();
    std::string name(pr.name);
    for (char &c : name)
        if (c == '"' || c == '\\') c = '_';
    return name + "/" + std::to_string(pr.multiProcessorCount);
}
std::set<int> tune_file_read;

void tune_file_load(int device)
{
    const char *path = getenv("SHAPE_B200_TUNING_CACHE");
    if (!path || !*path || tune_file_read.count(device)) return;
    tune_file_read.insert(device);
    FILE *fp = fopen(path, "r");
    if (!fp) return;
    const std::string tag = gpu_tag(device);
    char line[1024], gpu[256];
    while (fgets(line, sizeof line, fp)) {
        TuneKey k{};
        TuneChoice c{};
        if (sscanf(line,
                   "{\"gpu\": \"%255[^\"]\", \"form\": %d, \"exact\": %d, \"views\": %d, \"facets\": %d, "
                   "\"nonempty\": %d, \"maxcount16\": %d, \"variant\": %d, \"persistent\": %d, "
                   "\"ms\": [%lf, %lf, %lf, %lf]}",
                   gpu, &k.form, &k.exact, &k.nviews, &k.nf, &k.nonempty, &k.maxcount, &c.variant, &c.persistent,
                   &c.ms[0], &c.ms[1], &c.ms[2], &c.ms[3]) != 13)
            continue;
        if (tag != gpu || c.variant < 0 || c.variant > 1 || c.persistent < 0 || c.persistent > 1) continue;
        k.device = device;
        tune_cache.emplace(k, c);
    }
    fclose(fp);
}

void tune_file_save()
{
    const char *path = getenv("SHAPE_B200_TUNING_CACHE");
    if (!path || !*path) return;
    const std::string tmp = std::string(path) + ".tmp";
    FILE *fp = fopen(tmp.c_str(), "w");
    if (!fp) return;
    std::map<int, std::string> tags;
    for (const auto &kv : tune_cache) {
        const TuneKey &k = kv.first;
        const TuneChoice &c = kv.second;
        if (!tags.count(k.device)) tags[k.device] = gpu_tag(k.device);
        fprintf(fp,
                "{\"gpu\": \"%s\", \"form\": %d, \"exact\": %d, \"views\": %d, \"facets\": %d, "
                "\"nonempty\": %d, \"maxcount16\": %d, \"variant\": %d, \"persistent\": %d, "
                "\"ms\": [%.6g, %.6g, %.6g, %.6g]}\n",
                tags[k.device].c_str(), k.form, k.exact, k.nviews, k.nf, k.nonempty, k.maxcount, c.variant,
                c.persistent, c.ms[0], c.ms[1], c.ms[2], c.ms[3]);
    }
    fclose(fp);
    rename(tmp.c_str(), path);
}
}  // namespace

// Measures the raster stage of this form with each kernel and grid (one
// untimed and three timed eager runs each, the minimum kept) and keeps the
// fastest. Runs outside any capture, before the form's graph is built.
int EngineImpl::autotune(int form)
{
    const TuneKey key{device, form, form == SHAPE_FORM_BATCHED_FP32 ? fp32_exact : 0, nviews, nf,
                      tuned_nonempty, tuned_max_count / 16};
    {
        std::lock_guard<std::mutex> lk(tune_mu);
        tune_file_load(device);
        auto it = tune_cache.find(key);
        if (it != tune_cache.end()) {
            raster_variant[form] = it->second.variant;
            raster_persistent[form] = it->second.persistent;
            memcpy(tune_ms[form], it->second.ms, sizeof tune_ms[form]);
            tuned[form] = 1;
            return SHAPE_OK;
        }
    }
    cudaStream_t s = stream;
    CK(cudaMemcpyAsync(d_r, h_params, sizeof(double) * npar(), cudaMemcpyHostToDevice, s));
    cudaEvent_t ev[8];
    for (auto &x : ev) CK(cudaEventCreate(&x));
    int best = 0, rc = SHAPE_OK;
    double best_ms = 1e300;
    // the warp-independent kernel is a candidate for radar views only: a
    // batched FP64 launch that also holds lightcurve views keeps the
    // tile-per-CTA kernel
    const int ncand = (form == SHAPE_FORM_BATCHED_FP64 && !lcpts.empty()) ? 2 : 4;
    for (int c = 0; c < ncand && rc == SHAPE_OK; c++) {
        raster_variant[form] = c >> 1;
        raster_persistent[form] = c & 1;
        double m = 1e300;
        for (int rep = 0; rep < 4 && rc == SHAPE_OK; rep++) {
            rc = enqueue(form, ev);
            if (rc) break;
            cudaError_t ce = cudaStreamSynchronize(s);
            if (ce != cudaSuccess) { rc = set_err(SHAPE_E_CUDA, cudaGetErrorString(ce)); break; }
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[3], ev[4]);     // after bin -> after raster
            if (rep > 0) m = std::min(m, (double)t);
        }
        tune_ms[form][c] = m;
        if (m < best_ms) { best_ms = m; best = c; }
    }
    for (auto &x : ev) cudaEventDestroy(x);
    if (rc) return rc;
    raster_variant[form] = best >> 1;
    raster_persistent[form] = best & 1;
    tuned[form] = 1;
    std::lock_guard<std::mutex> lk(tune_mu);
    TuneChoice ch{raster_variant[form], raster_persistent[form], {}};
    memcpy(ch.ms, tune_ms[form], sizeof ch.ms);
    tune_cache[key] = ch;
    tune_file_save();
    return SHAPE_OK;
}

// 1 when the last launch has completed on the device, 0 otherwise.
int EngineImpl::poll()
{
    cudaError_t e = cudaEventQuery(ev1);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    return set_err(SHAPE_E_CUDA, std::string("cudaEventQuery: ") + cudaGetErrorString(e));
}

// Waits for the last launch and returns its summary.
int EngineImpl::finish(shape_eval_summary *out)
{
    CK(cudaEventSynchronize(ev1));
    CK(cudaEventElapsedTime(&last_ms, ev0, ev1));
    shape_eval_summary sm = *h_summary;
    sm.penalties = 0.0;
    if (!pen_type.empty()) {
        // objective() (src/shape/bestfit.c:789-866): reduced chi-square plus
        // penalties, then the bad-model factors
        if (h_msum[MSUM_SURF_ERR] != 0.0)
            return set_err(SHAPE_E_UNSUPPORTED, "check_surface: a ray crossed more than 100 facet edges");
        sm.penalties = penalty_sum(h_msum);
        double err = sm.chi2 / sm.dof + sm.penalties;
        if (pending_baddiam) err *= bad_objfactor * exp(pending_bdl);
        if (sm.posbnd) err *= bad_objfactor * exp(sm.posbnd_logfactor);
        if (sm.badposet) err *= bad_objfactor * exp(sm.badposet_logfactor);
        if (sm.badradar) err *= bad_objfactor * exp(sm.badradar_logfactor);
        sm.objective = err;
    } else if (pending_baddiam) {
        // bad-diameter factor depends only on the host-side scale factors
        const double bdl = pending_bdl;
        sm.objective = sm.chi2 / sm.dof * (bad_objfactor * exp(bdl));
        if (sm.posbnd) sm.objective *= bad_objfactor * exp(sm.posbnd_logfactor);
        if (sm.badposet) sm.objective *= bad_objfactor * exp(sm.badposet_logfactor);
        if (sm.badradar) sm.objective *= bad_objfactor * exp(sm.badradar_logfactor);
    }
    if (out) *out = sm;
    return SHAPE_OK;
}

}  // namespace shape

// ====================================================================== C ABI

using shape::EngineImpl;

extern "C" {

const char *shape_last_error(void) { return shape::g_err.c_str(); }
const char *shape_version(void) { return "shape-b200 0.2 (sm_100a)"; }

int shape_abi_sizes(size_t *out, int max)
{
    size_t v[] = {sizeof(shape_model_desc), sizeof(shape_radar_law), sizeof(shape_optical_law),
                  sizeof(shape_eval_params), sizeof(shape_deldop_frame), sizeof(shape_deldop_set),
                  sizeof(shape_lghtcrv_point), sizeof(shape_lghtcrv_set), sizeof(shape_deldop_result),
                  sizeof(shape_eval_summary), sizeof(shape_doppler_frame), sizeof(shape_doppler_set),
                  sizeof(shape_spin_state), sizeof(shape_ephem_point), sizeof(shape_poset_frame),
                  sizeof(shape_poset_set), sizeof(shape_poset_result)};
    int n = (int)(sizeof v / sizeof v[0]);
    for (int i = 0; i < n && i < max; i++) out[i] = v[i];
    return n;
}

int shape_engine_create(int device, shape_engine **out)
{
    if (!out) return shape::set_err(SHAPE_E_ARG, "null out");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return shape::set_err(SHAPE_E_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return shape::set_err(SHAPE_E_ARG, "bad device index");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    shape_engine *h = new shape_engine();
    h->impl.device = device;
    if (cudaStreamCreateWithFlags(&h->impl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&h->impl.ev0) != cudaSuccess || cudaEventCreate(&h->impl.ev1) != cudaSuccess) {
        delete h;
        return shape::set_err(SHAPE_E_CUDA, "stream/event creation failed");
    }
    *out = h;
    return SHAPE_OK;
}

void shape_engine_destroy(shape_engine *e)
{
    if (!e) return;
    cudaSetDevice(e->impl.device);
    delete e;
}

int shape_engine_set_model(shape_engine *h, const shape_model_desc *m)
{
    if (!h || !m || m->nv <= 0 || m->nf <= 0 || !m->a || !m->u || !m->r || !m->fv || !m->af_ptr)
        return shape::set_err(SHAPE_E_ARG, "set_model: invalid model description");
    EngineImpl &E = h->impl;
    E.nv = m->nv; E.nf = m->nf;
    E.a.assign(m->a, m->a + 3 * (size_t)m->nv);
    E.u.assign(m->u, m->u + 3 * (size_t)m->nv);
    E.r.assign(m->r, m->r + m->nv);
    // components: one (scale[]) or several (comp_*), each vertex's component
    // and each component's rotation matrix (euler2mat of its rotation
    // offsets, src/util/euler.c) and translation
    if (m->ncomp > 1) {
        if (!m->comp_nv || !m->comp_nf || !m->comp_scale || !m->comp_rot || !m->comp_off)
            return shape::set_err(SHAPE_E_ARG, "set_model: component arrays missing");
        long long sv = 0, sf = 0;
        for (int c = 0; c < m->ncomp; c++) {
            if (m->comp_nv[c] < 1 || m->comp_nf[c] < 1)
                return shape::set_err(SHAPE_E_ARG, "set_model: a component without vertices or facets");
            sv += m->comp_nv[c];
            sf += m->comp_nf[c];
        }
        if (sv != m->nv || sf != m->nf)
            return shape::set_err(SHAPE_E_ARG, "set_model: component sizes do not add up to nv / nf");
        E.ncomp = m->ncomp;
        E.scale.assign(m->comp_scale, m->comp_scale + 3 * (size_t)m->ncomp);
        E.vcomp.resize(m->nv);
        E.cxf.assign((size_t)shape::CXF_N * m->ncomp, 0.0);
        int v0 = 0;
        for (int c = 0; c < m->ncomp; c++) {
            for (int i = 0; i < m->comp_nv[c]; i++) E.vcomp[v0 + i] = c;
            v0 += m->comp_nv[c];
            double mm[3][3];
            const double *rot = m->comp_rot + 3 * (size_t)c, *off = m->comp_off + 3 * (size_t)c;
            shape::euler_zxz(mm, rot[0], rot[1], rot[2]);
            double *T = &E.cxf[(size_t)shape::CXF_N * c];
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++) T[3 * j + k] = mm[j][k];
            for (int j = 0; j < 3; j++) T[9 + j] = off[j];
            T[12] = (rot[0] == 0 && rot[1] == 0 && rot[2] == 0) ? 0.0 : 1.0;
            T[13] = (off[0] == 0.0 && off[1] == 0.0 && off[2] == 0.0) ? 0.0 : 1.0;
        }
    } else {
        E.ncomp = 1;
        E.scale.assign(m->scale, m->scale + 3);
        E.vcomp.clear();
        E.cxf.clear();
    }
    E.fv.assign(m->fv, m->fv + 3 * (size_t)m->nf);
    for (int k = 0; k < 3 * m->nf; k++)
        if (E.fv[k] < 0 || E.fv[k] >= m->nv) return shape::set_err(SHAPE_E_ARG, "set_model: facet vertex out of range");
    E.af_ptr.assign(m->af_ptr, m->af_ptr + m->nv + 1);
    int naf = E.af_ptr[m->nv];
    if (naf < 0 || E.af_ptr[0] != 0) return shape::set_err(SHAPE_E_ARG, "set_model: bad af_ptr");
    E.af_idx.assign(m->af_idx, m->af_idx + naf);
    for (int k = 0; k < naf; k++)
        if (E.af_idx[k] < 0 || E.af_idx[k] >= m->nf) return shape::set_err(SHAPE_E_ARG, "set_model: attached facet out of range");
    E.have_model = true;
    E.finalized = false;
    return SHAPE_OK;
}

int shape_engine_set_params(shape_engine *h, const shape_eval_params *p)
{
    if (!h || !p) return shape::set_err(SHAPE_E_ARG, "null argument");
    if (p->nsinc2 < 1 || p->sinc2width < 1) return shape::set_err(SHAPE_E_ARG, "nsinc2 and sinc2width must be >= 1");
    h->impl.params = *p;
    h->impl.finalized = false;
    return SHAPE_OK;
}

int shape_engine_add_deldop_set(shape_engine *h, const shape_deldop_set *set, int nframes,
                                const shape_deldop_frame *frames, const double *obs, const double *oov)
{
    if (!h || !set || nframes <= 0 || !frames || !obs || !oov)
        return shape::set_err(SHAPE_E_ARG, "add_deldop_set: invalid argument");
    EngineImpl &E = h->impl;
    shape::DdSetHost d;
    d.set = *set;
    d.frame0 = (int)E.frames.size();
    d.nframes = nframes;
    size_t off = 0;
    for (int k = 0; k < nframes; k++) {
        const shape_deldop_frame &F = frames[k];
        if (F.pos_n < 1 || F.ndel < 1 || F.ndop < 1 || !(F.km_per_pixel > 0))
            return shape::set_err(SHAPE_E_ARG, "add_deldop_set: bad frame size");
        E.frame_off.push_back((long long)E.obs.size());
        size_t D = (size_t)F.ndel * F.ndop;
        E.obs.insert(E.obs.end(), obs + off, obs + off + D);
        E.oov.insert(E.oov.end(), oov + off, oov + off + D);
        off += D;
        E.frames.push_back(F);
        E.fviews.emplace_back();
        E.frame_sdev.push_back(0.0);
        E.dof += F.dof;
        E.dof_deldop += F.dof;
    }
    E.setrecs.push_back(shape::SetRec{0, d.frame0, nframes});
    E.dd.push_back(d);
    E.finalized = false;
    return (int)E.setrecs.size() - 1;
}

// A delay-Doppler set whose frames are each rendered from several views
// (smearing, src/shape/calc_fits.c:475-594): views[f * nviews + k] is frame
// f's k-th view in the order the reference renders them, v0+1 .. v0+nviews
// modulo nviews, so the last is the view at the frame's epoch. A view
// supplies ae, oe, spin, deloff and dopoff (struct deldopview_t); the frame's
// other fields (sizes, weight, dof, calibration, COM and DC bins) are the
// epoch view's.
int shape_engine_add_deldop_set_views(shape_engine *h, const shape_deldop_set *set, int nframes, int nviews,
                                      const shape_deldop_frame *views, const double *obs, const double *oov)
{
    if (!h || !set || nframes <= 0 || nviews < 1 || !views || !obs || !oov)
        return shape::set_err(SHAPE_E_ARG, "add_deldop_set_views: invalid argument");
    std::vector<shape_deldop_frame> ep((size_t)nframes);
    for (int k = 0; k < nframes; k++) ep[k] = views[(size_t)k * nviews + nviews - 1];
    EngineImpl &E = h->impl;
    const int f0 = (int)E.frames.size();
    int rc = shape_engine_add_deldop_set(h, set, nframes, ep.data(), obs, oov);
    if (rc < 0 || nviews == 1) return rc;
    E.dd.back().nviews = nviews;
    for (int k = 0; k < nframes; k++) {
        const shape_deldop_frame *V = views + (size_t)k * nviews;
        std::vector<shape_deldop_frame> &fv = E.fviews[f0 + k];
        fv.assign(V, V + nviews);
        for (shape_deldop_frame &w : fv) {
            // the frame-level fields are the epoch view's
            shape_deldop_frame x = ep[k];
            memcpy(x.ae, w.ae, sizeof x.ae);
            memcpy(x.oe, w.oe, sizeof x.oe);
            memcpy(x.spin, w.spin, sizeof x.spin);
            x.deloff = w.deloff;
            x.dopoff = w.dopoff;
            w = x;
        }
    }
    return rc;
}

// A Doppler set runs as a delay-Doppler set of one-row frames (LONG_ORIG,
// spb = stride = 1, zero delay scale, delay bin 1), which reproduces
// pos2doppler's weights; the overflow spectrum is the Doppler frames' own.
int shape_engine_add_doppler_set(shape_engine *h, const shape_doppler_set *set, int nframes,
                                 const shape_doppler_frame *frames, const double *obs, const double *oov)
{
    if (!h || !set || nframes <= 0 || !frames || !obs || !oov)
        return shape::set_err(SHAPE_E_ARG, "add_doppler_set: invalid argument");
    if (!(set->dop_per_bin > 0)) return shape::set_err(SHAPE_E_ARG, "add_doppler_set: dop_per_bin must be > 0");
    EngineImpl &E = h->impl;
    shape::DdSetHost d;
    memset(&d.set, 0, sizeof d.set);
    d.set.del_per_pixel = 1.0;
    d.set.dop_per_pixel = set->dop_per_bin;
    d.set.Ftx = set->Ftx;
    d.set.dopscale = set->dopscale;
    d.set.codemethod = SHAPE_CODE_LONG_ORIG;
    d.set.spb = d.set.stride = 1;
    d.set.dopfftlen = 1;
    d.set.law = set->law;
    d.doppler = 1;
    d.frame0 = (int)E.frames.size();
    d.nframes = nframes;
    size_t off = 0;
    for (int k = 0; k < nframes; k++) {
        const shape_doppler_frame &P = frames[k];
        if (P.pos_n < 1 || P.ndop < 1 || !(P.km_per_pixel > 0))
            return shape::set_err(SHAPE_E_ARG, "add_doppler_set: bad frame size");
        shape_deldop_frame F;
        memset(&F, 0, sizeof F);
        F.pos_n = P.pos_n; F.km_per_pixel = P.km_per_pixel;
        memcpy(F.ae, P.ae, sizeof F.ae); memcpy(F.oe, P.oe, sizeof F.oe); memcpy(F.spin, P.spin, sizeof F.spin);
        F.deloff = 0.0; F.dopoff = P.dopoff;
        F.ndel = 1; F.ndop = P.ndop;
        F.delcom_vig = 1.0; F.dopcom_vig = P.dopcom_vig; F.dopDC_vig = 0.0;
        F.weight = P.weight; F.dof = P.dof; F.cal_floating = P.cal_floating; F.cal = P.cal;
        E.frame_off.push_back((long long)E.obs.size());
        E.obs.insert(E.obs.end(), obs + off, obs + off + P.ndop);
        E.oov.insert(E.oov.end(), oov + off, oov + off + P.ndop);
        off += (size_t)P.ndop;
        E.frames.push_back(F);
        E.fviews.emplace_back();
        E.frame_sdev.push_back(P.sdev);
        E.dof += P.dof;
        E.dof_doppler += P.dof;
    }
    E.setrecs.push_back(shape::SetRec{0, d.frame0, nframes});
    E.dd.push_back(d);
    E.finalized = false;
    return (int)E.setrecs.size() - 1;
}

int shape_engine_get_radar_overflow(shape_engine *h, double *out, int max)
{
    if (!h || !out) return shape::set_err(SHAPE_E_ARG, "null argument");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    const int n = std::min<int>(max, (int)E.fh.size());
    std::vector<double> dop(E.dop_frames.size() * shape::DOP_OVF_TERMS);
    if (!dop.empty()) {
        cudaError_t e = cudaMemcpy(dop.data(), E.d_ovf_out, sizeof(double) * dop.size(), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    }
    for (int f = 0; f < n; f++) {
        const int k = E.fh[f].dop_index;
        for (int j = 0; j < 4; j++) out[4 * f + j] = (k >= 0) ? dop[(size_t)k * shape::DOP_OVF_TERMS + j] : 0.0;
    }
    return n;
}

int shape_engine_add_lghtcrv_set(shape_engine *h, const shape_lghtcrv_set *set,
                                 const shape_lghtcrv_point *points)
{
    if (!h || !set || !points || set->ncalc < 1 || set->n < 1 || !set->x || !set->t || !set->obs ||
        !set->oneovervar)
        return shape::set_err(SHAPE_E_ARG, "add_lghtcrv_set: invalid argument");
    EngineImpl &E = h->impl;
    shape::LcSetHost L;
    L.set = *set;
    L.pt0 = (int)E.points.size();
    L.npts = set->ncalc;
    L.x.assign(set->x, set->x + set->ncalc);
    L.t.assign(set->t, set->t + set->n);
    L.obs.assign(set->obs, set->obs + set->n);
    L.oov.assign(set->oneovervar, set->oneovervar + set->n);
    L.set.x = L.set.t = L.set.obs = L.set.oneovervar = nullptr;
    for (int k = 0; k < set->ncalc; k++) {
        if (points[k].pos_n < 1 || !(points[k].km_per_pixel > 0))
            return shape::set_err(SHAPE_E_ARG, "add_lghtcrv_set: bad point size");
        E.points.push_back(points[k]);
    }
    E.dof += set->dof;
    E.dof_lghtcrv += set->dof;
    E.setrecs.push_back(shape::SetRec{1, (int)E.lc.size(), 1});
    E.lc.push_back(std::move(L));
    E.finalized = false;
    return (int)E.setrecs.size() - 1;
}

int shape_engine_add_poset_set(shape_engine *h, const shape_poset_set *set, int nframes,
                               const shape_poset_frame *frames, const double *obs, const double *oneovervar)
{
    if (!h || !set || nframes < 1 || !frames || !obs || !oneovervar)
        return shape::set_err(SHAPE_E_ARG, "add_poset_set: invalid argument");
    const int law = set->law.type;
    if (law != SHAPE_OPTLAW_LAMBERT && law != SHAPE_OPTLAW_LOMMEL && law != SHAPE_OPTLAW_KAASALAINEN)
        return shape::set_err(SHAPE_E_UNSUPPORTED, "add_poset_set: optical scattering law not supported");
    if (set->resample == SHAPE_RESAMPLE_BICUBIC)
        return shape::set_err(SHAPE_E_UNSUPPORTED, "add_poset_set: bicubic resampling is not supported");
    if (set->resample < SHAPE_RESAMPLE_NONE || set->resample > SHAPE_RESAMPLE_CUBICCONV)
        return shape::set_err(SHAPE_E_ARG, "add_poset_set: unknown resampling mode");
    EngineImpl &E = h->impl;
    shape::PosetHost H;
    H.set = *set;
    H.frame0 = E.nps_frames;
    size_t total = 0;
    for (int k = 0; k < nframes; k++) {
        const shape_poset_frame &F = frames[k];
        if (F.pos_n < 1 || !(F.km_per_pixel > 0) || F.ncol < 2 || F.nrow < 2 || !(F.fit_km_per_pixel > 0))
            return shape::set_err(SHAPE_E_ARG, "add_poset_set: bad frame size");
        if (set->resample == SHAPE_RESAMPLE_NONE && fabs(cos(F.northangle)) > 1.0e-10 &&
            fabs(sin(F.northangle)) > 1.0e-10)
            return shape::set_err(SHAPE_E_ARG, "add_poset_set: no interpolation with an oblique north angle");
        total += (size_t)F.ncol * F.nrow;
        H.frames.push_back(F);
    }
    H.obs.assign(obs, obs + total);
    H.oov.assign(oneovervar, oneovervar + total);
    for (const shape_poset_frame &F : H.frames) {
        E.dof += F.dof;
        E.dof_poset += F.dof;
    }
    E.setrecs.push_back(shape::SetRec{2, E.nps_frames, nframes});
    E.nps_frames += nframes;
    E.ps.push_back(std::move(H));
    E.finalized = false;
    return (int)E.setrecs.size() - 1;
}

int shape_engine_get_poset(shape_engine *h, int set, int frame, double *fit, double *brightness,
                           shape_poset_result *result)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "null engine");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    if (set < 0 || set >= (int)E.setrecs.size() || E.setrecs[set].type != 2)
        return shape::set_err(SHAPE_E_ARG, "get_poset: not a plane-of-sky set");
    const shape::SetRec &R = E.setrecs[set];
    if (frame < 0 || frame >= R.count) return shape::set_err(SHAPE_E_ARG, "get_poset: bad frame");
    const int g = R.first + frame;
    const shape::PosetFrameDev &D = E.psf[g];
    cudaSetDevice(E.device);
    cudaError_t e = cudaStreamSynchronize(E.stream);
    if (e == cudaSuccess && fit)
        e = cudaMemcpy(fit, E.d_ps_fit + D.img_base, sizeof(double) * (size_t)D.ncol * D.nrow,
                       cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && brightness) {
        const shape::LcPointDev &P = E.lcpts[D.point];
        const long long side = 2 * (long long)E.geoms[P.obs_view].n + 1;
        e = cudaMemcpy(brightness, E.d_ps_b + P.b_base, sizeof(double) * (size_t)(side * side),
                       cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess && result)
        e = cudaMemcpy(result, E.d_ps_res + g, sizeof(shape_poset_result), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, std::string("get_poset: ") + cudaGetErrorString(e));
    return SHAPE_OK;
}

int shape_engine_finalize(shape_engine *h)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "null engine");
    cudaSetDevice(h->impl.device);
    return h->impl.finalize();
}

int shape_engine_set_scale(shape_engine *h, int j, double value)
{
    if (!h || j < 0 || j >= 3 * h->impl.ncomp) return shape::set_err(SHAPE_E_ARG, "set_scale: bad index");
    h->impl.scale[j] = value;
    return SHAPE_OK;
}

int shape_engine_get_scale(shape_engine *h, int j, double *value)
{
    if (!h || !value || j < 0 || j >= 3 * h->impl.ncomp) return shape::set_err(SHAPE_E_ARG, "get_scale: bad index");
    *value = h->impl.scale[j];
    return SHAPE_OK;
}

int shape_engine_set_vertex_r(shape_engine *h, int i, double value)
{
    if (!h || i < 0 || i >= h->impl.nv) return shape::set_err(SHAPE_E_ARG, "set_vertex_r: bad index");
    h->impl.r[i] = value;
    return SHAPE_OK;
}

int shape_engine_get_vertex_r(shape_engine *h, int i, double *value)
{
    if (!h || !value || i < 0 || i >= h->impl.nv) return shape::set_err(SHAPE_E_ARG, "get_vertex_r: bad index");
    *value = h->impl.r[i];
    return SHAPE_OK;
}

int shape_engine_evaluate(shape_engine *h, int form, shape_eval_summary *out)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "null engine");
    cudaSetDevice(h->impl.device);
    return h->impl.evaluate(form, out);
}

int shape_engine_get_deldop_results(shape_engine *h, shape_deldop_result *out, int max)
{
    if (!h || !out) return shape::set_err(SHAPE_E_ARG, "null argument");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    int n = std::min<int>(max, (int)E.fh.size());
    if (n > 0) {
        cudaError_t e = cudaMemcpy(out, E.d_results, sizeof(shape_deldop_result) * n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    }
    return n;
}

int shape_engine_get_fit(shape_engine *h, int frame, double *fit)
{
    if (!h || !fit) return shape::set_err(SHAPE_E_ARG, "null argument");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    if (frame < 0 || frame >= (int)E.frames.size()) return shape::set_err(SHAPE_E_ARG, "bad frame");
    size_t D = (size_t)E.frames[frame].ndel * E.frames[frame].ndop;
    long long off = E.frame_off[frame];
    cudaError_t e;
    if (E.last_form == SHAPE_FORM_BATCHED_FP32) {
        std::vector<float> tmp(D);
        e = cudaMemcpy(tmp.data(), E.d_fit32 + off, sizeof(float) * D, cudaMemcpyDeviceToHost);
        for (size_t k = 0; k < D; k++) fit[k] = tmp[k];
    } else {
        e = cudaMemcpy(fit, E.d_fit64 + off, sizeof(double) * D, cudaMemcpyDeviceToHost);
    }
    if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    return SHAPE_OK;
}

int shape_engine_write_fitdat(shape_engine *h, int frame, double sdev, const char *path)
{
    if (!h || !path) return shape::set_err(SHAPE_E_ARG, "write_fitdat: null argument");
    if (!(sdev > 0.0)) return shape::set_err(SHAPE_E_ARG, "write_fitdat: sdev must be > 0");
    EngineImpl &E = h->impl;
    if (frame < 0 || frame >= (int)E.frames.size()) return shape::set_err(SHAPE_E_ARG, "write_fitdat: bad frame");
    const shape_deldop_frame &F = E.frames[frame];
    std::vector<double> fit((size_t)F.ndel * F.ndop);
    int rc = shape_engine_get_fit(h, frame, fit.data());
    if (rc) return rc;
    std::vector<shape_deldop_result> res(E.frames.size());
    rc = shape_engine_get_deldop_results(h, res.data(), (int)res.size());
    if (rc < 0) return rc;
    return shape_write_fitdat(path, F.ndel, F.ndop, fit.data(), res[frame].cal, sdev);
}

int shape_engine_keep_pos(shape_engine *h, int keep)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "null engine");
    h->impl.keep_pos = keep ? 1 : 0;
    return SHAPE_OK;
}

static int copy_pos(EngineImpl &E, int view, double *z, double *cose, double *cosi, int *facet)
{
    const shape::FrameGeom &g = E.geoms[view];
    size_t np = (size_t)g.side * g.side;
    bool f32 = (E.last_form == SHAPE_FORM_BATCHED_FP32);
    double *bufs[3] = {z, cose, cosi};
    void *src[3] = {E.d_pos_z, E.d_pos_cose, E.d_pos_cosi};
    for (int k = 0; k < 3; k++) {
        if (!bufs[k]) continue;
        cudaError_t e;
        if (f32 && k > 0 && g.kind == shape::VIEW_RADAR) {   // depth maps, and lightcurve views' cosines, are FP64 in both forms
            std::vector<float> tmp(np);
            e = cudaMemcpy(tmp.data(), (float *)src[k] + g.pos_base, sizeof(float) * np, cudaMemcpyDeviceToHost);
            for (size_t i = 0; i < np; i++) bufs[k][i] = tmp[i];
        } else {
            e = cudaMemcpy(bufs[k], (double *)src[k] + g.pos_base, sizeof(double) * np, cudaMemcpyDeviceToHost);
        }
        if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    }
    if (facet) {
        cudaError_t e = cudaMemcpy(facet, E.d_pos_f + g.pos_base, sizeof(int) * np, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    }
    return SHAPE_OK;
}

int shape_engine_get_pos(shape_engine *h, int frame, double *z, double *cose, int *facet)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "null engine");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    if (frame < 0 || frame >= (int)E.frames.size()) return shape::set_err(SHAPE_E_ARG, "bad frame");
    if (!E.keep_pos) return shape::set_err(SHAPE_E_STATE, "POS maps not kept (shape_engine_keep_pos)");
    return copy_pos(E, E.frame_view[frame], z, cose, nullptr, facet);
}

int shape_engine_get_lghtcrv_pos(shape_engine *h, int set, int point, double *z, double *cose,
                                 double *cosi, int *facet, double *zill, int *fill)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "null engine");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    if (set < 0 || set >= (int)E.setrecs.size() || E.setrecs[set].type != 1)
        return shape::set_err(SHAPE_E_ARG, "bad lightcurve set");
    const shape::LcSetHost &L = E.lc[E.setrecs[set].first];
    if (point < 0 || point >= L.npts) return shape::set_err(SHAPE_E_ARG, "bad point");
    const shape::LcPointDev &P = E.lcpts[L.pt0 + point];
    int rc = copy_pos(E, P.obs_view, z, cose, cosi, facet);
    if (rc) return rc;
    return copy_pos(E, P.sun_view, zill, nullptr, nullptr, fill);
}

int shape_engine_get_lghtcrv(shape_engine *h, int set, double *y, double *fit, double *cal, double *chi2)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "null engine");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    if (set < 0 || set >= (int)E.setrecs.size() || E.setrecs[set].type != 1)
        return shape::set_err(SHAPE_E_ARG, "bad lightcurve set");
    int k = E.setrecs[set].first;
    const shape::LcSetDev &L = E.lcdev[k];
    cudaError_t e = cudaSuccess;
    if (y) e = cudaMemcpy(y, L.y, sizeof(double) * L.npts, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && fit) e = cudaMemcpy(fit, L.fit, sizeof(double) * L.n, cudaMemcpyDeviceToHost);
    double o[4];
    if (e == cudaSuccess) e = cudaMemcpy(o, E.d_lc_out + 4 * k, sizeof o, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    if (cal) *cal = o[0];
    if (chi2) *chi2 = o[1];
    return SHAPE_OK;
}

int shape_engine_get_seen(shape_engine *h, unsigned char *seen)
{
    if (!h || !seen) return shape::set_err(SHAPE_E_ARG, "null argument");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    cudaError_t e = cudaMemcpy(seen, E.d_seen, E.nf, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    return SHAPE_OK;
}

int shape_engine_get_realized(shape_engine *h, double *x, double *vn, double *fn, double *area)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "null engine");
    EngineImpl &E = h->impl;
    if (E.last_form < 0) return shape::set_err(SHAPE_E_STATE, "no evaluation yet");
    std::vector<double4> tmp(std::max(E.nv, E.nf));
    cudaError_t e = cudaSuccess;
    if (x) {
        e = cudaMemcpy(tmp.data(), E.md.vx, sizeof(double4) * E.nv, cudaMemcpyDeviceToHost);
        for (int i = 0; i < E.nv; i++) { x[3 * i] = tmp[i].x; x[3 * i + 1] = tmp[i].y; x[3 * i + 2] = tmp[i].z; }
    }
    if (e == cudaSuccess && vn) {
        e = cudaMemcpy(tmp.data(), E.md.vn, sizeof(double4) * E.nv, cudaMemcpyDeviceToHost);
        for (int i = 0; i < E.nv; i++) { vn[3 * i] = tmp[i].x; vn[3 * i + 1] = tmp[i].y; vn[3 * i + 2] = tmp[i].z; }
    }
    if (e == cudaSuccess && fn) {
        e = cudaMemcpy(tmp.data(), E.md.fn, sizeof(double4) * E.nf, cudaMemcpyDeviceToHost);
        for (int i = 0; i < E.nf; i++) { fn[3 * i] = tmp[i].x; fn[3 * i + 1] = tmp[i].y; fn[3 * i + 2] = tmp[i].z; }
    }
    if (e == cudaSuccess && area) e = cudaMemcpy(area, E.md.area, sizeof(double) * E.nf, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(e));
    return SHAPE_OK;
}

int shape_engine_stage_times(shape_engine *h, int form, double *ms, int max)
{
    if (!h || !ms) return shape::set_err(SHAPE_E_ARG, "null argument");
    EngineImpl &E = h->impl;
    if (!E.finalized) return shape::set_err(SHAPE_E_STATE, "stage_times before finalize");
    if (form != SHAPE_FORM_BATCHED_FP64 && form != SHAPE_FORM_BATCHED_FP32)
        return shape::set_err(SHAPE_E_ARG, "stage_times: batched forms only");
    cudaSetDevice(E.device);
    cudaEvent_t ev[9];
    for (auto &x : ev) cudaEventCreate(&x);
    E.fill_params(E.h_params);
    E.fill_spin();
    cudaMemcpyAsync(E.d_r, E.h_params, sizeof(double) * E.npar(), cudaMemcpyHostToDevice, E.stream);
    cudaEventRecord(ev[0], E.stream);
    int rc = E.enqueue(form, ev + 1);
    cudaError_t ce = cudaStreamSynchronize(E.stream);
    int n = 0;
    if (rc == SHAPE_OK && ce == cudaSuccess) {
        for (int k = 0; k < 8 && k < max; k++, n++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            ms[k] = t;
        }
    }
    for (auto &x : ev) cudaEventDestroy(x);
    if (rc) return rc;
    if (ce != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(ce));
    E.last_form = form;
    return n;
}

int shape_engine_set_frame_view(shape_engine *h, int global_frame, const double ae[9], const double oe[9],
                                const double spin[3], double deloff, double dopoff)
{
    if (!h || !ae || !oe || !spin) return shape::set_err(SHAPE_E_ARG, "set_frame_view: null argument");
    shape::EngineImpl &E = h->impl;
    if (E.finalized) cudaSetDevice(E.device);
    return E.set_frame_view(global_frame, ae, oe, spin, deloff, dopoff);
}

int shape_engine_set_point_view(shape_engine *h, int point, const double ae[9], const double oe[9],
                                const double se[9])
{
    if (!h || !ae || !oe || !se) return shape::set_err(SHAPE_E_ARG, "set_point_view: null argument");
    shape::EngineImpl &E = h->impl;
    if (E.finalized) cudaSetDevice(E.device);
    return E.set_point_view(point, ae, oe, se);
}

int shape_engine_set_spin_model(shape_engine *h, const shape_spin_state *spin, const double *set_angleoff,
                                const double *set_omegaoff, const double *frame_t, const double *frame_orbspin)
{
    if (!h || !spin) return shape::set_err(SHAPE_E_ARG, "set_spin_model: null argument");
    shape::EngineImpl &E = h->impl;
    if (E.finalized) cudaSetDevice(E.device);
    return E.set_spin_model(*spin, set_angleoff, set_omegaoff, frame_t, frame_orbspin);
}

int shape_engine_set_spin_param(shape_engine *h, int kind, int index, double value)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "set_spin_param: null argument");
    shape::EngineImpl &E = h->impl;
    double *p = E.spin_param(kind, index);
    if (!p) return shape::set_err(E.have_spin ? SHAPE_E_ARG : SHAPE_E_STATE, "set_spin_param: no such spin parameter");
    const double old = *p;
    *p = value;
    if (E.spin_device && E.finalized) return SHAPE_OK;   // realized by the next evaluation
    if (E.finalized) cudaSetDevice(E.device);
    int rc = E.realize_views();
    if (rc) {                       // keep the last realizable state
        *p = old;
        E.realize_views();
    }
    return rc;
}

int shape_engine_get_spin_param(shape_engine *h, int kind, int index, double *value)
{
    if (!h || !value) return shape::set_err(SHAPE_E_ARG, "get_spin_param: null argument");
    double *p = h->impl.spin_param(kind, index);
    if (!p) return shape::set_err(h->impl.have_spin ? SHAPE_E_ARG : SHAPE_E_STATE,
                                  "get_spin_param: no such spin parameter");
    *value = *p;
    return SHAPE_OK;
}

int shape_engine_set_penalties(shape_engine *h, int n, const int *type, const double *weight)
{
    if (!h) return shape::set_err(SHAPE_E_ARG, "set_penalties: null argument");
    return h->impl.set_penalties(n, type, weight);
}

int shape_engine_get_penalties(shape_engine *h, double *base, int max)
{
    if (!h || (max > 0 && !base)) return shape::set_err(SHAPE_E_ARG, "get_penalties: null argument");
    const EngineImpl &E = h->impl;
    const int n = std::min<int>(max, (int)E.pen_base.size());
    for (int i = 0; i < n; i++) base[i] = E.pen_base[i];
    return (int)E.pen_base.size();
}

int shape_engine_get_active(shape_engine *h, unsigned char *vertex_act, unsigned char *facet_act)
{
    if (!h || !vertex_act || !facet_act) return shape::set_err(SHAPE_E_ARG, "get_active: null argument");
    EngineImpl &E = h->impl;
    if (E.last_form < 0 || E.pen_type.empty() || !E.d_sides)
        return shape::set_err(SHAPE_E_STATE, "get_active: no evaluation with penalties yet");
    if (E.ncomp == 1) {
        memset(vertex_act, 1, (size_t)E.nv);
        memset(facet_act, 1, (size_t)E.nf);
        return SHAPE_OK;
    }
    cudaSetDevice(E.device);
    cudaError_t e = cudaStreamSynchronize(E.stream);
    if (e == cudaSuccess) e = cudaMemcpy(vertex_act, E.d_act_v, (size_t)E.nv, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(facet_act, E.d_act_f, (size_t)E.nf, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, std::string("get_active: ") + cudaGetErrorString(e));
    return SHAPE_OK;
}

int shape_engine_set_fp32_exact(shape_engine *h, int exact)
{
    if (!h || (exact != 0 && exact != 1)) return shape::set_err(SHAPE_E_ARG, "set_fp32_exact: 0 or 1");
    shape::EngineImpl &E = h->impl;
    if (E.fp32_exact != exact && E.gexec[SHAPE_FORM_BATCHED_FP32]) {   // the captured graph has the other kernel
        cudaSetDevice(E.device);
        cudaGraphExecDestroy(E.gexec[SHAPE_FORM_BATCHED_FP32]);
        E.gexec[SHAPE_FORM_BATCHED_FP32] = nullptr;
    }
    if (E.fp32_exact != exact) E.tuned[SHAPE_FORM_BATCHED_FP32] = 0;
    E.fp32_exact = exact;
    return SHAPE_OK;
}

int shape_engine_set_spin_device(shape_engine *h, int on)
{
    if (!h || (on != 0 && on != 1)) return shape::set_err(SHAPE_E_ARG, "set_spin_device: 0 or 1");
    shape::EngineImpl &E = h->impl;
    if (E.finalized) cudaSetDevice(E.device);
    if (on == E.spin_device) return SHAPE_OK;
    E.invalidate_graphs();
    E.spin_device = on;
    if (!E.finalized) return SHAPE_OK;
    if (on) {
        int rc = E.setup_spin_device();
        if (rc) E.spin_device = 0;
        return rc;
    }
    // back to host realization: the host copies of the views are brought
    // up to date and uploaded
    E.n_spin_src = 0;
    return E.have_spin ? E.realize_views() : SHAPE_OK;
}

int shape_engine_get_frame_view(shape_engine *h, int global_frame, double ae[9], double spin[3])
{
    if (!h || !ae || !spin) return shape::set_err(SHAPE_E_ARG, "get_frame_view: null argument");
    shape::EngineImpl &E = h->impl;
    if (global_frame < 0 || global_frame >= (int)E.frames.size())
        return shape::set_err(SHAPE_E_ARG, "get_frame_view: frame out of range");
    shape_deldop_frame F = E.frames[global_frame];
    if (E.spin_device && E.finalized && E.n_spin_src > 0) {
        cudaSetDevice(E.device);
        cudaError_t ce = cudaMemcpyAsync(&F, E.d_frames_dev + global_frame, sizeof F, cudaMemcpyDeviceToHost, E.stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(E.stream);
        if (ce != cudaSuccess) return shape::set_err(SHAPE_E_CUDA, cudaGetErrorString(ce));
    }
    memcpy(ae, F.ae, sizeof F.ae);
    memcpy(spin, F.spin, sizeof F.spin);
    return SHAPE_OK;
}

// vary_params (src/shape/vary_params.c:84-327) from an FP64 evaluation of
// the current model: for the first dataset only, as the reference's loop
// over datasets stops after set 0 (vary_params.c:106), the dof-free sums of
// the subradar point's distance (delay-Doppler frames whose 0th
// delay-correction coefficient floats), the radar cross sections of frames
// with a fixed calibration, the lightcurve's fitted brightnesses when its
// calibration is fixed, and cos(subradar latitude) of frames whose Doppler
// scale floats, each weighted by the frame's (set's) weight; divided by the
// weight sums read_dat forms over every dataset
// (src/shape/read_dat.c:421-501, 686-692, 1051-1056, 1900-1906).
int shape_engine_vary_params(shape_engine *h, const shape_vary_options *opt, double out[4])
{
    if (!h || !opt || !out) return shape::set_err(SHAPE_E_ARG, "vary_params: null argument");
    EngineImpl &E = h->impl;
    if (!E.finalized) return shape::set_err(SHAPE_E_STATE, "vary_params before finalize");
    if (!E.ps.empty()) return shape::set_err(SHAPE_E_UNSUPPORTED, "vary_params: plane-of-sky sets");
    const int nsets = (int)E.setrecs.size();
    auto dfree = [&](const int *a, int s) { return a ? a[s] != 0 : false; };
    // the weight sums over every dataset
    double w_zmax = 0.0, w_xsec = 0.0, w_opt = 0.0, w_cos = 0.0;
    for (int s = 0; s < nsets; s++) {
        const shape::SetRec &R = E.setrecs[s];
        if (R.type == 0) {
            int ds = 0;
            while (ds < (int)E.dd.size() && E.dd[ds].frame0 != R.first) ds++;
            const bool dop = E.dd[ds].doppler != 0;
            for (int f = R.first; f < R.first + R.count; f++) {
                const shape_deldop_frame &F = E.frames[f];
                if (!dop && dfree(opt->delcor0_free, s)) w_zmax += F.weight;
                if (!F.cal_floating) w_xsec += F.weight;
                if (dfree(opt->dopscale_free, s)) w_cos += F.weight;
            }
        } else {
            const shape::LcSetHost &L = E.lc[R.first];
            if (!L.set.cal_floating) w_opt += L.set.weight * L.set.n;
        }
    }
    double sum_zmax = 0.0, sum_xsec = 0.0, sum_opt = 0.0, sum_cos = 0.0;
    if (nsets > 0) {
        const shape::SetRec &R = E.setrecs[0];
        if (R.type == 0 && !E.fviews[R.first].empty())
            return shape::set_err(SHAPE_E_UNSUPPORTED, "vary_params: the first dataset has smeared frames");
        if (E.finalized) cudaSetDevice(E.device);
        // the evaluation keeps its POS maps for the reads below; the
        // caller's setting comes back on every return path
        struct KeepPos {
            decltype(E.keep_pos) &ref, old;
            ~KeepPos() { ref = old; }
        } keep_guard{E.keep_pos, E.keep_pos};
        E.keep_pos = 1;
        shape_eval_summary sm;
        int rc = E.evaluate(SHAPE_FORM_PLAIN_FP64, &sm);
        if (rc) return rc;
        if (R.type == 0) {
            int ds = 0;
            while (ds < (int)E.dd.size() && E.dd[ds].frame0 != R.first) ds++;
            const bool dop = E.dd[ds].doppler != 0;
            const int nfr = (int)E.frames.size();
            std::vector<shape_deldop_result> res(nfr);
            if ((rc = shape_engine_get_deldop_results(h, res.data(), nfr)) < 0) return rc;
            std::vector<double> ovf(4 * (size_t)nfr);
            if ((rc = shape_engine_get_radar_overflow(h, ovf.data(), nfr)) < 0) return rc;
            for (int f = R.first; f < R.first + R.count; f++) {
                const shape_deldop_frame &F = E.frames[f];
                const bool zmax_on = opt->vary_delcor0 && !dop && dfree(opt->delcor0_free, 0);
                const bool xsec_on = opt->vary_radalb && !F.cal_floating;
                if (zmax_on) {
                    const int side = 2 * F.pos_n + 1;
                    std::vector<double> z((size_t)side * side), ce((size_t)side * side);
                    if ((rc = shape_engine_get_pos(h, f, z.data(), ce.data(), nullptr)) != SHAPE_OK) return rc;
                    double zmax = -SHAPE_HUGENUMBER;
                    const shape_deldop_result &r = res[f];
                    for (int x = r.xlim[0]; x <= r.xlim[1]; x++)
                        for (int y = r.ylim[0]; y <= r.ylim[1]; y++) {
                            const size_t p = (size_t)(x + F.pos_n) * side + (size_t)(y + F.pos_n);
                            if (ce[p] > 0.0) zmax = std::max(zmax, z[p]);
                        }
                    sum_zmax += zmax * F.weight;
                }
                if (xsec_on) {
                    std::vector<double> fit((size_t)F.ndel * F.ndop);
                    if ((rc = shape_engine_get_fit(h, f, fit.data())) != SHAPE_OK) return rc;
                    double xs = dop ? ovf[4 * (size_t)f + 2] : 0.0;    // overflow_xsec
                    for (double v : fit) xs += v;
                    xs *= res[f].cal;
                    sum_xsec += xs * F.weight;
                }
                if (opt->vary_dopscale && dfree(opt->dopscale_free, 0)) {
                    double oa[9];
                    shape::mul_bt(oa, F.oe, F.ae);
                    const double cd = sqrt(oa[6] * oa[6] + oa[7] * oa[7]);
                    sum_cos += cd * F.weight;
                }
            }
        } else if (opt->vary_optalb) {
            const shape::LcSetHost &L = E.lc[R.first];
            if (!L.set.cal_floating) {
                std::vector<double> y(L.set.ncalc), fit(L.set.n);
                double cal, chi2;
                if ((rc = shape_engine_get_lghtcrv(h, 0, y.data(), fit.data(), &cal, &chi2)) != SHAPE_OK) return rc;
                for (int i = 0; i < L.set.n; i++) sum_opt += fit[i] * L.set.weight;
            }
        }
    }
    out[0] = w_zmax > 0.0 ? sum_zmax / w_zmax : 0.0;
    out[1] = w_xsec > 0.0 ? sum_xsec / w_xsec : 0.0;
    out[2] = w_opt > 0.0 ? sum_opt / w_opt : 0.0;
    out[3] = w_cos > 0.0 ? sum_cos / w_cos : 0.0;
    return SHAPE_OK;
}

int shape_engine_set_raster_tuning(shape_engine *h, int mode)
{
    if (!h || mode < -1 || mode > 1) return shape::set_err(SHAPE_E_ARG, "set_raster_tuning: -1, 0 or 1");
    shape::EngineImpl &E = h->impl;
    if (E.finalized) cudaSetDevice(E.device);
    E.invalidate_graphs();
    E.tune_mode = mode;
    for (int f = 0; f < 3; f++) E.tuned[f] = 0;
    return SHAPE_OK;
}

int shape_engine_get_raster_tuning(shape_engine *h, int form, int *variant, int *persistent, double *ms)
{
    if (!h || form < 0 || form > 2) return shape::set_err(SHAPE_E_ARG, "get_raster_tuning: bad argument");
    const shape::EngineImpl &E = h->impl;
    if (variant) *variant = E.raster_variant[form];
    if (persistent) *persistent = E.raster_persistent[form];
    if (ms)
        for (int c = 0; c < 4; c++) ms[c] = E.tune_ms[form][c];
    return E.tuned[form];
}

int shape_engine_set_bin_capacity(shape_engine *h, int cap)
{
    if (!h || cap < 0 || cap > 65536) return shape::set_err(SHAPE_E_ARG, "set_bin_capacity: bad capacity");
    h->impl.fixed_cap = cap;
    h->impl.finalized = false;
    return SHAPE_OK;
}

int shape_engine_get_tuning(shape_engine *h, int *out, int max)
{
    if (!h || !out) return shape::set_err(SHAPE_E_ARG, "null argument");
    EngineImpl &E = h->impl;
    if (!E.finalized) return shape::set_err(SHAPE_E_STATE, "get_tuning before finalize");
    int v[5] = {E.cap, E.tuned_max_count, E.tuned_nonempty, E.ntiles, shape::TILE_W};
    int n = 0;
    for (; n < 5 && n < max; n++) out[n] = v[n];
    return n;
}

int shape_engine_kernels_per_eval(shape_engine *h, int form, int *count)
{
    if (!h || !count || form < 0 || form > 2) return shape::set_err(SHAPE_E_ARG, "bad argument");
    if (!h->impl.finalized) return shape::set_err(SHAPE_E_STATE, "kernels_per_eval before finalize");
    *count = h->impl.kernels_per_eval(form);
    return SHAPE_OK;
}

int shape_engine_last_time_ms(shape_engine *h, double *ms)
{
    if (!h || !ms) return shape::set_err(SHAPE_E_ARG, "null argument");
    *ms = h->impl.last_ms;
    return SHAPE_OK;
}

}  // extern "C"
