// EngineImpl: host-side state of one engine (model, datasets, device
// arenas, graphs). Shared by engine.cu (evaluation, C ABI) and server.cu
// (continuous-batching request loop).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.h"
#include "shape_b200.h"
#include "viewgeom.cuh"

namespace shape {

int report_error(int code, const std::string &msg);   // engine.cu

// A radar view's set-level pos2deldop constants (engine.cu); the
// view-level ones are in viewgeom.cuh.
void radar_set_consts(FrameGeom &g, const shape_deldop_set &S, const shape_eval_params &P, int law, int doppler);

struct DevMem {
    std::vector<void *> ptrs;
    std::vector<size_t> sizes;
    size_t bytes = 0;             // device bytes held (the engine's HBM footprint)
    template <typename T> int alloc(T **p, size_t count)
    {
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
        if (e != cudaSuccess)
            return report_error(SHAPE_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        ptrs.push_back(*p);
        sizes.push_back(count * sizeof(T));
        bytes += count * sizeof(T);
        return SHAPE_OK;
    }
    void release()
    {
        for (void *p : ptrs) cudaFree(p);
        ptrs.clear();
        sizes.clear();
        bytes = 0;
    }
    void release_one(void *p)
    {
        for (size_t k = 0; k < ptrs.size(); k++)
            if (ptrs[k] == p) {
                cudaFree(p);
                bytes -= sizes[k];
                ptrs.erase(ptrs.begin() + k);
                sizes.erase(sizes.begin() + k);
                return;
            }
    }
};

struct DdSetHost {
    shape_deldop_set set;       // a Doppler set is held as a one-row delay-Doppler set
    int frame0, nframes;
    int doppler = 0;            // 1: Doppler spectra (shape_engine_add_doppler_set)
    int nviews = 1;             // views per frame (smearing); frames[] holds each frame's epoch view
};
struct LcSetHost {
    shape_lghtcrv_set set;
    int pt0, npts;
    std::vector<double> x, t, obs, oov;
};

// A plane-of-sky set as added: its frames (global POS frame numbers from
// frame0) and their observed images back to back.
struct PosetHost {
    shape_poset_set set;
    std::vector<shape_poset_frame> frames;
    std::vector<double> obs, oov;
    int frame0;
};

struct EngineImpl {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // side branch of the batched graph (state reset, image clears, vertex
    // normals) and its fork / join events
    cudaStream_t stream2 = nullptr;   // batched graph branches: state reset and clears
    cudaStream_t stream3 = nullptr;   // ... and realize (vertices, facet and vertex normals)
    cudaEvent_t evf[4] = {nullptr, nullptr, nullptr, nullptr};
    float last_ms = 0.f;

    // model (host)
    int nv = 0, nf = 0;
    std::vector<double> a, u, r;
    // scale factors, 3 per component; several components: each vertex's
    // component and each component's transform (CXF_N doubles)
    int ncomp = 1;
    std::vector<double> scale = std::vector<double>(3, 1.0);
    std::vector<int> vcomp;
    std::vector<double> cxf;
    int *d_vcomp = nullptr;
    double *d_cxf = nullptr;
    int npar() const { return nv + 3 * ncomp; }   // free parameters uploaded per evaluation
    std::vector<int> fv, af_ptr, af_idx;
    bool have_model = false;
    shape_eval_params params{1, 1, 7, 0.0, 0.0, 1};
    double bad_objfactor = 2.0;

    // datasets (host)
    std::vector<DdSetHost> dd;
    std::vector<shape_deldop_frame> frames;
    // per frame: its views in the order the reference renders them (the
    // epoch view last); empty for a frame with one view
    std::vector<std::vector<shape_deldop_frame>> fviews;
    std::vector<long long> frame_off;   // element offsets into obs/oov/fit
    std::vector<double> obs, oov;
    std::vector<LcSetHost> lc;
    std::vector<shape_lghtcrv_point> points;
    std::vector<PosetHost> ps;          // plane-of-sky sets
    int nps_frames = 0;
    std::vector<SetRec> setrecs;
    std::vector<RadarLawDev> laws;
    double dof = 0, dof_deldop = 0, dof_doppler = 0, dof_lghtcrv = 0, dof_poset = 0;
    std::vector<double> frame_sdev;     // per radar frame: Doppler noise sdev (0 for delay-Doppler)

    // derived (host)
    std::vector<FrameGeom> geoms;
    std::vector<FrameHost> fh;
    std::vector<int2> work;                 // raster items
    std::vector<int> view_work0, view_nwork;
    std::vector<Chi2Item> chi2_items;
    std::vector<int> frame_view;
    std::vector<double> dop_extra, set_delpp, set_doppp;
    std::vector<LcPointDev> lcpts;
    std::vector<int2> lc_items;
    std::vector<int> pt_items;
    int nviews = 0, ntiles = 0;
    long long fit_elems = 0, pos_elems = 0;
    int cap = 512;

    // device
    bool finalized = false;
    DevMem mem;
    ModelDev md{};
    double *d_r = nullptr, *d_scale = nullptr, *d_a = nullptr, *d_u = nullptr;
    int *d_fv = nullptr, *d_afp = nullptr, *d_afi = nullptr;
    FrameGeom *d_geoms = nullptr;
    FrameState *d_states = nullptr;
    RadarLawDev *d_laws = nullptr;
    int2 *d_work = nullptr;
    double4 *d_vt64 = nullptr;
    int *d_bin_count = nullptr;
    int2 *d_bin_ids = nullptr;
    double *d_obs = nullptr, *d_oov = nullptr;
    double *d_fit64 = nullptr;
    float *d_fit32 = nullptr;
    void *d_pos_z = nullptr, *d_pos_cose = nullptr, *d_pos_cosi = nullptr;   // sized for double
    int *d_pos_f = nullptr;
    unsigned char *d_seen = nullptr;
    Chi2Item *d_chi2_items = nullptr;
    int *d_frame_view = nullptr;
    double *d_partials = nullptr;
    double *d_o2pre = nullptr;        // per chi-square item: o2 partial (model independent)
    int *d_chi2_counters = nullptr;   // fused chi-square / summary: per-frame items done, frames done
    bool fused_chi2 = false;          // batched forms run k_chi2_summary
    size_t fused_smem = 0;            // its dynamic shared memory
    FrameHost *d_fh = nullptr;
    shape_deldop_result *d_results = nullptr;
    double *d_set_delpp = nullptr, *d_set_doppp = nullptr, *d_dop_extra = nullptr;
    LcPointDev *d_lcpts = nullptr;
    int2 *d_lc_items = nullptr;
    int *d_pt_items = nullptr;
    double *d_lc_partials = nullptr;
    LcSetDev *d_lcsets = nullptr;
    double *d_lc_x = nullptr, *d_lc_t = nullptr, *d_lc_obs = nullptr, *d_lc_oov = nullptr;
    double *d_lc_y = nullptr, *d_lc_y2 = nullptr, *d_lc_fit = nullptr, *d_lc_out = nullptr;
    double *d_lc_dof = nullptr, *d_lc_npts = nullptr;
    // plane-of-sky frames: descriptors, images (obs, 1/var, fit), the sky
    // renderings' brightness and the per-frame results
    std::vector<PosetFrameDev> psf;
    std::vector<shape_lghtcrv_point> ps_points;   // the frames' view geometry, after the lightcurve points
    long long ps_img_elems = 0, ps_b_elems = 0;
    PosetFrameDev *d_psf = nullptr;
    double *d_ps_obs = nullptr, *d_ps_oov = nullptr, *d_ps_fit = nullptr, *d_ps_b = nullptr;
    shape_poset_result *d_ps_res = nullptr;
    SetRec *d_setrecs = nullptr;
    shape_eval_summary *d_summary_map = nullptr;   // device address of the mapped pinned h_summary
    std::vector<LcSetDev> lcdev;
    std::vector<int> dop_frames;        // global indices of the Doppler frames
    double *d_ovf = nullptr, *d_ovf_out = nullptr;
    int *d_dop_frames = nullptr;

    // penalty terms of the objective (shape_engine_set_penalties)
    std::vector<int> pen_type;
    std::vector<double> pen_weight, pen_base;
    int nsides = 0;                         // edges of the closed surface
    int4 *d_sides = nullptr;                // (v1, f1's third vertex, f1, f2); built on first use
    int *d_side_v2 = nullptr;               // several components: the edges' other ends
    int2 *d_comp_facets = nullptr;          // several components: (first facet, facets) each
    unsigned char *d_act_v = nullptr, *d_act_f = nullptr;   // check_surface's active flags
    int *d_surf_err = nullptr;
    double *d_msum_part = nullptr, *d_msum = nullptr;
    double *h_msum = nullptr;               // pinned [MSUM_N]
    int set_penalties(int n, const int *type, const double *weight);
    int prepare_penalties();
    int enqueue_model_sums();
    double penalty_sum(const double *ms);

    // pinned staging
    double *h_params = nullptr;             // r[nv], scale[3]
    shape_eval_summary *h_summary = nullptr;

    // graphs per form
    cudaGraphExec_t gexec[3] = {nullptr, nullptr, nullptr};
    int keep_pos = 0;
    int graph_keep_pos[3] = {0, 0, 0};
    int last_form = -1;

    ~EngineImpl() { release(); }

    void release()
    {
        for (auto &g : gexec)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        mem.release();
        if (h_params) { cudaFreeHost(h_params); h_params = nullptr; }
        if (h_summary) { cudaFreeHost(h_summary); h_summary = nullptr; }
        if (h_msum) { cudaFreeHost(h_msum); h_msum = nullptr; }
        if (h_spin) { cudaFreeHost(h_spin); h_spin = nullptr; }
        if (h_spin_off) { cudaFreeHost(h_spin_off); h_spin_off = nullptr; }
        if (ev0) { cudaEventDestroy(ev0); ev0 = nullptr; }
        if (ev1) { cudaEventDestroy(ev1); ev1 = nullptr; }
        for (auto &e : evf)
            if (e) { cudaEventDestroy(e); e = nullptr; }
        if (stream2) { cudaStreamDestroy(stream2); stream2 = nullptr; }
        if (stream3) { cudaStreamDestroy(stream3); stream3 = nullptr; }
        if (stream) { cudaStreamDestroy(stream); stream = nullptr; }
    }

    void invalidate_graphs()
    {
        for (auto &g : gexec)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    int finalize();
    int tune_bins();
    int set_frame_view(int fi, const double ae[9], const double oe[9], const double spin[3], double deloff,
                       double dopoff);
    int set_point_view(int pt, const double ae[9], const double oe[9], const double se[9]);
    // spin model of the views (shape_engine_set_spin_model)
    bool have_spin = false;
    shape_spin_state spin_st;
    std::vector<double> spin_angleoff, spin_omegaoff;   // 3 per dataset (setrecs order)
    std::vector<double> frame_t, frame_orbspin;         // per radar frame
    int set_spin_model(const shape_spin_state &sp, const double *ao, const double *oo, const double *t,
                       const double *orb);
    double *spin_param(int kind, int index);
    int realize_views();
    int refresh_views();
    // spin realization inside each evaluation (principal-axis rotators):
    // the graph copies the spin state and offsets from pinned memory and
    // k_realize_views rebuilds every view from them
    int spin_device = 0;
    int n_spin_src = 0;
    SpinViewSrc *d_spin_src = nullptr;
    shape_spin_state *d_spin = nullptr, *h_spin = nullptr;
    double *d_spin_off = nullptr, *h_spin_off = nullptr;
    shape_deldop_frame *d_frames_dev = nullptr;
    shape_deldop_set *d_ddsets = nullptr;
    shape_lghtcrv_point *d_points_dev = nullptr;
    int setup_spin_device();
    void fill_spin();
    int enqueue_spin();
    int enqueue(int form, cudaEvent_t *marks = nullptr);
    int launch(int form);
    int poll();
    int finish(shape_eval_summary *out);
    int pending_baddiam = 0;
    double pending_bdl = 0.0;
    size_t footprint() const { return mem.bytes + sizeof(double) * (size_t)npar() + sizeof(shape_eval_summary); }
    // copies the host description (model, switches, datasets) of another
    // engine; finalize() then builds this engine's own device state
    void clone_host_state(const EngineImpl &o)
    {
        nv = o.nv; nf = o.nf; a = o.a; u = o.u; r = o.r;
        scale = o.scale; ncomp = o.ncomp; vcomp = o.vcomp; cxf = o.cxf;
        fv = o.fv; af_ptr = o.af_ptr; af_idx = o.af_idx; have_model = o.have_model;
        params = o.params; bad_objfactor = o.bad_objfactor;
        dd = o.dd; frames = o.frames; frame_off = o.frame_off; obs = o.obs; oov = o.oov;
        fviews = o.fviews;
        lc = o.lc; points = o.points; setrecs = o.setrecs;
        ps = o.ps; nps_frames = o.nps_frames; dof_poset = o.dof_poset;
        dof = o.dof; dof_deldop = o.dof_deldop; dof_doppler = o.dof_doppler; dof_lghtcrv = o.dof_lghtcrv;
        frame_sdev = o.frame_sdev;
        fixed_cap = o.fixed_cap;
        fp32_exact = o.fp32_exact;
        tune_mode = o.tune_mode;
        have_spin = o.have_spin; spin_st = o.spin_st;
        spin_angleoff = o.spin_angleoff; spin_omegaoff = o.spin_omegaoff;
        frame_t = o.frame_t; frame_orbspin = o.frame_orbspin;
        spin_device = o.spin_device;
        finalized = false;
    }
    // bin tuning results
    int2 *d_work_sorted = nullptr;
    int tuned_max_count = 0, tuned_nonempty = 0;
    // the sorted work list holds radar tiles first (work_radar of them, the
    // first nonempty_radar non-empty at tuning), then lightcurve-view tiles
    // (nonempty_lc non-empty at tuning)
    int work_radar = 0, nonempty_radar = 0, nonempty_lc = 0;
    int fixed_cap = 0;            // > 0: bin capacity set by the caller, no autotuning
    int fp32_exact = 1;           // batched FP32: radar views by the exact raster variant too
    // Raster kernel per form (RasterArgs::variant) and grid (0: one CTA per
    // tile that was non-empty at bin tuning; 1: persistent, resident CTAs x
    // SMs striding over the tiles). tune_mode -1: the first batched
    // evaluation of a form measures the four candidates on this engine's
    // datasets and keeps the fastest (remembered per size class for other
    // engines of the process); 0 / 1: that kernel, one CTA per tile.
    int tune_mode = -1;
    int raster_variant[3] = {0, 0, 0};
    int raster_persistent[3] = {0, 0, 0};
    int tuned[3] = {0, 0, 0};
    double tune_ms[3][4] = {};    // raster ms of candidates (variant * 2 + persistent); 0: not measured
    int autotune(int form);
    int raster_grid(int form, int nonempty, const RasterArgs &a, bool f32) const;
    int evaluate(int form, shape_eval_summary *out);
    int kernels_per_eval(int form) const;
    void fill_params(double *dst) const
    {
        memcpy(dst, r.data(), sizeof(double) * nv);
        effective_scale(dst + nv, nullptr, nullptr);
    }
    // scale factors after realize_coordinates' SMALLRATIO guard
    // (src/shape/realize_mod.c:458-470; SMALLRATIO = 0.01, :138)
    void effective_scale(double *sc, int *baddiam, double *logf) const
    {
        int bd = 0;
        double lf = 0.0;
        for (int j = 0; j < 3 * ncomp; j++) {
            double v = scale[j];
            if (v <= 0.01) {
                bd = 1;
                lf += log(1 + 0.01 - v);
                v = 0.01 / (1 + 0.01 - v);
            }
            sc[j] = v;
        }
        if (baddiam) *baddiam = bd;
        if (logf) *logf = lf;
    }
};

}  // namespace shape

// the C ABI handle of an engine
struct shape_engine {
    shape::EngineImpl impl;
};
