// Kernel launchers of the SHAPE B200 engine (implemented in core.cu,
// raster_f64.cu, raster_f32.cu). All launches take the engine stream.
#pragma once

#include <cuda_runtime.h>

#include "engine_internal.h"
#include "shape_b200.h"

namespace shape {

// Programmatic dependent launch (batched forms): a kernel launched with
// launch_k(..., pdl = true) may be scheduled before the previous kernel on
// its stream has finished, and waits here, before its first access to that
// kernel's outputs, until it has (a no-op after an ordinary launch). The
// previous kernel does not trigger early, so waiting blocks take no SM
// slots from it; what is saved is the launch latency between the two.
#ifdef __CUDACC__
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
#endif

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl,
                     Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

// Per-component transform of a model with several components: the rotation
// matrix (9, row-major), the translation (3), whether to rotate and whether
// to translate (nonzero offsets), two spare slots.
constexpr int CXF_N = 16;

struct ModelDev {
    int nv, nf;
    const double *a, *u, *r, *scale;   // a,u: [nv*3]; scale: 3 per component
    const int *vcomp;                  // [nv] component of each vertex (null: one component)
    const double *cxf;                 // [ncomp * CXF_N] component transforms (null: one component)
    const int *fv;                     // [nf*3]
    const int *af_ptr, *af_idx;
    double4 *vx, *vn, *fn;             // realized
    double *area;
    int4 *fvi;                         // corner indices, padded
};

struct RasterArgs {
    const FrameGeom *geoms;
    const int2 *work;          // (view, tile) items
    int nwork;                 // items
    int grid;                  // CTAs (0: one per item); fewer CTAs stride over the rest
    int exact;                 // FP32 form: the exact variant (lightcurve views)
    int pdl;                   // programmatic dependent launch (launch_k)
    const void *vt;            // double4 view-frame vertices (both forms)
    const int4 *fvi;
    const double4 *vn;
    const double4 *fn;
    int nf;
    const int *bin_count;
    const int2 *bin_ids;        // (facet, tile-relative bbox) entries
    int cap;
    FrameState *states;
    const RadarLawDev *laws;
    void *fit;                 // T image arena (radar views)
    double *fit64;             // FP32 form: FP64 sums of the one-row (Doppler) frames, at their fit offsets
    void *pos_z, *pos_cose, *pos_cosi;  // POS maps: z double, cos(e) / cos(i) T (keep_pos or lightcurves)
    int *pos_f;
    unsigned char *seen;
    double mincosine_seen;
    int mark_seen;
    int keep_pos;
    double *ovf;               // Doppler overflow spectra (DOP_MAXOVERFLOW per Doppler frame)
    size_t smem_bytes;         // dynamic shared memory of the raster CTA (set by the launcher)
    // FP64 raster of a single view into images that already hold earlier
    // calls' results (posvis accumulating over model components): each pixel
    // starts from its z / facet / cos(e) / cos(i), and won[p] is set to 1
    // where this launch assigned pixel p. 0 for the engine's evaluations.
    int accumulate;
    unsigned char *won;
    // 0: the tile-per-CTA kernel (k_raster: the CTA's warps share one
    // sorted facet list and meet at block barriers); 1: the warp-independent
    // kernel (k_raster_w: each warp sorts and replays its own block's list)
    int variant;
    // FP32 form: the launch holds only lightcurve views, whose cosines the
    // exact variant recomputes in FP64 (a separate instantiation, so radar
    // launches carry none of it)
    int lc_views;
};

// core.cu (FP64, no FMA contraction)
void launch_realize(const ModelDev &m, cudaStream_t s);      // launch_realize_vf + launch_realize_vn
void launch_realize_vf(const ModelDev &m, cudaStream_t s);   // vertices, facet normals and areas
void launch_realize_vn(const ModelDev &m, cudaStream_t s);   // vertex normals (after _vf)

// Model sums for the penalty terms (penalty.cu), in this order.
// The sums run over the model's active facets, edges and vertices: all of
// them for one component; for several, those check_surface leaves active
// (not inside another component), with the counts of active edges and
// vertices and check_surface's error flag (an edge-crossing list overflow).
enum {
    MSUM_VOLUME, MSUM_COM, MSUM_IXX = MSUM_COM + 3, MSUM_IYY, MSUM_IZZ, MSUM_IXY, MSUM_IXZ, MSUM_IYZ,
    MSUM_NONSMOOTH, MSUM_CONCAVITY, MSUM_RDEV, MSUM_RDEV_MAX, MSUM_NSIDES, MSUM_NVERT, MSUM_SURF_ERR, MSUM_N
};
struct ModelSumArgs {
    ModelDev m;                 // realized model (vx, fn, fv, u, r, scale, vcomp)
    const int4 *sides;          // edges: (end vertex v1, f1's third vertex, f1, f2)
    const int *side_v2;         // the edges' other end vertices (several components)
    int nsides;
    int ncomp;
    const int2 *comp_facets;    // [ncomp] (first facet, facets) of each component
    unsigned char *act_v, *act_f;   // check_surface's flags (null: one component, all active)
    int *surf_err;              // check_surface's error flag (zeroed before it runs)
    double *part;               // [model_sums_blocks() * MSUM_N]
    double *out;                // [MSUM_N]
};
int model_sums_blocks();
void launch_model_sums(const ModelSumArgs &a, cudaStream_t s);   // two launches
void launch_check_surface(const ModelSumArgs &a, cudaStream_t s);   // several components: the active flags
void launch_reset_state(FrameState *st, int nviews, int *bin_count, int ntiles, cudaStream_t s);
// pdl: programmatic dependent launch (launch_k)
void launch_xform_f64(const FrameGeom *g, int nviews, const double4 *vx, int nv, double4 *vt,
                      cudaStream_t s, bool pdl = false);
// the transform of vertices realized on the fly (no dependency on k_realize_vf)
void launch_xform_realize_f64(const FrameGeom *g, int nviews, const ModelDev &m, double4 *vt, cudaStream_t s);
void launch_bin_f64(const FrameGeom *g, int view0, int nviews, const ModelDev &m, const double4 *vt,
                    FrameState *st, int *bin_count, int2 *bin_ids, int cap, cudaStream_t s, bool pdl = false);

struct Chi2Item { int frame; int start; int count; };
struct Chi2Args {
    const Chi2Item *items;
    int nitems;
    const double *obs, *oov;
    const void *fit;             // double or float
    const FrameGeom *geoms;      // radar views (for fit_base)
    const int *frame_view;       // global deldop frame -> view index
    double *partials;            // [nitems * 6]: o2, m2, om + compensations
    // [nitems * 2]: each item's o2 partial (sum and compensation), computed
    // once per dataset by the same code; null: o2 is summed per launch
    const double *o2pre;
};
void launch_chi2_partials(const Chi2Args &a, int fp32, cudaStream_t s);

struct FrameHost {             // per radar frame constants for finalize
    double weight, dof, cal_in;
    int cal_floating, badradar;
    double badradar_logfactor;
    int view;
    int set;
    int item0, nitems;
    int dop_index;             // Doppler frame: index of its overflow terms, else -1
    double sdev;               // Doppler frame: receiver noise sdev (overflow variance)
    // smeared frames (src/shape/calc_fits.c:475-594): views, whether any
    // view's footprint was too wide, and the sum of those views'
    // badradar log-factors (the objective adds dof * sum / views); the
    // frame's own badradar and badradar_logfactor are its epoch view's
    int nviews;
    int badradar_any;
    double badradar_lfsum;
};
struct FinalizeArgs {
    int nframes;
    const FrameHost *fh;
    const FrameGeom *geoms;
    const FrameState *states;
    const double *partials;
    shape_deldop_result *results;
    const double *set_delpp, *set_doppp;     // per set del/dop per pixel
    const double *dop_extra;                 // per frame
    const double *ovf_out;                   // per Doppler frame: DOP_OVF_TERMS values
};

// Doppler overflow spectra (src/shape/pos2doppler.c:451-499): per Doppler
// frame o2, m2, xsec, mean bin, and the badradar flag and log-factor of a
// model wider than the overflow spectrum.
constexpr int DOP_OVF_TERMS = 6;
struct DopOvfArgs {
    int n;                      // Doppler frames
    const int *frames;          // their global radar frame indices
    const FrameHost *fh;
    const FrameGeom *geoms;
    const FrameState *states;
    const double *ovf;          // overflow spectra
    double *out;                // [n * DOP_OVF_TERMS]
};
// FP32 form: the Doppler frames' FP64 sums rounded into the float fit
// images the chi-square reads (one block per Doppler frame).
void launch_dop_fit_f32(const int *dop_frames, int n, const FrameHost *fh, const FrameGeom *geoms,
                        const double *fit64, float *fit32, cudaStream_t s);
void launch_doppler_overflow(const DopOvfArgs &a, cudaStream_t s);

struct LcArgs {
    int npoints;
    const LcPointDev *pts;
    const FrameGeom *geoms;
    const FrameState *states;
    const int2 *items;          // (point, pixel start) work items
    int nitems;
    int chunk;                  // pixels per item
    const double *z, *zill;     // POS depth maps (FP64 in both forms)
    const void *cosi;           // T POS map
    void *cose;                 // masked in place, as posmask does
    const int *f, *fill;
    double *partials;           // brightness partial per item
    double *bimg;               // brightness images of plane-of-sky frames (LcPointDev::b_base)
    unsigned char *seen;
    double mincosine_seen;
    int mark_seen;
};
void launch_lc_photo(const LcArgs &a, int fp32, cudaStream_t s);

struct LcSetDev {
    int npts, n;                // calc points, observed points
    int pt0;                    // first calc point (global)
    int item0, nitems;          // photo items of this set's points are contiguous
    const double *x, *t, *obs, *oov;  // device arrays
    double *y, *y2, *fit;       // device outputs
    double weight, dof, cal_in;
    int cal_floating;
};
struct LcFinalizeArgs {
    int nsets;
    const LcSetDev *sets;
    const LcPointDev *pts;
    const FrameGeom *geoms;
    const FrameState *states;
    const int *pt_items;        // per point: first item, count (2 ints)
    const double *partials;
    double *set_out;            // per set: cal, chi2, posbnd flag, logfactor sum
    size_t smem_per_set;        // dynamic shared memory (lc_finalize_smem of the largest set), 0: global
};
constexpr size_t LC_FINALIZE_SMEM_MAX = 160 * 1024;
size_t lc_finalize_smem(int npts, int n);
cudaError_t configure_lc_finalize();
void launch_lc_finalize(const LcFinalizeArgs &a, cudaStream_t s);

// Spin realization inside an evaluation (spin.cu; principal-axis
// rotators): one thread per radar frame (its epoch view) or lightcurve point
// realizes ae (and a frame's spin vector) from the device spin state and
// its dataset's offsets, then the view constants as the host sets them.
struct SpinViewSrc {
    int kind;                   // 0 radar frame, 1 lightcurve point
    int index;                  // global radar frame or point index
    int rec;                    // dataset record: offsets at off[6 rec ..]
    int dd;                     // delay-Doppler set of a radar frame
    double t;                   // epoch (light-time corrected)
    double orb[3];              // orbital spin contribution (radar frames)
};
struct SpinRealizeArgs {
    int n;
    const SpinViewSrc *src;
    const shape_spin_state *spin;
    const double *off;                 // per record: angleoff[3], omegaoff[3]
    shape_deldop_frame *frames;        // ae and spin written
    const shape_deldop_set *ddsets;
    shape_lghtcrv_point *points;       // ae written
    FrameGeom *geoms;
    FrameHost *fh;
    double *dop_extra;
    LcPointDev *lcpts;
};
void launch_realize_views(const SpinRealizeArgs &a, cudaStream_t s);

struct SetRec { int type; int first; int count; };   // type 0 deldop (frames), 1 lightcurve (set index), 2 plane-of-sky (frames)

// Plane-of-sky frames (calc_poset after apply_photo, and chi2_poset): one
// block per frame resamples the brightness image onto the fit grid,
// checks that the grid holds every lit pixel and forms the chi-square.
struct PosetArgs {
    int nframes;
    const PosetFrameDev *frames;
    const LcPointDev *pts;
    const FrameGeom *geoms;
    const FrameState *states;
    const double *bimg;         // brightness images
    const double *obs, *oov;    // observed images and 1/variance
    double *fit;                // fit images
    shape_poset_result *res;    // per-frame results
};
void launch_poset_frames(const PosetArgs &a, cudaStream_t s);
struct SummaryArgs {
    int nsets;
    const SetRec *sets;
    const FrameHost *fh;
    const shape_deldop_result *results;
    const double *lc_out;       // per lightcurve set: cal, chi2, posbnd, logfactor sum
    const double *lc_dof;
    const double *lc_npts;
    const shape_poset_result *ps_res;   // plane-of-sky frames' results
    const PosetFrameDev *ps_frames;
    double dof_poset;           // plane-of-sky dof (calc_fits.c:408)
    double dof, dof_radar;      // all data / delay-Doppler + Doppler (calc_fits.c:409)
    double bad_objfactor;
    int baddiam;
    double baddiam_logfactor;
    shape_eval_summary *out;
    int nitems;                 // chi-square partial items (6 doubles each)
    int smem_frames;            // set by launch_summary: per-frame terms staged in shared memory
    int smem_partials;          // set by launch_summary: partials staged in shared memory too
};
constexpr size_t SUMMARY_SMEM_MAX = 160 * 1024;
size_t summary_smem(int nframes, int nitems, int *with_partials);
cudaError_t configure_summary();
// per-frame finalize (as launch_finalize_frames) fused with the totals
void launch_summary(const FinalizeArgs &fa, const SummaryArgs &a, cudaStream_t s);

// Chi-square partials + per-frame finalize + totals in one launch (the
// batched forms). Its shared staging (chi2_summary_smem bytes of dynamic
// shared memory) holds one frame's partials and then every frame's terms;
// chi2_summary_fits says whether a dataset fits in FUSED_STAGE_BYTES.
constexpr size_t FUSED_STAGE_BYTES = 24 * 1024;
size_t chi2_summary_smem(int nframes, int max_frame_items);
bool chi2_summary_fits(int nframes, int max_frame_items);
// counters: nframes + 1 ints, zero before the launch
void launch_chi2_summary(const Chi2Args &ca, const FinalizeArgs &fa, const SummaryArgs &sa, int *counters,
                         int fp32, cudaStream_t s, bool pdl, size_t smem);

// raster_f64.cu / raster_f32.cu
void launch_raster_f64(const RasterArgs &a, cudaStream_t s);
void launch_raster_f32(const RasterArgs &a, cudaStream_t s);
// resident CTAs per SM of the raster kernel these arguments select
int raster_occupancy_f64(const RasterArgs &a);
int raster_occupancy_f32(const RasterArgs &a);
cudaError_t configure_raster_f64();
cudaError_t configure_raster_f32();

}  // namespace shape
