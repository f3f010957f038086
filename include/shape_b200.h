/*
 * SHAPE model-evaluation engine for NVIDIA B200 (sm_100a): C ABI.
 *
 * The engine replaces the reference's CPU hot path
 *   realize_mod -> posclr/posvis -> pos2deldop / posmask+apply_photo
 *   -> calc_fits -> chi2
 * (h6294443/shape-cuda-v1.2: src/shape/realize_mod.c:153,
 * src/shape/posvis.c:84, src/shape/pos2deldop.c:176,
 * src/shape/posmask.c:58, src/shape/apply_photo.c:78,
 * src/shape/calc_fits.c:340, src/shape/chi2.c:240) with device-resident
 * model and frame state. A shim compiled into the reference program
 * converts struct mod_t / dat_t / par_t into the plain descriptions of
 * shape_types.h once, then calls shape_engine_evaluate where objective()
 * called calc_fits + chi2 (src/shape/bestfit.c:789-790).
 *
 * Conventions: every function returns SHAPE_OK (0) or a negative
 * SHAPE_E_* status; shape_last_error() gives a message for the calling
 * thread. Pointer arguments are plain host memory (pinned or not), except
 * the d_-prefixed arguments of shape_chi2_frames_noalloc, which are device
 * pointers the caller owns; no call returns a device pointer. An engine handle is bound to one CUDA
 * device and one stream; it is not thread-safe (use one handle per thread),
 * which matches the reference's single-threaded calc_fits.
 */
#ifndef SHAPE_B200_H
#define SHAPE_B200_H

#include <stddef.h>
#include "shape_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SHAPE_OK 0
#define SHAPE_E_ARG -1        /* invalid argument */
#define SHAPE_E_CUDA -2       /* CUDA runtime error (message in shape_last_error) */
#define SHAPE_E_STATE -3      /* call out of order (e.g. evaluate before finalize) */
#define SHAPE_E_UNSUPPORTED -4/* law / mode not supported by the device path */
#define SHAPE_E_NOMEM -5      /* device memory exhausted */
#define SHAPE_E_TIMEOUT -6    /* bounded wait expired */

/* Evaluation forms. */
#define SHAPE_FORM_PLAIN_FP64 0   /* per-frame launch sequence, FP64 end to end:
                                     facet maps bit-exact with the reference */
#define SHAPE_FORM_BATCHED_FP64 1 /* all frames per launch, CUDA graph, FP64 */
#define SHAPE_FORM_BATCHED_FP32 2 /* all frames per launch, CUDA graph, FP32
                                     raster/synthesis, FP64 rotations and
                                     compensated FP64 chi-square */

typedef struct shape_engine shape_engine;

/* Totals of one evaluation: what calc_fits leaves in par and chi2 returns. */
typedef struct shape_eval_summary {
    double chi2;               /* dat->chi2 (src/shape/chi2.c:392) */
    double dof;                /* dat->dof */
    double chi2_deldop, chi2_lghtcrv;
    int posbnd;                /* par->posbnd */
    double posbnd_logfactor;   /* par->posbnd_logfactor after /= dat->dof */
    int badradar;              /* par->badradar */
    double badradar_logfactor; /* after /= (dof_deldop + dof_doppler) */
    double objective;          /* (chi2/dof + penalties) times the bad-model
                                  factors, as objective() computes it
                                  (src/shape/bestfit.c:789-866) */
    double penalties;          /* the penalty sum (shape_engine_set_penalties;
                                  0 with none) */
    double chi2_poset;         /* plane-of-sky sets' part of chi2 */
    int badposet;              /* par->badposet */
    double badposet_logfactor; /* par->badposet_logfactor after /= dat->dof_poset */
} shape_eval_summary;

const char *shape_last_error(void);
const char *shape_version(void);
/* sizeof() of every struct in shape_types.h, in the order
 * model_desc, radar_law, optical_law, eval_params, deldop_frame,
 * deldop_set, lghtcrv_point, lghtcrv_set, deldop_result, eval_summary,
 * doppler_frame, doppler_set, spin_state, ephem_point, poset_frame,
 * poset_set, poset_result;
 * lets bindings verify their layouts. Returns the number written. */
int shape_abi_sizes(size_t *out, int max);

/* Create an engine on CUDA device `device`. */
int shape_engine_create(int device, shape_engine **out);
void shape_engine_destroy(shape_engine *e);

/* Model and datasets; replaces read_mod/read_dat's in-memory result. */
int shape_engine_set_model(shape_engine *e, const shape_model_desc *m);
int shape_engine_set_params(shape_engine *e, const shape_eval_params *p);
/* Appends a delay-Doppler set; obs and oneovervar hold every frame's
 * ndel*ndop image back to back. Returns the set index (>= 0) or a status. */
int shape_engine_add_deldop_set(shape_engine *e, const shape_deldop_set *set,
                                int nframes, const shape_deldop_frame *frames,
                                const double *obs, const double *oneovervar);
/* Appends a delay-Doppler set whose frames are each rendered from nviews
 * views (smearing, src/shape/calc_fits.c:475-594; the views of read_dat's
 * deldopview_t, src/shape/read_dat.c:868-899). views[f*nviews + k] is frame
 * f's k-th view in the reference's rendering order (v0+1 .. v0+nviews modulo
 * nviews), so the last one is the view at the frame's epoch; each view gives
 * ae, oe, spin, deloff and dopoff, and the epoch view gives the frame's other
 * fields. The fit image is the mean over the views; posbnd, the image limits
 * and the seen marks are the epoch view's; each view whose footprint is too
 * wide adds dof * log-factor / nviews to the badradar term. A frame with
 * several views refuses shape_engine_set_frame_view, and an engine holding
 * one refuses shape_engine_set_spin_model (SHAPE_E_UNSUPPORTED). */
int shape_engine_add_deldop_set_views(shape_engine *e, const shape_deldop_set *set, int nframes, int nviews,
                                      const shape_deldop_frame *views, const double *obs,
                                      const double *oneovervar);
int shape_engine_add_lghtcrv_set(shape_engine *e, const shape_lghtcrv_set *set,
                                 const shape_lghtcrv_point *points);
/* Appends a Doppler set (calc_doppler / pos2doppler / chi2_doppler,
 * src/shape/calc_fits.c:830, src/shape/pos2doppler.c:149,
 * src/shape/chi2.c:722); obs and oneovervar hold every frame's ndop bins back
 * to back. Its frames join the radar frames (fit, results, POS maps) as
 * 1 x ndop images; footprints that leave a spectrum go to its overflow
 * spectrum, whose chi-square terms enter the frame's o2 and m2. Returns the
 * set index (>= 0) or a status. */
int shape_engine_add_doppler_set(shape_engine *e, const shape_doppler_set *set,
                                 int nframes, const shape_doppler_frame *frames,
                                 const double *obs, const double *oneovervar);
/* A plane-of-sky set (calc_poset, src/shape/calc_fits.c:1156-1330, and
 * chi2_poset, src/shape/chi2.c): each frame is rendered from the observer
 * and from the sun (shadows by posmask), its brightness per POS pixel taken
 * by apply_photo, the brightness image resampled onto the frame's fit grid
 * by resampim (COM offsets, north angle, interpolation mode, rebinning),
 * checked by checkposet (badposet) and compared with the observed image
 * under a floating calibration. obs / oneovervar: the frames' ncol x nrow
 * images back to back (layout of shape_poset_frame). Bicubic resampling
 * returns SHAPE_E_UNSUPPORTED. Returns the set index. */
int shape_engine_add_poset_set(shape_engine *e, const shape_poset_set *set, int nframes,
                               const shape_poset_frame *frames, const double *obs, const double *oneovervar);
/* A plane-of-sky frame after the last evaluation: its fit image (ncol x
 * nrow, the layout of obs), its sky rendering's brightness image
 * ((2 pos_n + 1)^2, element (i, j) for i, j = -pos_n..pos_n at
 * (i + pos_n) * (2 pos_n + 1) + (j + pos_n), as pos->b[i][j]) and its
 * results; a NULL pointer skips that output. */
int shape_engine_get_poset(shape_engine *e, int set, int frame, double *fit, double *brightness,
                           shape_poset_result *result);

/* Allocates device state for everything added so far. */
int shape_engine_finalize(shape_engine *e);

/* Free parameters (src/shape/mkparlist.c:218-235): scale factor j (SIZEPAR;
 * j = 3 * component + axis for a model of several components) and vertex
 * deviation r of vertex i (SHAPEPAR; model-wide vertex index). */
int shape_engine_set_scale(shape_engine *e, int j, double value);
int shape_engine_set_vertex_r(shape_engine *e, int i, double value);
int shape_engine_get_vertex_r(shape_engine *e, int i, double *value);

/* One objective evaluation: realize_mod + calc_fits + chi2 on the device.
 * The model state set above goes host->device inside the call; the summary
 * comes back device->host. */
int shape_engine_evaluate(shape_engine *e, int form, shape_eval_summary *out);

/* Results of the last evaluation (device->host copies). Radar frames
 * (delay-Doppler and Doppler) in dataset order. */
int shape_engine_get_deldop_results(shape_engine *e, shape_deldop_result *out, int max);
/* Overflow-spectrum terms of the radar frames of the last evaluation, 4 per
 * frame: overflow_o2, overflow_m2, overflow_xsec, overflow_dopmean
 * (struct dopfrm_t, src/shape/shape2.h:1253-1256); zeros for delay-Doppler
 * frames, whose overflow terms the reference leaves at zero. Returns the
 * number of frames written. */
int shape_engine_get_radar_overflow(shape_engine *e, double *out, int max);
int shape_engine_get_fit(shape_engine *e, int global_frame, double *fit);
/* POS maps are kept only when enabled before the evaluation (they cost HBM
 * traffic): keep = 1 writes z, cos(e), cos(i) and facet maps of every frame. */
int shape_engine_keep_pos(shape_engine *e, int keep);
int shape_engine_get_pos(shape_engine *e, int global_frame, double *z, double *cose,
                         int *facet);
int shape_engine_get_lghtcrv_pos(shape_engine *e, int set, int point, double *z,
                                 double *cose, double *cosi, int *facet, double *zill,
                                 int *fill);
/* Lightcurve outputs: y[ncalc] (calc_lghtcrv's y), fit[n], cal, chi2. */
int shape_engine_get_lghtcrv(shape_engine *e, int set, double *y, double *fit,
                             double *cal, double *chi2);
int shape_engine_get_seen(shape_engine *e, unsigned char *seen);
/* Realized model (realize_coordinates outputs). */
int shape_engine_get_realized(shape_engine *e, double *x, double *vn, double *fn,
                              double *area);

/* Runs one evaluation of a batched form without its graph, with CUDA events
 * between stages, and writes the stage times in ms: [0] realize, [1] state
 * reset and image clears, [2] view transforms, [3] facet binning,
 * [4] tile raster + delay-Doppler synthesis, [5] chi-square partials,
 * [6] lightcurve shadowing + photometry, [7] finalize + summary. Datasets
 * whose chi-square partials, frame results and totals run as one kernel
 * (every radar frame's chunk list fits its staging) time that kernel in [7]
 * and leave [5] empty. Returns the number of stages written. */
int shape_engine_stage_times(shape_engine *e, int form, double *ms, int max);

/* Facet-bin capacity per 16x16 POS tile. 0 (default) lets finalize size it
 * from a dry-run binning of the model (next power of two above 1.25x the
 * fullest tile); tiles whose bin overflows are rasterized by an ordered scan
 * of all facets, which is exact but slow. Takes effect at the next finalize. */
int shape_engine_set_bin_capacity(shape_engine *e, int cap);
/* Batched FP32 form, radar views: 1 (default) redoes every pixel whose
 * coverage or depth-order decision lies within FP32 error by the FP64
 * form's rules, so facet maps are the FP64 form's (kept POS maps also get
 * the FP64 form's depths); 0 takes the FP32 decisions as they are (a pixel
 * within FP32 error of a facet edge or of a depth tie may take another
 * facet than the FP64 form: a faster raster, and a small frame's
 * chi-square may move by ~1e-4 when that happens). Lightcurve views are
 * always exact. Takes effect at the next evaluation. */
int shape_engine_set_fp32_exact(shape_engine *e, int exact);
/* vary_params (src/shape/vary_params.c:84-327): the four means the
 * reference computes for its joint adjustments of the 0th delay-correction
 * coefficient, the radar and optical albedos and the Doppler scale, from an
 * FP64 evaluation of the current model (the call evaluates with the POS maps
 * kept, so the last results are that evaluation's). As the reference does,
 * only the first dataset contributes (its loop over datasets ends after set
 * 0, vary_params.c:106), and the weight sums are read_dat's over every
 * dataset. vary_* are par->vary_delcor0 / vary_radalb / vary_optalb /
 * vary_dopscale (0 = VARY_NONE); delcor0_free and dopscale_free (per
 * dataset in add order, or NULL = none) tell whether a set's 0th
 * delay-correction coefficient and Doppler scale float (state != 'c'); a
 * frame or lightcurve counts as fixed-calibration when cal_floating is 0.
 * out = deldop_zmax, rad_xsec, opt_brightness, cos_subradarlat. A smeared
 * first dataset returns SHAPE_E_UNSUPPORTED. */
typedef struct shape_vary_options {
    int vary_delcor0, vary_radalb, vary_optalb, vary_dopscale;
    const int *delcor0_free;
    const int *dopscale_free;
} shape_vary_options;
int shape_engine_vary_params(shape_engine *e, const shape_vary_options *opt, double out[4]);

/* Raster kernel of the batched forms./* Raster kernel of the batched forms. mode -1 (default): the first batched
 * evaluation of each form times four candidates on this engine's datasets
 * (the tile-per-CTA kernel and the warp-independent kernel, each with one
 * CTA per non-empty tile or a persistent grid of resident CTAs on every
 * SM striding over the tiles) and keeps the fastest; the choice is
 * remembered for engines of the same size class in the process. mode 0 /
 * 1: that kernel, one CTA per tile, no timing. Every candidate computes the
 * same images. Lightcurve views always use the tile-per-CTA kernel (in the
 * FP32 form their own launch; in the FP64 form an engine with lightcurve
 * points tunes the grid only). */
int shape_engine_set_raster_tuning(shape_engine *e, int mode);
/* The raster choice of a form: *variant (0 tile-per-CTA, 1 warp-
 * independent), *persistent, and ms[4] (may be NULL) the measured raster
 * times of the candidates variant*2 + persistent (0 where not measured).
 * Returns 1 once the form is tuned, 0 before its first evaluation. */
int shape_engine_get_raster_tuning(shape_engine *e, int form, int *variant, int *persistent, double *ms);

/* A new view for radar frame global_frame (delay-Doppler and Doppler frames
 * numbered across sets in the order they were added), for spin, pole and
 * delay-correction trials without rebuilding the engine: ae, oe, spin,
 * deloff and dopoff as in shape_deldop_frame (deloff is ignored for Doppler
 * frames). The frame's view-dependent constants (posvis's observer <- body
 * matrix, src/shape/posvis.c:101-122; pos2deldop's Doppler axes, footprint
 * extents, shifts and badradar term, src/shape/pos2deldop.c:218-288) are
 * recomputed on the host exactly as at finalize and copied to the device on
 * the engine's stream, so the next evaluation of every form sees them and
 * captured graphs stay valid; the results equal those of an engine built
 * with the new view. Bin capacities keep their tuning (a tile that now
 * overflows takes the ordered full-scan path). Before finalize the frame's
 * descriptor is updated. Workloads a server already took from this engine
 * keep their views. */
int shape_engine_set_frame_view(shape_engine *e, int global_frame, const double ae[9], const double oe[9],
                                const double spin[3], double deloff, double dopoff);
/* The same for lightcurve point `point` (numbered across sets): its ae, oe
 * and se (src/shape/calc_fits.c:1634-1716). */
int shape_engine_set_point_view(shape_engine *e, int point, const double ae[9], const double oe[9],
                                const double se[9]);

/* Penalty types (par->pen.type; the reference's numbering, src/shape/const.h). */
#define SHAPE_PEN_NONSMOOTH 9
#define SHAPE_PEN_CONCAVITY 10
#define SHAPE_PEN_RDEV 11
#define SHAPE_PEN_VOLUME 12
#define SHAPE_PEN_COMDEV 13
#define SHAPE_PEN_INERTIADEV 14
#define SHAPE_PEN_INERTIADEV_UNI 15
#define SHAPE_PEN_PA3TILT 16
#define SHAPE_PEN_NONPA 17
#define SHAPE_PEN_NONPA_UNI 18
#define SHAPE_PEN_EULEROFFS 19
#define SHAPE_PEN_FLATTENING 20
#define SHAPE_PEN_MAXRDEV 21
#define SHAPE_PEN_IMPULSE 25

/* The penalty terms of the objective (par->pen; penalties,
 * src/shape/penalties.c:121-1236): n penalties of the given types and
 * weights (a negative weight takes the reciprocal of the penalty, as in the
 * reference). From the next evaluation on, the summary's objective is
 * (chi2/dof + the penalty sum) times the bad-model factors, and bestfit
 * minimises that. The model's moments and its edge and vertex sums are
 * reduced on the device after each evaluation (two more launches and a
 * small copy), and the penalties follow from them on the host. A model of
 * several components first gets check_surface's active flags
 * (src/shape/realize_mod.c:572-756; one more launch): vertices, facets
 * (by their centroids) and edges inside another component are left out of
 * the moments, the edge terms and the vertex deviations, as
 * compute_moments and penalties() leave them out. The
 * shape penalties need a closed surface. INERTIADEV, NONPA and IMPULSE need
 * the spin model. The photometric penalties, MAXELLIPDEV, NONCOSINE and
 * BIFURCATION return SHAPE_E_UNSUPPORTED. n = 0 removes the penalties.
 * Server workloads ignore them. */
int shape_engine_set_penalties(shape_engine *e, int n, const int *type, const double *weight);
/* Each penalty's value after its weight's sign rule (par->pen.base) at the
 * last evaluation, for up to max penalties; returns the penalty count. */
int shape_engine_get_penalties(shape_engine *e, double *base, int max);
/* check_surface's flags at the last evaluation with penalties (1: active,
 * 0: inside another component), nv vertices and nf facets in model order;
 * all 1 for a model of one component (src/shape/realize_mod.c:582-594).
 * SHAPE_E_STATE before such an evaluation. */
int shape_engine_get_active(shape_engine *e, unsigned char *vertex_act, unsigned char *facet_act);

/* The spin model of the engine's views, for spin fits (realize_spin,
 * src/shape/realize_spin.c:41-285): the spin state; each dataset's angle and
 * spin offsets (3 doubles per dataset, numbered as the add_*_set calls
 * returned them; NULL = zeros); each radar frame's view epoch (days,
 * light-time corrected; global frame numbering) and orbital spin
 * contribution (3 doubles per frame, ecliptic, rad/day; NULL = zeros).
 * Lightcurve points take their set's calculated epochs x[]. Every view's
 * ae (and a radar frame's spin vector) is realized now by
 * shape_realize_spin and replaces the one its dataset gave; oe and se are
 * kept. All datasets must be added first. */
int shape_engine_set_spin_model(shape_engine *e, const shape_spin_state *spin, const double *set_angleoff,
                                const double *set_omegaoff, const double *frame_t,
                                const double *frame_orbspin);
/* Spin realization inside each evaluation (principal-axis rotators): with
 * on = 1 the evaluation graph copies the spin state and dataset offsets
 * from pinned memory and a kernel realizes every radar frame's and
 * lightcurve point's ae (and a frame's spin vector) and view constants
 * before the raster, as shape_realize_spin and the host setup do (the
 * device's sin and cos may differ from the C library's in the last place).
 * shape_engine_set_spin_param then only records the value: a spin trial is
 * a graph replay with no host realization or view upload. Needs the spin
 * model (SHAPE_E_STATE without it) of a principal-axis rotator and single-
 * view frames (SHAPE_E_UNSUPPORTED otherwise); set_frame_view and
 * set_point_view are refused while it is on. on = 0 realizes on the host
 * again (the default). */
int shape_engine_set_spin_device(shape_engine *e, int on);
/* A radar frame's current ae (9, row-major) and spin vector (3): the
 * device-realized ones of the last evaluation in device spin mode. */
int shape_engine_get_frame_view(shape_engine *e, int global_frame, double ae[9], double spin[3]);
/* One spin parameter (SHAPE_PAR_SPIN_* / ANGLEOFF / OMEGAOFF) of the spin
 * model: set re-realizes every view and copies the view constants to the
 * device on the engine's stream (the next evaluation, graph replays
 * included, sees them). */
int shape_engine_set_spin_param(shape_engine *e, int kind, int index, double value);
int shape_engine_get_spin_param(shape_engine *e, int kind, int index, double *value);
/* Tuning state after finalize: [0] bin capacity, [1] largest tile count of
 * the dry run, [2] non-empty tiles, [3] tiles, [4] tile width in pixels.
 * Returns the number of values written. */
int shape_engine_get_tuning(shape_engine *e, int *out, int max);

/* Number of kernel launches one evaluation in `form` makes (after finalize). */
int shape_engine_kernels_per_eval(shape_engine *e, int form, int *count);

/* Device time of the last evaluation (CUDA events on the engine stream). */
int shape_engine_last_time_ms(shape_engine *e, double *ms);

/* ------------------------------------------------------------- bestfit */

/* Free parameter kinds (src/shape/mkparlist.c:218-235). */
#define SHAPE_PAR_SCALE 1      /* component scale factor index (SIZEPAR) */
#define SHAPE_PAR_VERTEX_R 2   /* vertex deviation r of vertex index (SHAPEPAR) */
/* Spin parameters (SPINPAR, src/shape/mkparlist.c:855-950); they need the
 * engine's spin model (shape_engine_set_spin_model). */
#define SHAPE_PAR_SPIN_ANGLE 3     /* spin.angle[index] (rad) */
#define SHAPE_PAR_SPIN_OMEGA 4     /* spin.omega[index] (rad/day) */
#define SHAPE_PAR_SPIN_INERTIA 5   /* spin.inertia[index] */
#define SHAPE_PAR_SPIN_OMEGADOT 6  /* spin.omegadot[index] (rad/day^2) */
#define SHAPE_PAR_SPIN_IMPULSE 7   /* spin.impulse[index / 3][index % 3] (rad/day) */
#define SHAPE_PAR_SPIN_LIB 8       /* index 0 lib_amp, 1 lib_freq, 2 lib_phase */
#define SHAPE_PAR_ANGLEOFF 9       /* angleoff[index % 3] of dataset index / 3 (rad) */
#define SHAPE_PAR_OMEGAOFF 10      /* omegaoff[index % 3] of dataset index / 3 (rad/day) */

/* One free parameter with its step and tolerances (par->fparstep,
 * fpartol, fparabstol; e.g. length_step/length_tol/length_abstol). */
typedef struct shape_fit_param {
    int kind;
    int index;
    double step, tol, abstol;
} shape_fit_param;

typedef struct shape_fit_options {
    int form;           /* SHAPE_FORM_* used for every trial evaluation */
    double term_prec;   /* stop when the fractional decrease of an iteration < term_prec */
    int term_maxiter;   /* 0 = no limit */
} shape_fit_options;

typedef struct shape_fit_result {
    double initial_objective, final_objective;
    int iterations, evaluations, trace_len;
} shape_fit_result;

/* The reference's bestfit (src/shape/bestfit.c:250-704) over the given free
 * parameters, without penalties: per parameter, bracket a minimum of the
 * objective starting from (value, value + step), then Brent-minimise it to
 * tol*|x| + abstol, adopt the minimum, and iterate over all parameters
 * until the objective's fractional decrease in an iteration is below
 * term_prec. Each trial is one device evaluation (a graph replay in the
 * batched forms). trace (optional, 2*trace_max doubles) receives the
 * (parameter number, trial value) of every trial in order. */
int shape_engine_bestfit(shape_engine *e, const shape_fit_param *params, int nparams,
                         const shape_fit_options *opt, shape_fit_result *res, double *trace,
                         int trace_max);
int shape_engine_get_scale(shape_engine *e, int j, double *value);

/* The two line searches of bestfit on a caller objective (host only, no
 * device use): bracketing (src/nr/mnbrak.c) and Brent's minimiser with an
 * absolute tolerance (src/nr/brent_abs.c). shape_brent_minimize returns the
 * iteration count (>= 1) or a negative status. */
typedef double (*shape_objective_fn)(double x, void *user);
int shape_bracket_minimum(shape_objective_fn f, void *user, double *ax, double *bx, double *cx,
                          double *fa, double *fb, double *fc);

/* The same bestfit iteration on a caller objective (host only): values[k]
 * is free parameter k; f returns the objective for the current values and
 * sets *posbnd / *badradar for the flags of that evaluation. Lets a host
 * program drive any objective (the reference's own calc_fits + chi2, or a
 * multi-GPU reduction) with this fit loop. */
typedef double (*shape_param_objective_fn)(const double *values, void *user, int *posbnd, int *badradar);
int shape_bestfit_host(shape_param_objective_fn f, void *user, double *values,
                       const shape_fit_param *params, int nparams, const shape_fit_options *opt,
                       shape_fit_result *res, double *trace, int trace_max);
int shape_brent_minimize(shape_objective_fn f, void *user, double ax, double bx, double cx,
                         double tol, double abstol, double *xmin, double *fmin);

/* Per-frame chi-square sums over images the CALLER already holds in device
 * memory, computed without allocating any device memory. It has no
 * counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc, such as a process whose device memory belongs to another
 * allocator (a PyTorch or pool-managed program under a hard memory cap) or a
 * latency-critical loop where cudaMalloc/cudaFree could synchronize the
 * device. Frame f occupies elements [frame_offsets[f], frame_offsets[f+1])
 * of d_obs, d_oneovervar and d_fit (device pointers, FP64); weight,
 * cal_floating and cal (host arrays of nframes) follow chi2_deldop. On return
 * out (host, 5*nframes doubles) holds o2, m2, om, cal and chi2 per frame.
 * Limits: at most 4096 frames and 65536*2048 elements in total; larger
 * requests fail with SHAPE_E_ARG. The scratch space is one fixed device
 * array (about 3.5 MB per device, kept until the process exits); the first
 * call on a device looks up its address, so make that first call outside
 * any stream capture. Kernels run on the legacy default stream and the call
 * returns after the results reach host memory; the caller's current device
 * is current again on return. Calls share the scratch
 * array: calls that overlap on the GPU (from several threads or streams)
 * race on it. */
int shape_chi2_frames_noalloc(int device, int nframes, const long long *frame_offsets,
                              const double *d_obs, const double *d_oneovervar,
                              const double *d_fit, const double *weight,
                              const int *cal_floating, const double *cal, double *out);

/* ---- One plane-of-sky view per call, on the caller's host images ----
 *
 * The device forms of the reference's posvis, pos2deldop, posmask,
 * apply_photo and posclr for callers that drive the plane of sky themselves
 * (the write / view / map actions, multi-component models, binary systems),
 * reached through the reference-signature wrappers of
 * shape-cuda-v1.2_b200/dropin/shape_b200_pos.c. Images are the caller's
 * host arrays of (2n+1)^2 elements in [i][j] order: element [i][j],
 * i, j in [-n, n], at (i+n)*(2n+1) + (j+n). Each call uploads what it reads,
 * runs on the device (FP64, the engine's kernels) and copies back what it
 * writes; calls on one device run one at a time. */

/* The plane-of-sky frame: struct pos_t's geometry (src/shape/shape2.h:1061-1094). */
typedef struct shape_pos_view {
    int n;                      /* pos->n */
    double km_per_pixel;        /* pos->km_per_pixel */
    double ae[9], oe[9], se[9]; /* pos->ae, pos->oe, pos->se (row-major) */
    int bistatic;               /* pos->bistatic */
} shape_pos_view;

/* struct pos_t's images and limits; an operation reads or writes only the
 * members it names, the others may be NULL. */
typedef struct shape_pos_images {
    double *b, *cose, *cosi, *z;    /* pos->b, cose, cosi, z */
    int *body, *comp, *f;           /* pos->body, comp, f */
    double *cosill, *zill;          /* sun view (bistatic) */
    int *bodyill, *compill, *fill;
    int xlim[2], ylim[2];           /* pos->xlim, ylim */
    int xlim2[2], ylim2[2];         /* pos->xlim2, ylim2 */
    double posbnd_logfactor;        /* pos->posbnd_logfactor */
} shape_pos_images;

/* posvis (src/shape/posvis.c:84-364; declared at src/shape/shape2.h:1503):
 * one model component (x, vn: nv x 3 vertex positions and normals; fv, fn:
 * nf x 3 facet corners and normals; body-fixed) seen from the observer
 * (src = 0: z, cose, f, and cosi when bistatic) or from the sun (src = 1:
 * zill, cosill, fill), accumulating over what the images hold: a pixel
 * changes only where this component is nearer. Pixels it assigns get
 * body and comp; xlim/ylim (xlim2/ylim2) widen as POSrect widens them;
 * posbnd_logfactor is set. Returns outbnd (0 or 1) or a negative status. */
int shape_posvis(int device, const shape_pos_view *view, shape_pos_images *img, int nv, const double *x,
                 const double *vn, int nf, const int *fv, const double *fn, const double orbit_offset[3],
                 int smooth, int src, int body, int comp);

/* pos2deldop (src/shape/pos2deldop.c:176-581; src/shape/shape2.h:1495):
 * adds the radar cross-section of every lit pixel of `body` within xlim /
 * ylim to fit (ndel x ndop, delay-row major) for the frame's view (oe,
 * spin, deloff, dopoff, COM and DC bins of `frame`; its km_per_pixel is
 * the view's), sets res's delay / Doppler limits and badradar terms and
 * *km2Hz (may be NULL). Returns badradar (0 or 1) or a negative status. */
int shape_pos2deldop(int device, const shape_pos_view *view, const shape_pos_images *img,
                     const shape_eval_params *par, const shape_deldop_set *set, const shape_deldop_frame *frame,
                     double orbit_xoff, double orbit_yoff, double orbit_dopoff, int body, double *fit,
                     shape_deldop_result *res, double *km2Hz);

/* posmask (src/shape/posmask.c:58-174; src/shape/shape2.h:1502): zeroes
 * cose where the sun view shows another facet, component or body nearer
 * the sun than the pixel by more than tol (reads z, f, comp, body and the
 * sun view's zill, fill, compill, bodyill). */
int shape_posmask(int device, const shape_pos_view *view, shape_pos_images *img, double tol);

/* apply_photo (src/shape/apply_photo.c:78-309; src/shape/shape2.h:1446)
 * for the Lambert, Lommel-Seeliger and Kaasalainen laws: writes b for every
 * lit pixel of `body` within xlim / ylim and *sum = their sum in the
 * reference's order (TINY, 1e-40, when 0). */
int shape_apply_photo(int device, const shape_optical_law *law, double phase, double intensityfactor,
                      const shape_pos_view *view, shape_pos_images *img, int body, double *sum);

/* posclr (src/shape/posclr.c:24-67; src/shape/shape2.h:1501): blank images
 * and empty limits. Host only. */
int shape_posclr(const shape_pos_view *view, shape_pos_images *img);

/* Continuous-batching evaluation server (one device). It has no counterpart
 * in the reference, whose fits evaluate one model at a time in one process;
 * it serves many fits (workloads) from one GPU. A workload is the host
 * description of a configured engine (model, switches, datasets), copied at
 * registration. The server keeps device-resident instances of workloads, at
 * most hbm_budget_bytes of device memory in total, and runs up to max_slots
 * requests at once, each on its instance's stream. A scheduler thread
 * serves the requests: it admits every waiting request it can, oldest
 * first, to an idle instance of its workload or to a new one when the
 * budget allows (idle instances of other workloads are evicted, least
 * recently used first, to make room); a request that cannot start does not
 * hold up those behind it, unless it has waited more than 20 ms, after
 * which later requests only get instances that already exist. A request
 * evaluates its workload at its own scale factors; its result is the same
 * as a lone shape_engine_evaluate of that workload at those scale factors.
 *
 * Online use: shape_server_start, then shape_server_submit as requests
 * arrive (any thread) and shape_server_poll / shape_server_wait for their
 * results; shape_server_stats_get covers the requests since start;
 * shape_server_stop finishes what was submitted and ends the thread.
 * shape_server_run replays a whole trace through the same scheduler: each
 * request is submitted at its arrival time (seconds after the call starts)
 * and its latency counts from then; its requests leave the ticket table
 * when it returns. */
typedef struct shape_server shape_server;
typedef struct shape_request {
    int workload;              /* index returned by shape_server_add_workload */
    double arrival_s;          /* seconds after shape_server_run starts */
    double scale[3];           /* ellipsoid scale factors of this request */
} shape_request;
typedef struct shape_request_result {
    double chi2, objective;
    double t_start, t_done;    /* seconds after shape_server_run starts */
    double latency_s;          /* t_done - arrival_s */
    double device_ms;          /* event time of the request's evaluation */
    int instance;              /* instance slot that served it */
} shape_request_result;
typedef struct shape_server_stats {
    double span_s;             /* first arrival window start to last completion */
    double requests_per_s;
    double frame_evals_per_s;  /* radar frames + lightcurve points evaluated per second */
    double p50_latency_s, p99_latency_s;
    double mean_concurrency;   /* time-averaged requests in flight */
    int peak_concurrency;
    int instances_created, instances_evicted;
    double peak_hbm_bytes;     /* peak device bytes held by instances during the run */
} shape_server_stats;
/* Spin realization of one dataset (replaces realize_spin + inteuler,
 * src/shape/realize_spin.c:41-285, src/shape/inteuler.c:85-210): for each of
 * n view epochs t[k] (days), the ecliptic -> body matrix ae[9k..9k+8]
 * (row-major) and the total spin vector in ecliptic coordinates
 * spin_out[3k..3k+2] = orbspin[3k..] + ae^T (w + omegaoff), w being the
 * body-frame spin vector evolved from t0 with the impulses met on the way.
 * angleoff / omegaoff: the dataset's angle and spin offsets. Host code.
 * Principal-axis states: the reference's values (same operations and order).
 * Non-principal-axis states: Euler's equations and the orientation
 * integrated between impulse epochs by an adaptive Dormand-Prince 5(4)
 * method at local error 1e-13, in time measured from each interval's start
 * (the reference's brute-force integration, with its own integrator; its
 * periodic method is not provided): within ~1e-12 of the exact solution
 * over days, where the reference's stepping of the absolute epoch leaves
 * it ~1e-8 away. More than
 * SHAPE_MAX_IMPULSES impulses, or a non-positive moment of inertia for a
 * non-principal-axis state, return SHAPE_E_ARG. */
int shape_realize_spin(const shape_spin_state *spin, const double angleoff[3], const double omegaoff[3], int n,
                       const double *t, const double *orbspin, double *ae, double *spin_out);

/* A view's geometry from ephemerides at epoch t (ephem2mat,
 * src/shape/ephem2mat.c:33-228), with the reference's operations: RA, Dec
 * and distance interpolated linearly in the asteroid ephemeris (nast >= 2
 * entries, ascending t; RA across the 0/360 line), the ecliptic ->
 * observer matrix oe (row-major), the plane-of-sky motion's contribution s
 * to the apparent spin vector (ecliptic, rad/day), and the distance (AU).
 * With a solar ephemeris (sun non-NULL; the bistatic case) also the
 * ecliptic -> solar matrix se, the solar phase angle and the azimuth of the
 * Sun in the plane of the sky; otherwise both angles are 0. An epoch
 * outside a table returns SHAPE_E_ARG. Host code. */
int shape_ephem_view(const shape_ephem_point *ast, int nast, const shape_ephem_point *sun, int nsun, double t,
                     double oe[9], double se[9], double s[3], double *solar_phase, double *solar_azimuth,
                     double *dist);

/* A radar view's epoch and geometry as the reference's dataset reader sets
 * them (src/shape/read_dat.c:866-900): shape_ephem_view at t_obs (the
 * view's epoch from the .obs file), then, with perform_ltc
 * (par->perform_ltc), the epoch less the one-way light time (5.775518328e-3
 * day per AU of the distance found) and the ephemeris evaluated again.
 * Writes the view epoch (for shape_realize_spin), oe and the orbital spin
 * contribution. */
int shape_ephem_radar_view(const shape_ephem_point *ast, int nast, double t_obs, int perform_ltc, double *t_view,
                           double oe[9], double orbspin[3]);

/* A view's delay and Doppler offsets (bins) from its dataset's
 * delay-correction polynomial (deldopoffs, src/shape/deldopoffs.c:17-42):
 * a[0..n] in usec and usec/day^k about epoch t0; deloff = (a0 + sum a_k
 * (t - t0)^k) / del_per_pixel, dopoff = -(d delay / dt) Ftx /
 * (dop_per_pixel 86400), in the reference's operation order. These are the
 * shape_deldop_frame / shape_engine_set_frame_view offsets; a Doppler set
 * uses dopoff only. */
int shape_delcor_offsets(const double *a, int n, double t0, double t_view, double del_per_pixel,
                         double dop_per_pixel, double Ftx, double *deloff, double *dopoff);

/* ------------------------------------------------------------- model files */

/* A SHAPE model file (.mod) as read_mod reads it (src/shape/read_mod.c:204-227,
 * read_shape :289-542, read_photo :544-1953, read_spin :1954-2140), for the
 * models the engine evaluates: one vertex component with zero component
 * offsets and rotations, radar laws none / cosine / gaussian / hagfors /
 * cosine_qs / gauss+cosine / hagfors+cosine / cosine+cosine, optical laws
 * none / lambertian / lommel / kaasalainen, and the spin section. Comments
 * in curly braces are skipped; numbers must fill their token. Angles come
 * out in radians, spin rates in rad/day and epochs in Julian days, by
 * read_spin's operations. Syntax errors return SHAPE_E_ARG and valid but
 * unsupported content SHAPE_E_UNSUPPORTED, both with the line number in
 * shape_last_error(). Host code; the handle owns all arrays. */
typedef struct shape_mod_file shape_mod_file;
int shape_mod_read(const char *path, shape_mod_file **out);
void shape_mod_free(shape_mod_file *m);
/* The shape as shape_engine_set_model takes it (arrays owned by m; the
 * attached-facet lists in increasing facet order, as setupvertices builds
 * them). */
int shape_mod_model(const shape_mod_file *m, shape_model_desc *out);
/* Law ilaw of the file; returns the number of laws (law = NULL: count
 * only). A "none" law has type 0. */
int shape_mod_radar_law(const shape_mod_file *m, int ilaw, shape_radar_law *law);
int shape_mod_optical_law(const shape_mod_file *m, int ilaw, shape_optical_law *law);
/* The spin state (pa set as read_spin sets it). */
int shape_mod_spin(const shape_mod_file *m, shape_spin_state *spin);
/* The file's floating parameters (state f) that the engine can vary, in the
 * reference's parameter-list order (src/shape/mkparlist.c): scale factors,
 * vertex deviations, spin angles, spin rates, moments of inertia, spin-rate
 * changes, impulses, libration. kind and index are set, step and the
 * tolerances are 0 (they come from the .par file). Returns the count. */
int shape_mod_free_params(const shape_mod_file *m, shape_fit_param *out, int max);
/* Writes m as a model file that read_mod (and shape_mod_read) reads back:
 * the parameter states of the file m came from, numbers with 17
 * significant digits. Shape values round-trip exactly. Angles and rates
 * are written back in degrees, which can change their last bit. Epochs
 * become calendar dates to the second, as jd2cal rounds them
 * (src/astro/jdcal.c:16-33). */
int shape_mod_write(const shape_mod_file *m, const char *path);
/* Copies an engine's current scale factors, vertex deviations and (when it
 * has a spin model) spin parameters into m, as a fit leaves them; m must
 * describe the engine's model. */
int shape_mod_take_engine(shape_mod_file *m, shape_engine *e);

/* One radar data file into a frame's obs and 1/variance arrays (read_deldop
 * / read_doppler, src/shape/read_dat.c:800-856, 1150-1176, 2074-2260): a
 * stored image of ndel x ndop (a Doppler spectrum: ndel = 1) in raw
 * float32, RDF (header lines up to one starting with '.', then float32) or
 * ASCII, told apart by the first 128 bytes as the reference does (FITS
 * returns SHAPE_E_UNSUPPORTED). Each value is rounded to float, the window
 * idel_use x idop_use (1-based, inclusive) is kept, delay-major, and
 * multiplied by sdev. gamma != 1 applies the delay-Doppler gamma transform
 * (par->dd_gamma; pass 1 for Doppler data). 1/variance is 1/sdev^2, or
 * with nlooks > 0 (par->speckle) 1/(sdev^2 + (obs/sqrt(nlooks))^2), times
 * pixweight (a full-size weight image, or NULL). big_endian: the data's
 * byte order for float32 files (par->endian; the reference's default is
 * big-endian). Host code. */
int shape_read_radar_data(const char *path, int ndel, int ndop, const int idel_use[2], const int idop_use[2],
                          int big_endian, double sdev, double gamma, double nlooks, const double *pixweight,
                          double *obs, double *oneovervar);

/* A lightcurve data file (read_lghtcrv, src/shape/read_dat.c:1925-1956):
 * n points of epoch (JD), magnitude and magnitude error, whitespace-
 * separated with comments in curly braces. Writes each point's epoch, its
 * intensity relative to the Sun exp(-0.4 ln10 (mag - sun_appmag)) and
 * 1/variance with the error 0.4 ln10 magerr intensity, in the reference's
 * operation order. Host code. */
int shape_read_lghtcrv_data(const char *path, int n, double sun_appmag, double *t, double *obs,
                            double *oneovervar);

/* ------------------------------------------------------------- .obs files */

/* The switches of the .par file that the dataset reader uses. */
typedef struct shape_obs_options {
    int perform_ltc;        /* par->perform_ltc: light-time correction of view epochs */
    double dd_gamma;        /* par->dd_gamma (1: none) */
    int speckle;            /* par->speckle */
    int big_endian;         /* par->endian == BIG_ENDIAN_DATA (the reference's default) */
} shape_obs_options;

/* A SHAPE observation file (.obs; read_dat, src/shape/read_dat.c:409-527)
 * whose datasets are delay-Doppler sets (read_deldop, :528-900) or Doppler
 * sets (read_doppler, :920-1180) or lightcurve / heliocurve sets
 * (read_lghtcrv, :1667-2063); smeared delay-Doppler frames and
 * pixel-weighting masks are read, gzipped data files, smeared Doppler
 * frames or lightcurve points and plane-of-sky sets return
 * SHAPE_E_UNSUPPORTED. A frame with a pixel-weighting mask
 * (mask_SS_FF.txt, FFF for sets of more than 100 frames, in the set's data
 * directory unless shape_obs_set_maskdir names another) keeps the window
 * of its positive weights: its ndel x ndop, COM and DC bins count from the
 * window, its dof is weight x the positive weights, and its 1/variance is
 * multiplied by the weights (src/shape/read_dat.c:696-762, 845-852,
 * 1059-1118). The '=' state of angle and
 * spin offsets and of delay-correction polynomials takes the last earlier
 * set's value, as the reference's realize_angleoff, realize_omegaoff and
 * realize_delcor do (src/shape/realize_spin.c:283-337,
 * src/shape/realize_delcor.c:60-146); '=' on the first set, or a tied
 * polynomial of another degree or epoch, is SHAPE_E_ARG. Host code. */
typedef struct shape_obs_file shape_obs_file;
int shape_obs_read(const char *path, shape_obs_file **out);
/* The .par file's mask directory (par->maskdir): the masks of every
 * weighted frame are read again from dir (a missing file is SHAPE_E_ARG). */
int shape_obs_set_maskdir(shape_obs_file *o, const char *dir);
void shape_obs_free(shape_obs_file *o);
int shape_obs_nsets(const shape_obs_file *o);
/* 0: set s is a delay-Doppler set (shape_obs_set / shape_obs_frames);
 * 1: a Doppler set (shape_obs_doppler); 2: a lightcurve or heliocurve set
 * (shape_obs_lghtcrv_info / shape_obs_lghtcrv); 3: a plane-of-sky set
 * (shape_obs_poset_info / shape_obs_poset). */
int shape_obs_set_type(const shape_obs_file *o, int s);
/* A plane-of-sky set (read_poset, src/shape/read_dat.c:1392-1560): its
 * optical law index and frame count; each frame's image file (the data
 * directory joined with its name) and pixel-weighting flag. The images are
 * FITS files, which this library does not read (cfitsio is not part of
 * it); the caller reads them. */
int shape_obs_poset_info(const shape_obs_file *o, int s, int *ioptlaw, int *nframes);
int shape_obs_poset_file(const shape_obs_file *o, int s, int frame, char *path, int size, int *pixels_weighted);
/* The geometry of the set's frames (one view per frame): oe, se and the
 * solar phase by ephem2mat at the frame epoch (light-time corrected when
 * opt->perform_ltc is set), ae from the spin model at that epoch, the fit
 * grid's km per pixel (angular pixel size times the distance before the
 * light-time correction, as read_poset computes it), the north angle, the
 * COM offsets and the weight. pos_n, km_per_pixel, ncol, nrow, colcom_vig,
 * rowcom_vig and dof are left as the caller set them (set_up_pos and the
 * image). Smeared plane-of-sky frames return SHAPE_E_UNSUPPORTED. */
int shape_obs_poset(const shape_obs_file *o, int s, const shape_spin_state *spin, const shape_obs_options *opt,
                    shape_poset_frame *frames);
/* Set s's radar setup (set->law is kept: take it from the model's radar
 * law iradlaw), its frame count, angle and spin offsets (rad, rad/day) and
 * the number of data elements of its frames. iradlaw is >= 0 (a negative
 * index fails in shape_obs_read); the file does not know the model, so the
 * caller checks iradlaw < the model's number of radar laws, as
 * read_deldop does (src/shape/read_dat.c:557-562). */
int shape_obs_set(const shape_obs_file *o, int s, shape_deldop_set *set, int *iradlaw, int *nframes,
                  double angleoff[3], double omegaoff[3], size_t *nelem);
/* Set s's frames for shape_engine_add_deldop_set: each view's epoch and oe
 * from the ephemeris (shape_ephem_radar_view), deloff and dopoff from the
 * delay-correction polynomial (shape_delcor_offsets), ae and the spin
 * vector from the spin state (shape_realize_spin, with the set's offsets
 * and the orbital spin), the data file read from the set's directory
 * (shape_read_radar_data), the weight, dof and calibration. pos_n and
 * km_per_pixel come from the .par file. obs and oneovervar receive each
 * frame's image in frame order (nelem doubles); sdev (or NULL) each
 * frame's sdev. A set with several views per frame (smearing) returns
 * SHAPE_E_UNSUPPORTED here: read it with shape_obs_frames_views. */
int shape_obs_frames(const shape_obs_file *o, int s, const shape_spin_state *spin, int pos_n, double km_per_pixel,
                     const shape_obs_options *opt, shape_deldop_frame *frames, double *obs, double *oneovervar,
                     double *sdev);
/* Views per frame of set s and the index v0 of the view at the frame's
 * epoch (smearing mode center: nviews / 2, first: 0; src/shape/read_dat.c:
 * 635-646). */
int shape_obs_views(const shape_obs_file *o, int s, int *nviews, int *v0);
/* Set s's frames for shape_engine_add_deldop_set_views: nframes * nviews
 * views, each built as shape_obs_frames builds a frame at the view's epoch
 * t0 + (k - v0) * view interval (src/shape/read_dat.c:868-899), listed per
 * frame in rendering order (views (v0+1+j) % nviews, the epoch view last). */
int shape_obs_frames_views(const shape_obs_file *o, int s, const shape_spin_state *spin, int pos_n,
                           double km_per_pixel, const shape_obs_options *opt, shape_deldop_frame *views, double *obs,
                           double *oneovervar, double *sdev);

/* A Doppler set's setup (set->law is kept) and frames for
 * shape_engine_add_doppler_set, built as shape_obs_frames builds
 * delay-Doppler frames (dopoff from the delay-correction polynomial's
 * rate, src/shape/dopoffs.c:19-40). obs and oneovervar receive each
 * frame's spectrum in frame order. */
int shape_obs_doppler(const shape_obs_file *o, int s, const shape_spin_state *spin, int pos_n, double km_per_pixel,
                      const shape_obs_options *opt, shape_doppler_set *set, shape_doppler_frame *frames, double *obs,
                      double *oneovervar);

/* Lightcurve set s (read_lghtcrv, src/shape/read_dat.c:1667-2063; its data
 * file, named in the .obs file relative to the current directory, is read
 * by shape_obs_read): the index of its optical law in the model, and its
 * numbers of calculated and observed points. One view per point. A
 * heliocurve set is read as the reference reads it: as a lightcurve set,
 * its two tables taken as the asteroid's and the Sun's ephemerides
 * (src/shape/read_dat.c:495-502 passes the lightcurve type). */
int shape_obs_lghtcrv_info(const shape_obs_file *o, int s, int *ioptlaw, int *ncalc, int *n);
/* The set ready for shape_engine_add_lghtcrv_set: set (its law member is
 * kept: take it from the model's optical law ioptlaw), ncalc points, the
 * calculated epochs x[ncalc] (light-time corrected with perform_ltc) with
 * each point's observer, Sun and body matrices and solar phase, and the
 * observation epochs t[n], intensities obs[n] (magnitudes relative to
 * sun_appmag, the .par file's sun_appmag for this law) and 1/variance; set
 * points at the caller's x, t, obs and oneovervar arrays. As read_lghtcrv
 * and realize_spin give them (src/shape/realize_spin.c:223-260). */
int shape_obs_lghtcrv(const shape_obs_file *o, int s, const shape_spin_state *spin, int pos_n, double km_per_pixel,
                      const shape_obs_options *opt, double sun_appmag, shape_lghtcrv_set *set,
                      shape_lghtcrv_point *points, double *x, double *t, double *obs, double *oneovervar);

/* The listfit output of one radar frame (chi2_deldop with listfit,
 * src/shape/chi2.c:525-560): ndel*ndop lines "%13.6e" of cal * fit / sdev,
 * delay-major (fit host memory). */
int shape_write_fitdat(const char *path, int ndel, int ndop, const double *fit, double cal, double sdev);
/* The same for radar frame global_frame of the engine's last evaluation:
 * its fit image and calibration, with the frame's sdev (deldop->frame[f]
 * .sdev; the engine keeps none for delay-Doppler frames). */
int shape_engine_write_fitdat(shape_engine *e, int global_frame, double sdev, const char *path);

int shape_server_create(int device, size_t hbm_budget_bytes, int max_slots, shape_server **out);
void shape_server_destroy(shape_server *s);
/* engine: a configured engine (model and datasets added; it need not be
 * finalized). form: SHAPE_FORM_*. Returns the workload index (>= 0) or a
 * negative status. */
int shape_server_add_workload(shape_server *s, shape_engine *engine, int form);
/* Device bytes one instance of workload w holds (0 before its first instance). */
int shape_server_workload_bytes(shape_server *s, int w, size_t *bytes);
int shape_server_run(shape_server *s, const shape_request *req, int n, shape_request_result *res,
                     shape_server_stats *stats);
/* Starts the scheduler thread (and a statistics window). */
int shape_server_start(shape_server *s);
/* Queues one request of workload w at scale factors scale[3] (NULL: 1, 1,
 * 1); *ticket identifies it. Its arrival time is the time of the call. */
int shape_server_submit(shape_server *s, int w, const double scale[3], long long *ticket);
/* 1 and *res when the request is done, 0 while it is not (poll), or a
 * negative status; shape_server_wait waits up to timeout_s seconds and
 * returns SHAPE_E_TIMEOUT if it is still not done. Result times are
 * seconds on the server's clock (since shape_server_create). After a
 * device failure every open request reports the failure's status. */
int shape_server_poll(shape_server *s, long long ticket, shape_request_result *res);
int shape_server_wait(shape_server *s, long long ticket, double timeout_s, shape_request_result *res);
/* Throughput and latency percentiles of the requests completed since
 * shape_server_start. */
int shape_server_stats_get(shape_server *s, shape_server_stats *stats);
/* Completes every submitted request, then ends the scheduler thread. */
int shape_server_stop(shape_server *s);

#ifdef __cplusplus
}
#endif
#endif
