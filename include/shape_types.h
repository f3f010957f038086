/*
 * Plain-data descriptions of SHAPE's model-evaluation inputs, shared by the
 * B200 engine's C ABI (shape_b200.h) and by the CPU oracle used in tests.
 *
 * Every struct holds plain numbers and host pointers only. Array layouts
 * mirror the reference's NR matrices so that a shim can fill them from the
 * reference structs without reordering:
 *   - POS images (struct pos_t, src/shape/shape2.h:1061-1094) are
 *     (2n+1) x (2n+1), x index i in [-n, n] major, y index j contiguous:
 *     element [i][j] lives at (i+n)*(2n+1) + (j+n);
 *   - delay-Doppler images (struct deldopfrm_t obs/fit/oneovervar,
 *     src/shape/shape2.h:1114-1182) are ndel x ndop, delay row major:
 *     element [idel][idop] (1-based in the reference) lives at
 *     (idel-1)*ndop + (idop-1);
 *   - 3x3 transforms are row-major double[9], the reference's double[3][3].
 */
#ifndef SHAPE_TYPES_H
#define SHAPE_TYPES_H

#ifdef __cplusplus
extern "C" {
#endif

/* Constants of the reference (src/shape/const.h:134-193). */
#define SHAPE_HUGENUMBER 1.0e20
#define SHAPE_SMALLVAL 1.0e-10
#define SHAPE_TINYCALFACT 1.0e-40
#define SHAPE_KM2US 6.67128190396304
#define SHAPE_KM2HZFACT 7.72139109254982e-5
#define SHAPE_MAXBINS 100
#define SHAPE_AU 1.4959787061e8
#define SHAPE_PIE 3.141592653589793

/* Delay-Doppler code methods (src/shape/const.h:159-161). */
#define SHAPE_CODE_SHORT 0
#define SHAPE_CODE_LONG_ORIG 1
#define SHAPE_CODE_LONG_MOD 2

/* Radar scattering laws evaluated by radlaw (src/shape/radlaw.c:44-148,
 * type codes from src/shape/shape2.h:847-880). The facet-dependent laws
 * (TABULARLAW, HARMCOSINE_DIFF, INHOCOSINE_DIFF) are not supported. */
#define SHAPE_RADLAW_COSINE_DIFF 1
#define SHAPE_RADLAW_GAUSSIAN 2
#define SHAPE_RADLAW_HAGFORS 3
#define SHAPE_RADLAW_COSINE_QS 4
#define SHAPE_RADLAW_GAUSSIAN_COSINE 5
#define SHAPE_RADLAW_HAGFORS_COSINE 6
#define SHAPE_RADLAW_COSINE_COSINE 7

/* Optical scattering laws evaluated by apply_photo
 * (src/shape/apply_photo.c:85-133, 226-248; codes src/shape/shape2.h:902-960).
 * Hapke and the facet-dependent (harm/inho) laws are not supported. */
#define SHAPE_OPTLAW_LAMBERT 2
#define SHAPE_OPTLAW_LOMMEL 3
#define SHAPE_OPTLAW_KAASALAINEN 11

/* One VERTEX-type model component (struct vertices_t, src/shape/shape2.h:797-805;
 * struct vertex_t/facet_t :723-748). Realization follows realize_coordinates
 * (src/shape/realize_mod.c:444-479, 532-563): x = scale * (u*r + a). */
typedef struct shape_model_desc {
    int nv;                 /* vertices */
    int nf;                 /* facets */
    const double *a;        /* [nv][3] base points (vertex_t.a) */
    const double *u;        /* [nv][3] directions of variation (vertex_t.u) */
    const double *r;        /* [nv] deviations along u (vertex_t.r.val) */
    double scale[3];        /* component scale factors (vertices_t.scalefactor[].val) */
    const int *fv;          /* [nf][3] facet corner vertex indices (facet_t.v) */
    const int *af_ptr;      /* [nv+1] CSR offsets into af_idx */
    const int *af_idx;      /* attached-facet lists (vertex_t.af), in model-file order */
    /* Several VERTEX components (shape_t.comp, src/shape/shape2.h:812-826):
     * ncomp > 1 lists them back to back in a/u/r (comp_nv vertices each)
     * and fv (comp_nf facets each), fv and af_idx holding model-wide
     * indices. Each component has its scale factors (comp_scale, replacing
     * scale[] above), rotation offsets (comp_rot: Euler angles, rad) and
     * translation offsets (comp_off, km): realize_mod scales, rotates and
     * translates its vertices (src/shape/realize_mod.c:444-512), and posvis
     * renders the components in order (src/shape/calc_fits.c:507-513).
     * ncomp 0 or 1: one component, scale[] above (the other fields unused). */
    int ncomp;
    const int *comp_nv;     /* [ncomp] */
    const int *comp_nf;     /* [ncomp] */
    const double *comp_scale;   /* [ncomp][3] */
    const double *comp_rot;     /* [ncomp][3] */
    const double *comp_off;     /* [ncomp][3] */
} shape_model_desc;

/* Radar scattering law parameters (union radscat_t, src/shape/shape2.h:852-900). */
typedef struct shape_radar_law {
    int type;               /* SHAPE_RADLAW_* */
    double diff_R, diff_C;  /* diffuse cosine law: RC_t.R, RC_t.C (or hybrid.diff) */
    double qs_R, qs_C;      /* quasispecular part: quasispec_t.R, .C (or hybrid.qs) */
    double qs_cos_cutoff;   /* quasispec_t.cos_cutoff */
} shape_radar_law;

/* Optical scattering law parameters (union optscat_t, src/shape/shape2.h:902-992). */
typedef struct shape_optical_law {
    int type;               /* SHAPE_OPTLAW_* */
    double R;               /* R_t.R (Lambert, Lommel) or kaas_t.R */
    double wt, A0, D, k;    /* kaas_t fields (Kaasalainen only) */
} shape_optical_law;

/* Evaluation switches taken from struct par_t (src/shape/shape2.h:415-710). */
typedef struct shape_eval_params {
    int pos_smooth;         /* par->pos_smooth (default 1, src/shape/read_par.c:1372) */
    int nsinc2;             /* par->nsinc2 */
    int sinc2width;         /* par->sinc2width */
    double mask_tol;        /* par->mask_tol (posmask shadow tolerance, km) */
    double mincosine_seen;  /* par->mincosine_seen */
    int mark_seen;          /* 1 = update per-facet "seen" flags (s != par->exclude_seen) */
} shape_eval_params;

/* One delay-Doppler frame with a single view (struct deldopfrm_t +
 * struct deldopview_t, src/shape/shape2.h:1097-1182). */
typedef struct shape_deldop_frame {
    int pos_n;              /* POS half-width n: (2n+1)^2 pixels */
    double km_per_pixel;    /* pos_t.km_per_pixel */
    double ae[9];           /* view ecliptic -> body transform */
    double oe[9];           /* view ecliptic -> observer transform */
    double spin[3];         /* view total spin vector, ecliptic coords (rad/day) */
    double deloff, dopoff;  /* view delay / Doppler offsets (bins) */
    int ndel, ndop;         /* delay rows, Doppler columns */
    double delcom_vig;      /* COM delay bin (1-based) after vignetting */
    double dopcom_vig;      /* COM Doppler bin (1-based) after vignetting */
    double dopDC_vig;       /* DC Doppler bin (1-based) after vignetting */
    double weight;          /* frame weight */
    double dof;             /* frame degrees of freedom */
    int cal_floating;       /* cal.state == 'f' */
    double cal;             /* cal.val when not floating */
} shape_deldop_frame;

/* Set-level delay-Doppler parameters (struct deldop_t, src/shape/shape2.h:1184-1215). */
typedef struct shape_deldop_set {
    double del_per_pixel;   /* usec per row */
    double dop_per_pixel;   /* Hz per column */
    double Ftx;             /* transmitter frequency (MHz) */
    double dopscale;        /* dopscale.val */
    int codemethod;         /* SHAPE_CODE_* */
    int spb;                /* samples per baud */
    int stride;             /* spb between adjacent rows */
    int dopfftlen;          /* Doppler FFT length */
    shape_radar_law law;    /* photo->radar[deldop->iradlaw] */
} shape_deldop_set;

/* One Doppler frame (spectrum) with a single view (struct dopfrm_t +
 * struct dopview_t, src/shape/shape2.h:1217-1263). */
typedef struct shape_doppler_frame {
    int pos_n;              /* POS half-width n: (2n+1)^2 pixels */
    double km_per_pixel;    /* pos_t.km_per_pixel */
    double ae[9];           /* view ecliptic -> body transform */
    double oe[9];           /* view ecliptic -> observer transform */
    double spin[3];         /* view total spin vector, ecliptic coords (rad/day) */
    double dopoff;          /* view Doppler offset (bins) */
    int ndop;               /* Doppler bins after vignetting */
    double dopcom_vig;      /* COM Doppler bin (1-based) after vignetting */
    double weight;          /* frame weight */
    double dof;             /* frame degrees of freedom */
    int cal_floating;       /* cal.state == 'f' */
    double cal;             /* cal.val when not floating */
    double sdev;            /* receiver noise sdev: variance of the overflow
                               spectrum bins (src/shape/pos2doppler.c:459-476) */
} shape_doppler_frame;

/* Set-level Doppler parameters (struct doppler_t, src/shape/shape2.h:1266-1287). */
typedef struct shape_doppler_set {
    double dop_per_bin;     /* Hz per bin */
    double Ftx;             /* transmitter frequency (MHz) */
    double dopscale;        /* dopscale.val */
    shape_radar_law law;    /* photo->radar[doppler->iradlaw] */
} shape_doppler_set;

/* One calculated lightcurve epoch (struct crvrend_t, src/shape/shape2.h:1344-1356). */
/* A model's spin state (struct spin_t, src/shape/shape2.h:1007-1020), values
 * only: Euler angles of the principal axes at epoch t0, the body-frame spin
 * vector and its rate of change, spin impulses (body frame, applied at their
 * epochs) and a libration of the third Euler angle. */
#define SHAPE_MAX_IMPULSES 10

/* One ephemeris entry (struct ephpnt_t, src/shape/shape2.h:1047-1052). */
typedef struct shape_ephem_point {
    double t;               /* Julian date */
    double ra, dec;         /* equatorial right ascension, declination (rad) */
    double dist;            /* distance (AU) */
} shape_ephem_point;     /* MAXIMP, src/shape/shape2.h:1003 */
typedef struct shape_spin_state {
    int pa;                       /* 1: principal-axis rotator */
    double t0;                    /* epoch of the initial conditions (days) */
    double angle[3];              /* Euler angles phi, theta, psi (rad) */
    double omega[3];              /* spin vector, body coordinates (rad/day) */
    double omegadot[3];           /* its rate of change (rad/day^2) */
    int n_impulse;                /* spin impulses, at most SHAPE_MAX_IMPULSES */
    double t_impulse[SHAPE_MAX_IMPULSES];
    double impulse[SHAPE_MAX_IMPULSES][3];
    double lib_amp, lib_freq, lib_phase;   /* psi libration: amplitude, frequency, phase */
    double inertia[3];            /* principal moments of inertia (non-principal-axis rotation) */
} shape_spin_state;

typedef struct shape_lghtcrv_point {
    int pos_n;
    double km_per_pixel;
    double ae[9], oe[9], se[9];
    double solar_phase;     /* lghtcrv->solar_phase[i] (radians) */
} shape_lghtcrv_point;

/* Lightcurve set (struct lghtcrv_t, src/shape/shape2.h:1358-1398) with one view per point. */
typedef struct shape_lghtcrv_set {
    int ncalc;              /* calculated epochs */
    int n;                  /* observed points */
    const double *x;        /* [ncalc] calculated epochs (ascending) */
    const double *t;        /* [n] observation epochs */
    const double *obs;      /* [n] observed intensities */
    const double *oneovervar; /* [n] 1/variance */
    double weight, dof;
    int cal_floating;
    double cal;
    shape_optical_law law;  /* photo->optical[lghtcrv->ioptlaw] */
} shape_lghtcrv_set;

/* Plane-of-sky frame (struct posetfrm_t, src/shape/shape2.h:1303-1325) with
 * one view: the sky rendering's POS window and view geometry, and the fit
 * grid the rendering is resampled onto (calc_poset,
 * src/shape/calc_fits.c:1156-1330). The observed image and its 1/variance
 * are ncol x nrow arrays, element (i, j) (1-based column i, row j) at
 * (i - 1) * nrow + (j - 1), as frame->obs.b[i][j]. */
typedef struct shape_poset_frame {
    int pos_n;              /* sky rendering: (2 pos_n + 1)^2 pixels */
    double km_per_pixel;    /* frame->pos.km_per_pixel */
    double ae[9], oe[9], se[9];
    double solar_phase;     /* view[v0].solar_phase (radians) */
    int ncol, nrow;         /* fit image (after vignetting) */
    double fit_km_per_pixel;/* frame->fit.km_per_pixel */
    double colcom_vig, rowcom_vig;  /* 1-based COM column and row at zero offsets */
    double xoff, yoff;      /* frame->off[0..1].val (fit-grid pixels) */
    double northangle;      /* radians, clockwise heading of north */
    double weight, dof;
} shape_poset_frame;

/* resampim interpolation modes (par->poset_resample, src/util/resampim.c) */
#define SHAPE_RESAMPLE_NONE 0
#define SHAPE_RESAMPLE_NEAREST 1
#define SHAPE_RESAMPLE_BILINEAR 2
#define SHAPE_RESAMPLE_BICUBIC 3     /* not supported (SHAPE_E_UNSUPPORTED) */
#define SHAPE_RESAMPLE_CUBICCONV 4

/* Plane-of-sky set (struct poset_t, src/shape/shape2.h:1328-1341) with one
 * view per frame; the calibration always floats (chi2_poset). */
typedef struct shape_poset_set {
    shape_optical_law law;  /* photo->optical[poset->ioptlaw] */
    int resample;           /* par->poset_resample: SHAPE_RESAMPLE_* */
    int rebin;              /* par->image_rebin */
} shape_poset_set;

/* Per-frame results of a plane-of-sky frame. */
typedef struct shape_poset_result {
    int outbnd;             /* 1: the observer view's posvis returned 1; 2: the sun view's; 3: both */
    double posbnd_logsum;   /* sum over those views of dof/2 * posbnd_logfactor (calc_poset) */
    int badposet;           /* checkposet returned 1 */
    double badposet_logfactor;  /* checkposet's log area ratio */
    double o2, m2, om;      /* chi-square partial sums */
    double cal;             /* om/m2, or TINYCALFACT when om <= 0 */
    double chi2;            /* frame chi-square */
} shape_poset_result;

/* Per-frame results of one radar frame evaluation (delay-Doppler image or
 * Doppler spectrum; a Doppler frame leaves the delay fields at their blank
 * values, and its o2 / m2 include the overflow spectrum's terms). */
typedef struct shape_deldop_result {
    int outbnd;             /* posvis returned 1 (model beyond POS window) */
    double posbnd_logfactor;/* pos_t.posbnd_logfactor */
    int badradar;           /* pos2deldop returned 1 */
    double badradar_logfactor;
    int xlim[2], ylim[2];   /* POS region touched by the model */
    int idellim[2], idoplim[2];
    double dellim[2], doplim[2];
    double o2, m2, om;      /* chi-square partial sums */
    double cal;             /* calibration used (floating: om/m2) */
    double chi2;            /* frame chi-square */
} shape_deldop_result;

#ifdef __cplusplus
}
#endif
#endif
