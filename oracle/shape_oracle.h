/*
 * CPU oracle for SHAPE's model-evaluation hot path. TEST INFRASTRUCTURE ONLY:
 * this code is the checker used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py. The product (libshape_b200.so) never links,
 * loads or calls it.
 *
 * It restates, in plain C over flat arrays, the reference CPU algorithm of
 * h6294443/shape-cuda-v1.2 for one VERTEX component and one body, keeping
 * the floating-point operation order of the reference so that FP64 results
 * match bit for bit. Each function cites the reference lines it follows.
 * Parity of this restatement is pinned against the reference's own code
 * compiled in oracle/_ref (oracle/build_ref.sh) through golden vectors in
 * tests/golden/.
 */
#ifndef SHAPE_ORACLE_H
#define SHAPE_ORACLE_H

#include "../include/shape_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Realized vertex model (outputs of realize_coordinates). */
typedef struct orc_real {
    int nv, nf;
    double *x;      /* [nv][3] vertex coordinates */
    double *vn;     /* [nv][3] vertex normals */
    double *fn;     /* [nf][3] facet normals */
    double *area;   /* [nf] facet areas */
    const int *fv;  /* [nf][3] */
} orc_real;

/* One POS image with the arrays of struct pos_t that the path uses. Body and
 * component maps are implied: one body (0) and one component (0), so
 * body = comp = (f >= 0 ? 0 : -1). */
typedef struct orc_pos {
    int n;
    double kmpp;
    double ae[9], oe[9], se[9];
    int bistatic;
    double *b, *cose, *cosi, *z;  /* [(2n+1)^2] */
    int *f;
    double *cosill, *zill;        /* bistatic only */
    int *fill;
    int xlim[2], ylim[2], xlim2[2], ylim2[2];
    double posbnd_logfactor;
} orc_pos;

void orc_realize_vertex(const shape_model_desc *m, double *x, double *vn,
                        double *fn, double *area);
void orc_posclr(orc_pos *pos);
int orc_posvis(const orc_real *real, const double orbit_offset[3], orc_pos *pos,
               int smooth, int src);
void orc_posmask(orc_pos *pos, double tol);
double orc_radlaw(const shape_radar_law *law, double cosinc);
int orc_pos2deldop(const shape_eval_params *par, const shape_deldop_set *set,
                   const shape_deldop_frame *frm, const orc_pos *pos,
                   double *fit, shape_deldop_result *res);
int orc_pos2doppler(const shape_eval_params *par, const shape_doppler_set *set,
                    const shape_doppler_frame *frm, const orc_pos *pos, double *fit,
                    shape_deldop_result *res, double ovf[4]);
void orc_chi2_doppler_frame(const double *obs, const double *oneovervar, const double *fit,
                            int ndop, double ovf_o2, double ovf_m2, double weight,
                            int cal_floating, double cal_in, double *o2, double *m2,
                            double *om, double *cal, double *chi2);
void orc_doppler_frame(const shape_eval_params *par, const orc_real *real,
                       const shape_doppler_set *set, const shape_doppler_frame *frm,
                       const double *obs, const double *oneovervar,
                       orc_pos *pos, double *fit, unsigned char *seen,
                       shape_deldop_result *res);
double orc_apply_photo(const shape_optical_law *law, double phase,
                       double intensityfactor, orc_pos *pos);
void orc_chi2_frame(const double *obs, const double *oneovervar, const double *fit,
                    int npix, double weight, int cal_floating, double cal_in,
                    double *o2, double *m2, double *om, double *cal, double *chi2);

/* One delay-Doppler frame of calc_deldop (posclr, posvis, seen marks,
 * clrmat, pos2deldop; src/shape/calc_fits.c:492-551) followed by its
 * chi2_deldop term (src/shape/chi2.c:405-460). pos must be allocated for
 * frm->pos_n. seen may be NULL. Returns nothing; results go to res/fit. */
void orc_deldop_frame(const shape_eval_params *par, const orc_real *real,
                      const shape_deldop_set *set, const shape_deldop_frame *frm,
                      const double *obs, const double *oneovervar,
                      orc_pos *pos, double *fit, unsigned char *seen,
                      shape_deldop_result *res);

/* A smeared delay-Doppler frame (src/shape/calc_fits.c:475-594): views in
 * rendering order, the epoch view last; fit receives the mean over the
 * views. *badradar_term is the frame's badradar contribution (dof *
 * log-factor / nviews summed over the views flagged) and *badradar_any its
 * flag; res holds the epoch view's posbnd, limits and the chi-square terms. */
void orc_deldop_frame_views(const shape_eval_params *par, const orc_real *real,
                            const shape_deldop_set *set, int nviews, const shape_deldop_frame *views,
                            const double *obs, const double *oneovervar,
                            orc_pos *pos, double *fit, unsigned char *seen,
                            shape_deldop_result *res, int *badradar_any, double *badradar_term);

/* One calculated lightcurve point of calc_lghtcrv
 * (src/shape/calc_fits.c:1629-1716): returns y[i]. outbnd_logsum receives the
 * 0.5-weighted posbnd log-factor sum for this point and *outbnd the flag. */
double orc_lghtcrv_point(const shape_eval_params *par, const orc_real *real,
                         const shape_optical_law *law, const shape_lghtcrv_point *pt,
                         orc_pos *pos, unsigned char *seen, int *outbnd,
                         double *outbnd_logsum);

/* Natural cubic spline (second derivatives) and its evaluation. */
void orc_spline_natural(const double *x, const double *y, int n, double *y2);
double orc_splint(const double *x, const double *y, const double *y2, int n, double t);

/* Allocation helpers for orc_pos. */
int orc_pos_alloc(orc_pos *pos, int n, int bistatic);
void orc_pos_free(orc_pos *pos);

#ifdef __cplusplus
}
#endif
#endif
