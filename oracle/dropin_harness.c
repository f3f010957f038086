/*
 * Test harness of the calc_fits drop-in (shape-cuda-v1.2_b200/dropin/
 * shape_b200_dropin.c), compiled by oracle/build_dropin.sh with the drop-in's
 * entry points renamed so that they sit beside the reference's own calc_fits
 * in one process. Each function runs on a session made by ref_harness.c.
 */
#include "head.h"

#include "ref_session.h"

void calc_fits_b200dropin(struct par_t *par, struct mod_t *mod, struct dat_t *dat);
double calc_fits_chi2_b200dropin(struct par_t *par, struct mod_t *mod, struct dat_t *dat);

/* realize_mod, the drop-in calc_fits, then the reference's chi2 on the
 * written-back fit images: objective()'s sequence (src/shape/bestfit.c:748-790). */
double ref_dropin_evaluate(void *h)
{
    ref_session *S = h;
    realize_mod(&S->par, &S->mod);
    calc_fits_b200dropin(&S->par, &S->mod, &S->dat);
    return chi2(&S->par, &S->dat, 0);
}

/* realize_mod, then the drop-in's combined calc_fits + chi2 (totals only). */
double ref_dropin_objective(void *h)
{
    ref_session *S = h;
    realize_mod(&S->par, &S->mod);
    return calc_fits_chi2_b200dropin(&S->par, &S->mod, &S->dat);
}

/* dat->chi2, set chi2 and per-frame chi2 / cal of set s (for comparisons). */
void ref_get_chi2s(void *h, int s, double *dat_chi2, double *set_chi2, double *frame_chi2,
                   double *frame_cal)
{
    ref_session *S = h;
    *dat_chi2 = S->dat.chi2;
    *set_chi2 = S->dat.set[s].chi2;
    if (S->dat.set[s].type == DELAY) {
        struct deldop_t *dd = &S->dat.set[s].desc.deldop;
        for (int f = 0; f < dd->nframes; f++) {
            frame_chi2[f] = dd->frame[f].chi2;
            frame_cal[f] = dd->frame[f].cal.val;
        }
    } else if (S->dat.set[s].type == DOPPLER) {
        struct doppler_t *dp = &S->dat.set[s].desc.doppler;
        for (int f = 0; f < dp->nframes; f++) {
            frame_chi2[f] = dp->frame[f].chi2;
            frame_cal[f] = dp->frame[f].cal.val;
        }
    } else if (S->dat.set[s].type == LGHTCRV) {
        frame_chi2[0] = S->dat.set[s].chi2;
        frame_cal[0] = S->dat.set[s].desc.lghtcrv.cal.val;
    }
}

/* ------------------------------------------------------------------------
 * The plane-of-sky drop-ins (shape-cuda-v1.2_b200/dropin/shape_b200_pos.c,
 * compiled with the prefix b200dropin_) beside the reference's own posclr,
 * posvis, pos2deldop, posmask and apply_photo, on POS frames allocated the
 * reference's way. `which` = 0 runs the reference's routine, 1 the drop-in.
 */
int b200dropin_posvis(struct vertices_t *verts, double orbit_offset[3], struct pos_t *pos, int smooth, int src,
                      int body, int comp);
int b200dropin_pos2deldop(struct par_t *par, struct photo_t *photo, double orbit_xoff, double orbit_yoff,
                          double orbit_dopoff, struct deldop_t *deldop, int body, int set, int frm, int v);
void b200dropin_posclr(struct pos_t *pos);
void b200dropin_posmask(struct pos_t *pos, double tol);
double b200dropin_apply_photo(struct mod_t *mod, int ilaw, double phase, double intensityfactor,
                              struct pos_t *pos, int body, int s, int frm);

void *dh_pos_new(int n, double kmpp, const double *ae, const double *oe, const double *se, int bistatic)
{
    struct pos_t *pos = calloc(1, sizeof *pos);
    pos->n = n;
    pos->km_per_pixel = kmpp;
    pos->b = matrix(-n, n, -n, n); pos->cose = matrix(-n, n, -n, n); pos->cosi = matrix(-n, n, -n, n);
    pos->z = matrix(-n, n, -n, n);
    pos->body = imatrix(-n, n, -n, n); pos->comp = imatrix(-n, n, -n, n); pos->f = imatrix(-n, n, -n, n);
    pos->cosill = matrix(-n, n, -n, n); pos->zill = matrix(-n, n, -n, n);
    pos->bodyill = imatrix(-n, n, -n, n); pos->compill = imatrix(-n, n, -n, n); pos->fill = imatrix(-n, n, -n, n);
    pos->bistatic = bistatic;
    /* matrix() leaves the rows uninitialized and posclr only clears the
     * sun view's images of a bistatic frame: a fixed fill makes two frames
     * comparable, and shows any write to images the routines must not touch */
    for (int i = -n; i <= n; i++)
        for (int j = -n; j <= n; j++) {
            pos->b[i][j] = pos->cose[i][j] = pos->cosi[i][j] = pos->z[i][j] = 0.25;
            pos->cosill[i][j] = pos->zill[i][j] = 0.25;
            pos->body[i][j] = pos->comp[i][j] = pos->f[i][j] = -7;
            pos->bodyill[i][j] = pos->compill[i][j] = pos->fill[i][j] = -7;
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            pos->ae[i][j] = ae[3 * i + j]; pos->oe[i][j] = oe[3 * i + j]; pos->se[i][j] = se[3 * i + j];
        }
    return pos;
}

void dh_pos_free(void *p)
{
    struct pos_t *pos = p;
    const int n = pos->n;
    free_matrix(pos->b, -n, n, -n, n); free_matrix(pos->cose, -n, n, -n, n);
    free_matrix(pos->cosi, -n, n, -n, n); free_matrix(pos->z, -n, n, -n, n);
    free_imatrix(pos->body, -n, n, -n, n); free_imatrix(pos->comp, -n, n, -n, n);
    free_imatrix(pos->f, -n, n, -n, n); free_matrix(pos->cosill, -n, n, -n, n);
    free_matrix(pos->zill, -n, n, -n, n); free_imatrix(pos->bodyill, -n, n, -n, n);
    free_imatrix(pos->compill, -n, n, -n, n); free_imatrix(pos->fill, -n, n, -n, n);
    free(pos);
}

void dh_posclr(void *p, int which)
{
    if (which) b200dropin_posclr(p); else posclr(p);
}

/* posvis of the session's realized model component (realize_mod first). */
int dh_posvis(void *h, void *p, int which, const double *off, int smooth, int src, int body, int comp)
{
    ref_session *S = h;
    struct vertices_t *verts = &S->mod.shape.comp[0].real;
    double o[3] = {off[0], off[1], off[2]};
    return which ? b200dropin_posvis(verts, o, p, smooth, src, body, comp) : posvis(verts, o, p, smooth, src, body, comp);
}

void dh_posmask(void *p, int which, double tol)
{
    if (which) b200dropin_posmask(p, tol); else posmask(p, tol);
}

double dh_apply_photo(void *h, void *p, int which, int ilaw, double phase, double intensityfactor, int body)
{
    ref_session *S = h;
    return which ? b200dropin_apply_photo(&S->mod, ilaw, phase, intensityfactor, p, body, 0, 0)
                 : apply_photo(&S->mod, ilaw, phase, intensityfactor, p, body, 0, 0);
}

/* Copies of every image and limit of a POS frame ([i][j] order). */
void dh_pos_get(void *p, double *b, double *cose, double *cosi, double *z, int *body, int *comp, int *f,
                double *cosill, double *zill, int *bodyill, int *compill, int *fill, int lims[8],
                double *logfactor)
{
    struct pos_t *pos = p;
    const int n = pos->n, side = 2 * n + 1;
    for (int i = -n; i <= n; i++)
        for (int j = -n; j <= n; j++) {
            size_t q = (size_t)(i + n) * side + (size_t)(j + n);
            b[q] = pos->b[i][j]; cose[q] = pos->cose[i][j]; cosi[q] = pos->cosi[i][j]; z[q] = pos->z[i][j];
            body[q] = pos->body[i][j]; comp[q] = pos->comp[i][j]; f[q] = pos->f[i][j];
            cosill[q] = pos->cosill[i][j]; zill[q] = pos->zill[i][j];
            bodyill[q] = pos->bodyill[i][j]; compill[q] = pos->compill[i][j]; fill[q] = pos->fill[i][j];
        }
    lims[0] = pos->xlim[0]; lims[1] = pos->xlim[1]; lims[2] = pos->ylim[0]; lims[3] = pos->ylim[1];
    lims[4] = pos->xlim2[0]; lims[5] = pos->xlim2[1]; lims[6] = pos->ylim2[0]; lims[7] = pos->ylim2[1];
    *logfactor = pos->posbnd_logfactor;
}

/* pos2deldop of delay-Doppler frame f of set s: the frame's POS is cleared
 * and filled by the reference's posvis from the frame's view (as
 * calc_deldop does, src/shape/calc_fits.c:492-540), optionally a second
 * body at orbit offset off2 (body 1), the fit image is cleared, then the
 * reference's or the drop-in's pos2deldop runs for `body`. Outputs are
 * read with ref_get_deldop_frame. Returns badradar. */
int dh_pos2deldop(void *h, int s, int f, int which, const double *off2, double xoff, double yoff,
                  double dopoff, int body)
{
    ref_session *S = h;
    struct deldop_t *dd = &S->dat.set[s].desc.deldop;
    struct deldopfrm_t *fr = &dd->frame[f];
    struct pos_t *pos = &fr->pos;
    realize_mod(&S->par, &S->mod);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) { pos->ae[i][j] = fr->view[0].ae[i][j]; pos->oe[i][j] = fr->view[0].oe[i][j]; }
    posclr(pos);
    double o0[3] = {0.0, 0.0, 0.0};
    struct vertices_t *verts = &S->mod.shape.comp[0].real;
    posvis(verts, o0, pos, (int)S->par.pos_smooth, 0, 0, 0);
    if (off2) {
        double o1[3] = {off2[0], off2[1], off2[2]};
        posvis(verts, o1, pos, (int)S->par.pos_smooth, 0, 1, 0);
    }
    for (int i = 1; i <= fr->ndel; i++)
        for (int j = 1; j <= fr->ndop; j++) fr->fit[i][j] = 0.0;
    return which ? b200dropin_pos2deldop(&S->par, &S->mod.photo, xoff, yoff, dopoff, dd, body, s, f, 0)
                 : pos2deldop(&S->par, &S->mod.photo, xoff, yoff, dopoff, dd, body, s, f, 0);
}
