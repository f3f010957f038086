/*
 * Drop-in replacements of the reference's plane-of-sky routines for the
 * B200 engine, with the reference's signatures (src/shape/shape2.h:1446,
 * 1495, 1501-1503):
 *
 *   int posvis(struct vertices_t *verts, double orbit_offset[3],
 *              struct pos_t *pos, int smooth, int src, int body, int comp)
 *   int pos2deldop(struct par_t *par, struct photo_t *photo,
 *                  double orbit_xoff, double orbit_yoff, double orbit_dopoff,
 *                  struct deldop_t *deldop, int body, int set, int frm, int v)
 *   void posclr(struct pos_t *pos)
 *   void posmask(struct pos_t *pos, double tol)
 *   double apply_photo(struct mod_t *mod, int ilaw, double phase,
 *                      double intensityfactor, struct pos_t *pos, int body,
 *                      int s, int frm)
 *
 * Like shape_b200_dropin.c this file is compiled inside the reference tree
 * with its own head.h and linked against libshape_b200.so; in a build that
 * uses it, the reference's posvis.c, pos2deldop.c, posclr.c, posmask.c and
 * apply_photo.c are left out. Each call gathers the NR-offset rows of the
 * POS matrices (allocated row by row, src/nr/nrutil.c:59-74) into one
 * [i][j] array per image, runs the engine's one-view entry point on the
 * device (shape_posvis, shape_pos2deldop, shape_posmask, shape_apply_photo)
 * and scatters what it wrote back into the rows, with the reference's side
 * effects on pos and deldop. Unsupported inputs (facet-dependent laws)
 * stop in bailout(), the reference's error convention.
 *
 * Environment: SHAPE_B200_DEVICE = CUDA device index (default 0). Compile
 * with -DSHAPE_B200_POS_PREFIX=name_ to give the five functions other names
 * (the tests run them beside the reference's own).
 */
#include "head.h"

#include <stdlib.h>
#include <string.h>

#include "shape_b200.h"
#include "shape_b200_dropin_common.h"

#ifdef SHAPE_B200_POS_PREFIX
#define B200_CAT2(a, b) a##b
#define B200_CAT(a, b) B200_CAT2(a, b)
#define B200_NAME(f) B200_CAT(SHAPE_B200_POS_PREFIX, f)
#else
#define B200_NAME(f) f
#endif

static int b200_pos_device(void)
{
    const char *e = getenv("SHAPE_B200_DEVICE");
    return e ? atoi(e) : 0;
}

/* ------------------------------------------------- NR rows <-> flat arrays */

static double *gather_d(double **m, int n)
{
    const int side = 2 * n + 1;
    double *a = malloc(sizeof(double) * (size_t)side * side);
    if (!a) bailout("shape_b200: out of host memory\n");
    for (int i = -n; i <= n; i++) memcpy(a + (size_t)(i + n) * side, &m[i][-n], sizeof(double) * side);
    return a;
}

static int *gather_i(int **m, int n)
{
    const int side = 2 * n + 1;
    int *a = malloc(sizeof(int) * (size_t)side * side);
    if (!a) bailout("shape_b200: out of host memory\n");
    for (int i = -n; i <= n; i++) memcpy(a + (size_t)(i + n) * side, &m[i][-n], sizeof(int) * side);
    return a;
}

static void scatter_d(double **m, double *a, int n)
{
    const int side = 2 * n + 1;
    for (int i = -n; i <= n; i++) memcpy(&m[i][-n], a + (size_t)(i + n) * side, sizeof(double) * side);
    free(a);
}

static void scatter_i(int **m, int *a, int n)
{
    const int side = 2 * n + 1;
    for (int i = -n; i <= n; i++) memcpy(&m[i][-n], a + (size_t)(i + n) * side, sizeof(int) * side);
    free(a);
}

static void pos_view_of(const struct pos_t *pos, shape_pos_view *v)
{
    memset(v, 0, sizeof *v);
    v->n = pos->n;
    v->km_per_pixel = pos->km_per_pixel;
    rm9(v->ae, (double(*)[3])pos->ae);
    rm9(v->oe, (double(*)[3])pos->oe);
    rm9(v->se, (double(*)[3])pos->se);
    v->bistatic = pos->bistatic;
}

static void pos_limits_in(const struct pos_t *pos, shape_pos_images *im)
{
    im->xlim[0] = pos->xlim[0]; im->xlim[1] = pos->xlim[1];
    im->ylim[0] = pos->ylim[0]; im->ylim[1] = pos->ylim[1];
    im->xlim2[0] = pos->xlim2[0]; im->xlim2[1] = pos->xlim2[1];
    im->ylim2[0] = pos->ylim2[0]; im->ylim2[1] = pos->ylim2[1];
}

/* ---------------------------------------------------------------- posvis */

int B200_NAME(posvis)(struct vertices_t *verts, double orbit_offset[3], struct pos_t *pos, int smooth, int src,
                      int body, int comp)
{
    const int nv = verts->nv, nf = verts->nf, n = pos->n;
    double *x = malloc(sizeof(double) * 3 * (size_t)nv), *vn = malloc(sizeof(double) * 3 * (size_t)nv);
    double *fn = malloc(sizeof(double) * 3 * (size_t)nf);
    int *fv = malloc(sizeof(int) * 3 * (size_t)nf);
    if (!x || !vn || !fn || !fv) bailout("shape_b200: out of host memory\n");
    for (int i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) { x[3 * i + k] = verts->v[i].x[k]; vn[3 * i + k] = verts->v[i].n[k]; }
    for (int f = 0; f < nf; f++)
        for (int k = 0; k < 3; k++) { fn[3 * f + k] = verts->f[f].n[k]; fv[3 * f + k] = verts->f[f].v[k]; }
    shape_pos_view view;
    memset(&view, 0, sizeof view);
    pos_view_of(pos, &view);
    shape_pos_images im;
    memset(&im, 0, sizeof im);
    pos_limits_in(pos, &im);
    if (src) {
        im.zill = gather_d(pos->zill, n); im.cosill = gather_d(pos->cosill, n);
        im.fill = gather_i(pos->fill, n); im.bodyill = gather_i(pos->bodyill, n);
        im.compill = gather_i(pos->compill, n);
    } else {
        im.z = gather_d(pos->z, n); im.cose = gather_d(pos->cose, n);
        if (pos->bistatic) im.cosi = gather_d(pos->cosi, n);
        im.f = gather_i(pos->f, n); im.body = gather_i(pos->body, n); im.comp = gather_i(pos->comp, n);
    }
    int outbnd = shape_posvis(b200_pos_device(), &view, &im, nv, x, vn, nf, fv, fn, orbit_offset, smooth, src,
                              body, comp);
    b200_check(outbnd, "posvis");
    free(x); free(vn); free(fn); free(fv);
    if (src) {
        scatter_d(pos->zill, im.zill, n); scatter_d(pos->cosill, im.cosill, n);
        scatter_i(pos->fill, im.fill, n); scatter_i(pos->bodyill, im.bodyill, n);
        scatter_i(pos->compill, im.compill, n);
        pos->xlim2[0] = im.xlim2[0]; pos->xlim2[1] = im.xlim2[1];
        pos->ylim2[0] = im.ylim2[0]; pos->ylim2[1] = im.ylim2[1];
    } else {
        scatter_d(pos->z, im.z, n); scatter_d(pos->cose, im.cose, n);
        if (pos->bistatic) scatter_d(pos->cosi, im.cosi, n);
        scatter_i(pos->f, im.f, n); scatter_i(pos->body, im.body, n); scatter_i(pos->comp, im.comp, n);
        pos->xlim[0] = im.xlim[0]; pos->xlim[1] = im.xlim[1];
        pos->ylim[0] = im.ylim[0]; pos->ylim[1] = im.ylim[1];
    }
    pos->posbnd_logfactor = im.posbnd_logfactor;
    return outbnd;
}

/* ------------------------------------------------------------ pos2deldop */

int B200_NAME(pos2deldop)(struct par_t *par, struct photo_t *photo, double orbit_xoff, double orbit_yoff,
                          double orbit_dopoff, struct deldop_t *deldop, int body, int set, int frm, int v)
{
    (void)set;
    struct deldopfrm_t *frame = &deldop->frame[frm];
    struct pos_t *pos = &frame->pos;
    const int n = pos->n, ndel = frame->ndel, ndop = frame->ndop;
    shape_pos_view view;
    memset(&view, 0, sizeof view);
    pos_view_of(pos, &view);
    shape_pos_images im;
    memset(&im, 0, sizeof im);
    pos_limits_in(pos, &im);
    im.z = gather_d(pos->z, n);
    im.cose = gather_d(pos->cose, n);
    im.body = gather_i(pos->body, n);
    shape_eval_params ep;
    memset(&ep, 0, sizeof ep);
    ep.nsinc2 = par->nsinc2;
    ep.sinc2width = par->sinc2width;
    shape_deldop_set S;
    memset(&S, 0, sizeof S);
    S.del_per_pixel = deldop->del_per_pixel;
    S.dop_per_pixel = deldop->dop_per_pixel;
    S.Ftx = deldop->Ftx;
    S.dopscale = deldop->dopscale.val;
    S.codemethod = deldop->codemethod;
    S.spb = deldop->spb;
    S.stride = deldop->stride;
    S.dopfftlen = deldop->dopfftlen;
    S.law = radar_law_of(photo, deldop->iradlaw);
    shape_deldop_frame F;
    memset(&F, 0, sizeof F);
    F.pos_n = n;
    F.km_per_pixel = pos->km_per_pixel;
    rm9(F.oe, frame->view[v].oe);
    for (int k = 0; k < 3; k++) F.spin[k] = frame->view[v].spin[k];
    F.deloff = frame->view[v].deloff;
    F.dopoff = frame->view[v].dopoff;
    F.ndel = ndel;
    F.ndop = ndop;
    F.delcom_vig = frame->delcom_vig;
    F.dopcom_vig = frame->dopcom_vig;
    F.dopDC_vig = frame->dopDC_vig;
    /* the caller's fit image, added to (src/shape/calc_fits.c:538 clears it) */
    double *fit = malloc(sizeof(double) * (size_t)ndel * ndop);
    if (!fit) bailout("shape_b200: out of host memory\n");
    for (int i = 1; i <= ndel; i++) memcpy(fit + (size_t)(i - 1) * ndop, &frame->fit[i][1], sizeof(double) * ndop);
    shape_deldop_result res;
    memset(&res, 0, sizeof res);
    double km2Hz = 0.0;
    int badradar = shape_pos2deldop(b200_pos_device(), &view, &im, &ep, &S, &F, orbit_xoff, orbit_yoff,
                                    orbit_dopoff, body, fit, &res, &km2Hz);
    b200_check(badradar, "pos2deldop");
    for (int i = 1; i <= ndel; i++) memcpy(&frame->fit[i][1], fit + (size_t)(i - 1) * ndop, sizeof(double) * ndop);
    free(fit);
    free(im.z); free(im.cose); free(im.body);
    frame->view[v].km2Hz = km2Hz;
    frame->idellim[0] = res.idellim[0]; frame->idellim[1] = res.idellim[1];
    frame->idoplim[0] = res.idoplim[0]; frame->idoplim[1] = res.idoplim[1];
    frame->dellim[0] = res.dellim[0]; frame->dellim[1] = res.dellim[1];
    frame->doplim[0] = res.doplim[0]; frame->doplim[1] = res.doplim[1];
    frame->badradar_logfactor = res.badradar_logfactor;
    /* this version of the reference keeps no overflow image
       (src/shape/pos2deldop.c:512-519) */
    frame->overflow_o2 = frame->overflow_m2 = frame->overflow_xsec = 0.0;
    frame->overflow_delmean = frame->overflow_dopmean = 0.0;
    return badradar;
}

/* ---------------------------------------------------------------- posclr */

void B200_NAME(posclr)(struct pos_t *pos)
{
    /* the caller's host images: cleared where they are (src/shape/posclr.c:24-67) */
    const int n = pos->n;
    for (int i = -n; i <= n; i++)
        for (int j = -n; j <= n; j++) {
            pos->b[i][j] = pos->cose[i][j] = pos->cosi[i][j] = 0.0;
            pos->z[i][j] = -HUGENUMBER;
            pos->body[i][j] = pos->comp[i][j] = pos->f[i][j] = -1;
        }
    pos->xlim[0] = pos->ylim[0] = n;
    pos->xlim[1] = pos->ylim[1] = -n;
    if (pos->bistatic) {
        for (int i = -n; i <= n; i++)
            for (int j = -n; j <= n; j++) {
                pos->cosill[i][j] = 0.0;
                pos->zill[i][j] = -HUGENUMBER;
                pos->bodyill[i][j] = pos->compill[i][j] = pos->fill[i][j] = -1;
            }
        pos->xlim2[0] = pos->ylim2[0] = n;
        pos->xlim2[1] = pos->ylim2[1] = -n;
    }
}

/* --------------------------------------------------------------- posmask */

void B200_NAME(posmask)(struct pos_t *pos, double tol)
{
    const int n = pos->n;
    shape_pos_view view;
    memset(&view, 0, sizeof view);
    pos_view_of(pos, &view);
    shape_pos_images im;
    memset(&im, 0, sizeof im);
    im.z = gather_d(pos->z, n); im.zill = gather_d(pos->zill, n); im.cose = gather_d(pos->cose, n);
    im.f = gather_i(pos->f, n); im.comp = gather_i(pos->comp, n); im.body = gather_i(pos->body, n);
    im.fill = gather_i(pos->fill, n); im.compill = gather_i(pos->compill, n);
    im.bodyill = gather_i(pos->bodyill, n);
    b200_check(shape_posmask(b200_pos_device(), &view, &im, tol), "posmask");
    scatter_d(pos->cose, im.cose, n);
    free(im.z); free(im.zill); free(im.f); free(im.comp); free(im.body);
    free(im.fill); free(im.compill); free(im.bodyill);
}

/* ----------------------------------------------------------- apply_photo */

double B200_NAME(apply_photo)(struct mod_t *mod, int ilaw, double phase, double intensityfactor,
                              struct pos_t *pos, int body, int s, int frm)
{
    (void)s; (void)frm;
    const int n = pos->n;
    shape_optical_law law = optical_law_of(&mod->photo, ilaw);
    shape_pos_view view;
    memset(&view, 0, sizeof view);
    pos_view_of(pos, &view);
    shape_pos_images im;
    memset(&im, 0, sizeof im);
    pos_limits_in(pos, &im);
    im.b = gather_d(pos->b, n); im.cose = gather_d(pos->cose, n); im.cosi = gather_d(pos->cosi, n);
    im.body = gather_i(pos->body, n);
    double sum = 0.0;
    b200_check(shape_apply_photo(b200_pos_device(), &law, phase, intensityfactor, &view, &im, body, &sum),
               "apply_photo");
    scatter_d(pos->b, im.b, n);
    free(im.cose); free(im.cosi); free(im.body);
    return sum;
}
