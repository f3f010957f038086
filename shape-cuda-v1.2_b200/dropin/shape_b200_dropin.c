/*
 * Drop-in replacement of the reference's calc_fits for the B200 engine.
 *
 * This file is compiled INSIDE the reference tree, next to
 * src/shape/calc_fits.c, with the reference's own head.h, and linked against
 * libshape_b200.so:
 *
 *   void calc_fits(struct par_t *par, struct mod_t *mod, struct dat_t *dat)
 *       keeps the signature of src/shape/calc_fits.c:340 (declared at
 *       src/shape/shape2.h:1451). It evaluates every dataset on the GPU and
 *       writes back what the reference's calc_fits leaves in par, mod and dat:
 *       par->posbnd / posbnd_logfactor / badradar / badradar_logfactor
 *       (src/shape/calc_fits.c:349-354, 407-409), facet "seen" flags
 *       (:358-360, 522-530), every delay-Doppler frame's fit image, region
 *       limits and badradar_logfactor (src/shape/pos2deldop.c:279-288,
 *       337-354, 543-548), every lightcurve's y and fit arrays
 *       (src/shape/calc_fits.c:1712-1716, 1923-1933), every Doppler frame's
 *       fit spectrum, limits and overflow-spectrum terms
 *       (src/shape/pos2doppler.c:170-176, 451-499), and, for the write
 *       action, the POS z / cos(e) / facet images. The reference's chi2()
 *       (src/shape/chi2.c:240) then runs unchanged on those images.
 *
 *   double calc_fits_chi2_b200(struct par_t *par, struct mod_t *mod,
 *                              struct dat_t *dat)
 *       replaces the two lines `calc_fits(spar, smod, sdat); err =
 *       chi2(spar, sdat, 0);` of objective() (src/shape/bestfit.c:789-790).
 *       It evaluates on the GPU and copies back only the totals: the par
 *       flags above, cal and chi2 of every frame and lightcurve, set chi2 and
 *       dat->chi2, which it returns. No fit image crosses PCIe.
 *
 * The engine is built on the first call and rebuilt whenever the data or
 * the view geometry change (a fingerprint of everything except the free
 * shape parameters is compared on every call); the vertex deviations r and
 * the component scale factors, the parameters bestfit varies in a shape fit
 * (src/shape/mkparlist.c:218-235), are pushed on every call.
 *
 * Supported inputs (anything else stops with bailout(), the reference's
 * error convention): one VERTEX component; delay-Doppler, Doppler,
 * lightcurve and plane-of-sky sets with one view per frame/point (speckle
 * off; no bicubic plane-of-sky resampling); radar laws COSINELAW_DIFF,
 * GAUSSIANLAW, HAGFORSLAW, COSINELAW_QS and the three hybrids; optical laws
 * LAMBERTLAW, LOMMEL and KAASALAINEN; dd_gamma = 1; exclude_seen not naming
 * a set of the dataset.
 *
 * Environment: SHAPE_B200_FORM = plain_fp64 | batched_fp64 (default) |
 * batched_fp32; SHAPE_B200_DEVICE = CUDA device index (default 0).
 * Set SHAPE_B200_CALC_FITS to another name at compile time to build the
 * replacement beside the reference's own calc_fits (as the tests do).
 */
#include "head.h"

#include <stdint.h>

#include "shape_b200.h"
#include "shape_b200_dropin_common.h"

#ifndef SHAPE_B200_CALC_FITS
#define SHAPE_B200_CALC_FITS calc_fits
#endif
#ifndef SHAPE_B200_CALC_FITS_CHI2
#define SHAPE_B200_CALC_FITS_CHI2 calc_fits_chi2_b200
#endif

static shape_engine *g_eng = NULL;
static uint64_t g_fingerprint = 0;
static int g_form = SHAPE_FORM_BATCHED_FP64;
static int g_keep_pos = 0;

/* ------------------------------------------------------------ fingerprint */

static uint64_t fnv(uint64_t h, const void *p, size_t n)
{
    const unsigned char *b = (const unsigned char *)p;
    for (size_t k = 0; k < n; k++) {
        h ^= b[k];
        h *= 1099511628211ULL;
    }
    return h;
}
#define FNV(h, x) ((h) = fnv((h), &(x), sizeof(x)))

/* Everything the engine was built from except the free shape parameters. */
static uint64_t b200_fingerprint(const struct par_t *par, const struct mod_t *mod,
                                 const struct dat_t *dat)
{
    uint64_t h = 1469598103934665603ULL;
    const void *pm = mod, *pd = dat;
    FNV(h, pm); FNV(h, pd);
    FNV(h, par->pos_smooth); FNV(h, par->nsinc2); FNV(h, par->sinc2width);
    FNV(h, par->mask_tol); FNV(h, par->mincosine_seen); FNV(h, par->exclude_seen);
    FNV(h, par->bad_objfactor); FNV(h, par->action); FNV(h, par->speckle);
    FNV(h, mod->shape.ncomp);
    const struct photo_t *ph = &mod->photo;
    for (int k = 0; k < ph->nradlaws; k++) {
        FNV(h, ph->radtype[k]);
        h = fnv(h, &ph->radar[k], sizeof(union radscat_t));
    }
    for (int k = 0; k < ph->noptlaws; k++) {
        FNV(h, ph->opttype[k]);
        h = fnv(h, &ph->optical[k], sizeof(union optscat_t));
    }
    FNV(h, dat->nsets);
    for (int s = 0; s < dat->nsets; s++) {
        const struct set_t *set = &dat->set[s];
        FNV(h, set->type);
        if (set->type == DELAY) {
            const struct deldop_t *dd = &set->desc.deldop;
            FNV(h, dd->nframes); FNV(h, dd->nviews); FNV(h, dd->iradlaw);
            FNV(h, dd->del_per_pixel); FNV(h, dd->dop_per_pixel); FNV(h, dd->Ftx);
            FNV(h, dd->dopscale.val); FNV(h, dd->codemethod); FNV(h, dd->spb);
            FNV(h, dd->stride); FNV(h, dd->dopfftlen);
            for (int f = 0; f < dd->nframes; f++) {
                const struct deldopfrm_t *fr = &dd->frame[f];
                FNV(h, fr->ndel); FNV(h, fr->ndop); FNV(h, fr->pos.n);
                FNV(h, fr->pos.km_per_pixel); FNV(h, fr->weight); FNV(h, fr->dof);
                FNV(h, fr->cal.state);
                if (fr->cal.state != 'f') FNV(h, fr->cal.val);
                FNV(h, fr->delcom_vig); FNV(h, fr->dopcom_vig); FNV(h, fr->dopDC_vig);
                const void *po = fr->obs, *pv = fr->oneovervar;
                FNV(h, po); FNV(h, pv);
                const struct deldopview_t *v = &fr->view[dd->v0];
                FNV(h, v->ae); FNV(h, v->oe); FNV(h, v->spin); FNV(h, v->deloff); FNV(h, v->dopoff);
            }
        } else if (set->type == DOPPLER) {
            const struct doppler_t *dp = &set->desc.doppler;
            FNV(h, dp->nframes); FNV(h, dp->nviews); FNV(h, dp->iradlaw);
            FNV(h, dp->dop_per_bin); FNV(h, dp->Ftx); FNV(h, dp->dopscale.val);
            for (int f = 0; f < dp->nframes; f++) {
                const struct dopfrm_t *fr = &dp->frame[f];
                FNV(h, fr->ndop); FNV(h, fr->pos.n); FNV(h, fr->pos.km_per_pixel);
                FNV(h, fr->weight); FNV(h, fr->dof); FNV(h, fr->sdev); FNV(h, fr->cal.state);
                if (fr->cal.state != 'f') FNV(h, fr->cal.val);
                FNV(h, fr->dopcom_vig);
                const void *po = fr->obs, *pv = fr->oneovervar;
                FNV(h, po); FNV(h, pv);
                const struct dopview_t *v = &fr->view[dp->v0];
                FNV(h, v->ae); FNV(h, v->oe); FNV(h, v->spin); FNV(h, v->dopoff);
            }
        } else if (set->type == POS) {
            const struct poset_t *po = &set->desc.poset;
            FNV(h, po->nframes); FNV(h, po->nviews); FNV(h, po->ioptlaw);
            FNV(h, par->poset_resample); FNV(h, par->image_rebin);
            for (int f = 0; f < po->nframes; f++) {
                const struct posetfrm_t *fr = &po->frame[f];
                const struct posetview_t *v = &fr->view[po->v0];
                FNV(h, fr->ncol); FNV(h, fr->nrow); FNV(h, fr->pos.n); FNV(h, fr->pos.km_per_pixel);
                FNV(h, fr->fit.km_per_pixel); FNV(h, fr->colcom_vig); FNV(h, fr->rowcom_vig);
                FNV(h, fr->off[0].val); FNV(h, fr->off[1].val); FNV(h, fr->northangle);
                FNV(h, fr->weight); FNV(h, fr->dof);
                const void *po_ = fr->obs.b, *pv = fr->oneovervar;
                FNV(h, po_); FNV(h, pv);
                FNV(h, v->ae); FNV(h, v->oe); FNV(h, v->se); FNV(h, v->solar_phase);
            }
        } else if (set->type == LGHTCRV) {
            const struct lghtcrv_t *lc = &set->desc.lghtcrv;
            FNV(h, lc->n); FNV(h, lc->ncalc); FNV(h, lc->nviews); FNV(h, lc->ioptlaw);
            FNV(h, lc->weight); FNV(h, lc->dof); FNV(h, lc->cal.state);
            if (lc->cal.state != 'f') FNV(h, lc->cal.val);
            const void *po = lc->obs, *pv = lc->oneovervar;
            FNV(h, po); FNV(h, pv);
            for (int i = 1; i <= lc->n; i++) FNV(h, lc->t[i][lc->v0]);
            for (int i = 1; i <= lc->ncalc; i++) {
                const struct crvrend_t *r = &lc->rend[i];
                FNV(h, lc->x[i]); FNV(h, lc->solar_phase[i]);
                FNV(h, r->pos.n); FNV(h, r->pos.km_per_pixel);
                FNV(h, r->ae); FNV(h, r->oe); FNV(h, r->se);
            }
        }
    }
    return h;
}

static void b200_build(struct par_t *par, struct mod_t *mod, struct dat_t *dat)
{
    if (mod->shape.ncomp != 1 || mod->shape.comp[0].type != VERTEX)
        b200_unsupported("model must be a single VERTEX component");
    if (par->dd_gamma != 1.0) b200_unsupported("dd_gamma != 1");
    if (par->exclude_seen >= 0 && par->exclude_seen < dat->nsets)
        b200_unsupported("exclude_seen names a dataset");
    if (par->speckle) b200_unsupported("speckle noise in the Doppler overflow variance");
    const char *fs = getenv("SHAPE_B200_FORM");
    g_form = SHAPE_FORM_BATCHED_FP64;
    if (fs && !strcmp(fs, "plain_fp64")) g_form = SHAPE_FORM_PLAIN_FP64;
    if (fs && !strcmp(fs, "batched_fp32")) g_form = SHAPE_FORM_BATCHED_FP32;
    const char *ds = getenv("SHAPE_B200_DEVICE");
    int device = ds ? atoi(ds) : 0;

    if (g_eng) shape_engine_destroy(g_eng);
    g_eng = NULL;
    b200_check(shape_engine_create(device, &g_eng), "engine_create");

    struct comp_t *c = &mod->shape.comp[0];
    struct vertices_t *real = &c->real;
    int nv = real->nv, nf = real->nf;
    double *a = malloc(sizeof(double) * 3 * nv), *u = malloc(sizeof(double) * 3 * nv);
    double *r = malloc(sizeof(double) * nv);
    int *fv = malloc(sizeof(int) * 3 * nf), *afp = malloc(sizeof(int) * (nv + 1));
    int naf = 0;
    for (int i = 0; i < nv; i++) naf += real->v[i].naf;
    int *afi = malloc(sizeof(int) * (naf > 0 ? naf : 1));
    afp[0] = 0;
    for (int i = 0; i < nv; i++) {
        for (int j = 0; j < 3; j++) { a[3 * i + j] = real->v[i].a[j]; u[3 * i + j] = real->v[i].u[j]; }
        r[i] = real->v[i].r.val;
        for (int k = 0; k < real->v[i].naf; k++) afi[afp[i] + k] = real->v[i].af[k];
        afp[i + 1] = afp[i] + real->v[i].naf;
    }
    for (int f = 0; f < nf; f++)
        for (int j = 0; j < 3; j++) fv[3 * f + j] = real->f[f].v[j];
    shape_model_desc m;
    memset(&m, 0, sizeof m);
    m.nv = nv; m.nf = nf; m.a = a; m.u = u; m.r = r; m.fv = fv; m.af_ptr = afp; m.af_idx = afi;
    for (int j = 0; j < 3; j++) m.scale[j] = c->desc.ver.scalefactor[j].val;
    b200_check(shape_engine_set_model(g_eng, &m), "set_model");
    free(a); free(u); free(r); free(fv); free(afp); free(afi);

    shape_eval_params ep;
    memset(&ep, 0, sizeof ep);
    ep.pos_smooth = par->pos_smooth;
    ep.nsinc2 = par->nsinc2;
    ep.sinc2width = par->sinc2width;
    ep.mask_tol = par->mask_tol;
    ep.mincosine_seen = par->mincosine_seen;
    ep.mark_seen = 1;
    b200_check(shape_engine_set_params(g_eng, &ep), "set_params");

    for (int s = 0; s < dat->nsets; s++) {
        struct set_t *set = &dat->set[s];
        if (set->type == DELAY) {
            struct deldop_t *dd = &set->desc.deldop;
            if (dd->nviews != 1) b200_unsupported("delay-Doppler smearing (nviews > 1)");
            shape_deldop_set S;
            memset(&S, 0, sizeof S);
            S.del_per_pixel = dd->del_per_pixel; S.dop_per_pixel = dd->dop_per_pixel;
            S.Ftx = dd->Ftx; S.dopscale = dd->dopscale.val; S.codemethod = dd->codemethod;
            S.spb = dd->spb; S.stride = dd->stride; S.dopfftlen = dd->dopfftlen;
            S.law = radar_law_of(&mod->photo, dd->iradlaw);
            shape_deldop_frame *F = calloc((size_t)dd->nframes, sizeof *F);
            size_t total = 0;
            for (int f = 0; f < dd->nframes; f++) total += (size_t)dd->frame[f].ndel * dd->frame[f].ndop;
            double *obs = malloc(sizeof(double) * (total ? total : 1));
            double *oov = malloc(sizeof(double) * (total ? total : 1));
            size_t off = 0;
            for (int f = 0; f < dd->nframes; f++) {
                struct deldopfrm_t *fr = &dd->frame[f];
                struct deldopview_t *v = &fr->view[dd->v0];
                shape_deldop_frame *G = &F[f];
                G->pos_n = fr->pos.n; G->km_per_pixel = fr->pos.km_per_pixel;
                rm9(G->ae, v->ae); rm9(G->oe, v->oe);
                for (int j = 0; j < 3; j++) G->spin[j] = v->spin[j];
                G->deloff = v->deloff; G->dopoff = v->dopoff;
                G->ndel = fr->ndel; G->ndop = fr->ndop;
                G->delcom_vig = fr->delcom_vig; G->dopcom_vig = fr->dopcom_vig;
                G->dopDC_vig = fr->dopDC_vig;
                G->weight = fr->weight; G->dof = fr->dof;
                G->cal_floating = (fr->cal.state == 'f');
                G->cal = fr->cal.val;
                for (int i = 1; i <= fr->ndel; i++)
                    for (int j = 1; j <= fr->ndop; j++, off++) {
                        obs[off] = fr->obs[i][j];
                        oov[off] = fr->oneovervar[i][j];
                    }
            }
            int rc = shape_engine_add_deldop_set(g_eng, &S, dd->nframes, F, obs, oov);
            free(F); free(obs); free(oov);
            b200_check(rc, "add_deldop_set");
        } else if (set->type == DOPPLER) {
            struct doppler_t *dp = &set->desc.doppler;
            if (dp->nviews != 1) b200_unsupported("Doppler smearing (nviews > 1)");
            shape_doppler_set S;
            memset(&S, 0, sizeof S);
            S.dop_per_bin = dp->dop_per_bin; S.Ftx = dp->Ftx; S.dopscale = dp->dopscale.val;
            S.law = radar_law_of(&mod->photo, dp->iradlaw);
            shape_doppler_frame *F = calloc((size_t)dp->nframes, sizeof *F);
            size_t total = 0;
            for (int f = 0; f < dp->nframes; f++) total += (size_t)dp->frame[f].ndop;
            double *obs = malloc(sizeof(double) * (total ? total : 1));
            double *oov = malloc(sizeof(double) * (total ? total : 1));
            size_t off = 0;
            for (int f = 0; f < dp->nframes; f++) {
                struct dopfrm_t *fr = &dp->frame[f];
                struct dopview_t *v = &fr->view[dp->v0];
                shape_doppler_frame *G = &F[f];
                G->pos_n = fr->pos.n; G->km_per_pixel = fr->pos.km_per_pixel;
                rm9(G->ae, v->ae); rm9(G->oe, v->oe);
                for (int j = 0; j < 3; j++) G->spin[j] = v->spin[j];
                G->dopoff = v->dopoff;
                G->ndop = fr->ndop; G->dopcom_vig = fr->dopcom_vig;
                G->weight = fr->weight; G->dof = fr->dof;
                G->cal_floating = (fr->cal.state == 'f'); G->cal = fr->cal.val;
                G->sdev = fr->sdev;
                for (int j = 1; j <= fr->ndop; j++, off++) {
                    obs[off] = fr->obs[j];
                    oov[off] = fr->oneovervar[j];
                }
            }
            int rc = shape_engine_add_doppler_set(g_eng, &S, dp->nframes, F, obs, oov);
            free(F); free(obs); free(oov);
            b200_check(rc, "add_doppler_set");
        } else if (set->type == LGHTCRV) {
            struct lghtcrv_t *lc = &set->desc.lghtcrv;
            if (lc->nviews != 1) b200_unsupported("lightcurve smearing (nviews > 1)");
            shape_lghtcrv_set L;
            memset(&L, 0, sizeof L);
            double *x = malloc(sizeof(double) * lc->ncalc), *t = malloc(sizeof(double) * lc->n);
            double *obs = malloc(sizeof(double) * lc->n), *oov = malloc(sizeof(double) * lc->n);
            for (int i = 1; i <= lc->ncalc; i++) x[i - 1] = lc->x[i];
            for (int i = 1; i <= lc->n; i++) {
                t[i - 1] = lc->t[i][lc->v0];
                obs[i - 1] = lc->obs[i];
                oov[i - 1] = lc->oneovervar[i];
            }
            L.ncalc = lc->ncalc; L.n = lc->n; L.x = x; L.t = t; L.obs = obs; L.oneovervar = oov;
            L.weight = lc->weight; L.dof = lc->dof;
            L.cal_floating = (lc->cal.state == 'f'); L.cal = lc->cal.val;
            L.law = optical_law_of(&mod->photo, lc->ioptlaw);
            shape_lghtcrv_point *P = calloc((size_t)lc->ncalc, sizeof *P);
            for (int i = 1; i <= lc->ncalc; i++) {
                struct crvrend_t *rd = &lc->rend[i];
                P[i - 1].pos_n = rd->pos.n;
                P[i - 1].km_per_pixel = rd->pos.km_per_pixel;
                rm9(P[i - 1].ae, rd->ae); rm9(P[i - 1].oe, rd->oe); rm9(P[i - 1].se, rd->se);
                P[i - 1].solar_phase = lc->solar_phase[i];
            }
            int rc = shape_engine_add_lghtcrv_set(g_eng, &L, P);
            free(x); free(t); free(obs); free(oov); free(P);
            b200_check(rc, "add_lghtcrv_set");
        } else if (set->type == POS) {
            struct poset_t *po = &set->desc.poset;
            if (po->nviews != 1) b200_unsupported("plane-of-sky smearing (nviews > 1)");
            shape_poset_set PS;
            memset(&PS, 0, sizeof PS);
            PS.law = optical_law_of(&mod->photo, po->ioptlaw);
            PS.resample = par->poset_resample;
            PS.rebin = par->image_rebin;
            shape_poset_frame *F = calloc((size_t)po->nframes, sizeof *F);
            size_t total = 0;
            for (int f = 0; f < po->nframes; f++) total += (size_t)po->frame[f].ncol * po->frame[f].nrow;
            double *obs = malloc(sizeof(double) * total), *oov = malloc(sizeof(double) * total);
            size_t off = 0;
            for (int f = 0; f < po->nframes; f++) {
                struct posetfrm_t *fr = &po->frame[f];
                struct posetview_t *v = &fr->view[po->v0];
                shape_poset_frame *G = &F[f];
                G->pos_n = fr->pos.n; G->km_per_pixel = fr->pos.km_per_pixel;
                rm9(G->ae, v->ae); rm9(G->oe, v->oe); rm9(G->se, v->se);
                G->solar_phase = v->solar_phase;
                G->ncol = fr->ncol; G->nrow = fr->nrow; G->fit_km_per_pixel = fr->fit.km_per_pixel;
                G->colcom_vig = fr->colcom_vig; G->rowcom_vig = fr->rowcom_vig;
                G->xoff = fr->off[0].val; G->yoff = fr->off[1].val; G->northangle = fr->northangle;
                G->weight = fr->weight; G->dof = fr->dof;
                for (int i = 1; i <= fr->ncol; i++)
                    for (int j = 1; j <= fr->nrow; j++, off++) {
                        obs[off] = fr->obs.b[i][j];
                        oov[off] = fr->oneovervar[i][j];
                    }
            }
            int rc = shape_engine_add_poset_set(g_eng, &PS, po->nframes, F, obs, oov);
            free(F); free(obs); free(oov);
            b200_check(rc, "add_poset_set");
        } else {
            b200_unsupported("dataset type");
        }
    }
    g_keep_pos = (par->action == WRITE);
    b200_check(shape_engine_keep_pos(g_eng, g_keep_pos), "keep_pos");
    b200_check(shape_engine_finalize(g_eng), "finalize");
}

/* Builds or reuses the engine, pushes the free shape parameters, evaluates. */
static void b200_evaluate(struct par_t *par, struct mod_t *mod, struct dat_t *dat,
                          shape_eval_summary *sm)
{
    uint64_t fp = b200_fingerprint(par, mod, dat);
    if (!g_eng || fp != g_fingerprint) {
        b200_build(par, mod, dat);
        g_fingerprint = fp;
    }
    struct comp_t *c = &mod->shape.comp[0];
    for (int j = 0; j < 3; j++)
        b200_check(shape_engine_set_scale(g_eng, j, c->desc.ver.scalefactor[j].val), "set_scale");
    for (int i = 0; i < c->real.nv; i++)
        b200_check(shape_engine_set_vertex_r(g_eng, i, c->real.v[i].r.val), "set_vertex_r");
    b200_check(shape_engine_evaluate(g_eng, g_form, sm), "evaluate");

    /* flags of calc_fits (src/shape/calc_fits.c:349-354, 407-409) */
    par->posbnd = sm->posbnd;
    par->posbnd_logfactor = sm->posbnd_logfactor;
    par->badposet = sm->badposet;
    par->badposet_logfactor = sm->badposet_logfactor;
    par->badradar = sm->badradar;
    par->badradar_logfactor = sm->badradar_logfactor;

    /* facet "seen" flags */
    int nf = c->real.nf;
    unsigned char *seen = malloc((size_t)nf);
    b200_check(shape_engine_get_seen(g_eng, seen), "get_seen");
    for (int f = 0; f < nf; f++) c->real.f[f].seen = seen[f];
    free(seen);
}

/* Radar frames in the engine's order: delay-Doppler and Doppler sets in
 * dataset order. */
static int total_frames(const struct dat_t *dat)
{
    int n = 0;
    for (int s = 0; s < dat->nsets; s++) {
        if (dat->set[s].type == DELAY) n += dat->set[s].desc.deldop.nframes;
        if (dat->set[s].type == DOPPLER) n += dat->set[s].desc.doppler.nframes;
    }
    return n;
}

/* Per-frame limits, log-factor, cal and chi2 from the engine's results. */
/* Plane-of-sky frames: fit images and sky brightness written back, and
 * with_chi2: cal, frame and set chi-square (chi2_poset's side effects). */
static void copy_poset_results(struct dat_t *dat, int with_chi2)
{
    for (int s = 0; s < dat->nsets; s++) {
        if (dat->set[s].type != POS) continue;
        struct poset_t *po = &dat->set[s].desc.poset;
        double set_chi2 = 0.0;
        for (int f = 0; f < po->nframes; f++) {
            struct posetfrm_t *fr = &po->frame[f];
            const int n = fr->pos.n, side = 2 * n + 1;
            double *fit = malloc(sizeof(double) * (size_t)fr->ncol * fr->nrow);
            double *b = malloc(sizeof(double) * (size_t)side * side);
            shape_poset_result r;
            b200_check(shape_engine_get_poset(g_eng, s, f, fit, b, &r), "get_poset");
            size_t k = 0;
            for (int i = 1; i <= fr->ncol; i++)
                for (int j = 1; j <= fr->nrow; j++) fr->fit.b[i][j] = fit[k++];
            for (int i = -n; i <= n; i++)
                for (int j = -n; j <= n; j++) fr->pos.b[i][j] = b[(size_t)(i + n) * side + (size_t)(j + n)];
            free(fit); free(b);
            if (with_chi2) {
                fr->cal.val = r.cal;
                fr->chi2 = r.chi2;
                set_chi2 += r.chi2;
            }
        }
        if (with_chi2) dat->set[s].chi2 = set_chi2;
    }
}

static void copy_frame_results(struct dat_t *dat, int with_chi2)
{
    int nfr = total_frames(dat);
    if (nfr == 0) return;
    shape_deldop_result *R = malloc(sizeof *R * (size_t)nfr);
    double *O = malloc(sizeof(double) * 4 * (size_t)nfr);
    b200_check(shape_engine_get_deldop_results(g_eng, R, nfr), "get_deldop_results");
    b200_check(shape_engine_get_radar_overflow(g_eng, O, nfr), "get_radar_overflow");
    int g = 0;
    for (int s = 0; s < dat->nsets; s++) {
        if (dat->set[s].type == DOPPLER) {
            struct doppler_t *dp = &dat->set[s].desc.doppler;
            double set_chi2 = 0.0;
            for (int f = 0; f < dp->nframes; f++, g++) {
                struct dopfrm_t *fr = &dp->frame[f];
                const shape_deldop_result *q = &R[g];
                for (int k = 0; k < 2; k++) {
                    fr->pos.xlim[k] = q->xlim[k]; fr->pos.ylim[k] = q->ylim[k];
                    fr->idoplim[k] = q->idoplim[k]; fr->doplim[k] = q->doplim[k];
                }
                fr->badradar_logfactor = q->badradar_logfactor;
                fr->pos.posbnd_logfactor = q->posbnd_logfactor;
                fr->overflow_o2 = O[4 * g + 0];
                fr->overflow_m2 = O[4 * g + 1];
                fr->overflow_xsec = O[4 * g + 2];
                fr->overflow_dopmean = O[4 * g + 3];
                if (with_chi2) {
                    if (fr->cal.state == 'f') fr->cal.val = q->cal;
                    fr->chi2 = q->chi2;
                    set_chi2 += q->chi2;
                }
            }
            if (with_chi2) dat->set[s].chi2 = set_chi2;
            continue;
        }
        if (dat->set[s].type != DELAY) continue;
        struct deldop_t *dd = &dat->set[s].desc.deldop;
        double set_chi2 = 0.0;
        for (int f = 0; f < dd->nframes; f++, g++) {
            struct deldopfrm_t *fr = &dd->frame[f];
            const shape_deldop_result *q = &R[g];
            for (int k = 0; k < 2; k++) {
                fr->pos.xlim[k] = q->xlim[k]; fr->pos.ylim[k] = q->ylim[k];
                fr->idellim[k] = q->idellim[k]; fr->idoplim[k] = q->idoplim[k];
                fr->dellim[k] = q->dellim[k]; fr->doplim[k] = q->doplim[k];
            }
            fr->badradar_logfactor = q->badradar_logfactor;
            fr->pos.posbnd_logfactor = q->posbnd_logfactor;
            if (with_chi2) {
                if (fr->cal.state == 'f') fr->cal.val = q->cal;
                fr->chi2 = q->chi2;
                set_chi2 += q->chi2;
            }
        }
        if (with_chi2) dat->set[s].chi2 = set_chi2;
    }
    free(R);
    free(O);
}

void SHAPE_B200_CALC_FITS(struct par_t *par, struct mod_t *mod, struct dat_t *dat)
{
    shape_eval_summary sm;
    memset(&sm, 0, sizeof sm);
    b200_evaluate(par, mod, dat, &sm);
    copy_frame_results(dat, 0);
    copy_poset_results(dat, 0);
    size_t maxd = 1;
    for (int s = 0; s < dat->nsets; s++) {
        if (dat->set[s].type == DELAY)
            for (int f = 0; f < dat->set[s].desc.deldop.nframes; f++) {
                size_t D = (size_t)dat->set[s].desc.deldop.frame[f].ndel * dat->set[s].desc.deldop.frame[f].ndop;
                if (D > maxd) maxd = D;
            }
        if (dat->set[s].type == DOPPLER)
            for (int f = 0; f < dat->set[s].desc.doppler.nframes; f++)
                if ((size_t)dat->set[s].desc.doppler.frame[f].ndop > maxd)
                    maxd = (size_t)dat->set[s].desc.doppler.frame[f].ndop;
    }
    double *buf = malloc(sizeof(double) * maxd);
    int g = 0;
    for (int s = 0; s < dat->nsets; s++) {
        struct set_t *set = &dat->set[s];
        if (set->type == DELAY) {
            struct deldop_t *dd = &set->desc.deldop;
            for (int f = 0; f < dd->nframes; f++, g++) {
                struct deldopfrm_t *fr = &dd->frame[f];
                b200_check(shape_engine_get_fit(g_eng, g, buf), "get_fit");
                size_t k = 0;
                for (int i = 1; i <= fr->ndel; i++)
                    for (int j = 1; j <= fr->ndop; j++) fr->fit[i][j] = buf[k++];
                if (g_keep_pos) {
                    int n = fr->pos.n, side = 2 * n + 1;
                    size_t np = (size_t)side * side;
                    double *z = malloc(sizeof(double) * np), *ce = malloc(sizeof(double) * np);
                    int *fa = malloc(sizeof(int) * np);
                    b200_check(shape_engine_get_pos(g_eng, g, z, ce, fa), "get_pos");
                    for (int i = -n; i <= n; i++)
                        for (int j = -n; j <= n; j++) {
                            size_t p = (size_t)(i + n) * side + (size_t)(j + n);
                            fr->pos.z[i][j] = z[p]; fr->pos.cose[i][j] = ce[p]; fr->pos.f[i][j] = fa[p];
                        }
                    free(z); free(ce); free(fa);
                }
            }
        } else if (set->type == DOPPLER) {
            struct doppler_t *dp = &set->desc.doppler;
            for (int f = 0; f < dp->nframes; f++, g++) {
                struct dopfrm_t *fr = &dp->frame[f];
                b200_check(shape_engine_get_fit(g_eng, g, buf), "get_fit");
                for (int j = 1; j <= fr->ndop; j++) fr->fit[j] = buf[j - 1];
                if (g_keep_pos) {
                    int n = fr->pos.n, side = 2 * n + 1;
                    size_t np = (size_t)side * side;
                    double *z = malloc(sizeof(double) * np), *ce = malloc(sizeof(double) * np);
                    int *fa = malloc(sizeof(int) * np);
                    b200_check(shape_engine_get_pos(g_eng, g, z, ce, fa), "get_pos");
                    for (int i = -n; i <= n; i++)
                        for (int j = -n; j <= n; j++) {
                            size_t p = (size_t)(i + n) * side + (size_t)(j + n);
                            fr->pos.z[i][j] = z[p]; fr->pos.cose[i][j] = ce[p]; fr->pos.f[i][j] = fa[p];
                        }
                    free(z); free(ce); free(fa);
                }
            }
        } else if (set->type == LGHTCRV) {
            struct lghtcrv_t *lc = &set->desc.lghtcrv;
            double *y = malloc(sizeof(double) * lc->ncalc), *fit = malloc(sizeof(double) * lc->n);
            b200_check(shape_engine_get_lghtcrv(g_eng, s, y, fit, NULL, NULL), "get_lghtcrv");
            for (int i = 1; i <= lc->ncalc; i++) lc->y[i] = y[i - 1];
            for (int i = 1; i <= lc->n; i++) lc->fit[i] = fit[i - 1];
            free(y); free(fit);
        }
    }
    free(buf);
}

double SHAPE_B200_CALC_FITS_CHI2(struct par_t *par, struct mod_t *mod, struct dat_t *dat)
{
    shape_eval_summary sm;
    memset(&sm, 0, sizeof sm);
    b200_evaluate(par, mod, dat, &sm);
    copy_frame_results(dat, 1);
    copy_poset_results(dat, 1);
    for (int s = 0; s < dat->nsets; s++) {
        struct set_t *set = &dat->set[s];
        if (set->type != LGHTCRV) continue;
        double cal, chi2v;
        b200_check(shape_engine_get_lghtcrv(g_eng, s, NULL, NULL, &cal, &chi2v), "get_lghtcrv");
        if (set->desc.lghtcrv.cal.state == 'f') set->desc.lghtcrv.cal.val = cal;
        set->chi2 = chi2v;
    }
    dat->chi2 = sm.chi2;
    return sm.chi2;
}
