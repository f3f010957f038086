/*
 * Direct-call harness around the REFERENCE SHAPE CPU code (test
 * infrastructure only; compiled by oracle/build_ref.sh into
 * oracle/_ref/libshape_ref.so together with the reference sources, which are
 * compiled where they lie under the reference tree).
 *
 * It fills the reference's own structs (struct mod_t / dat_t / par_t,
 * src/shape/shape2.h) from the plain descriptions of include/shape_types.h
 * and calls the reference entry points unchanged:
 *   realize_mod (src/shape/realize_mod.c:153), calc_fits
 *   (src/shape/calc_fits.c:340), chi2 (src/shape/chi2.c:240), and the line
 *   searches mnbrak / brent_abs (src/nr/mnbrak.c, src/nr/brent_abs.c).
 * POS sizes are per frame (pos_scope LOCAL with a per-frame n), as in the
 * reference's set_up_pos (src/shape/read_dat.c:1303-1380), so frames of
 * different sizes can share one dataset.
 */
#include "head.h"

#include "shape_types.h"
#include "ref_session.h"

static void ref_alloc_pos(struct pos_t *pos, int n, double kmpp, int bistatic)
{
    memset(pos, 0, sizeof *pos);
    pos->n = n;
    pos->km_per_pixel = kmpp;
    pos->b = matrix(-n, n, -n, n);
    pos->cosi = matrix(-n, n, -n, n);
    pos->cose = matrix(-n, n, -n, n);
    pos->z = matrix(-n, n, -n, n);
    pos->body = imatrix(-n, n, -n, n);
    pos->comp = imatrix(-n, n, -n, n);
    pos->f = imatrix(-n, n, -n, n);
    pos->cosill = matrix(-n, n, -n, n);
    pos->zill = matrix(-n, n, -n, n);
    pos->bodyill = imatrix(-n, n, -n, n);
    pos->compill = imatrix(-n, n, -n, n);
    pos->fill = imatrix(-n, n, -n, n);
    pos->bistatic = bistatic;
    /* defined contents before any routine writes them: a drop-in that
     * writes only some maps leaves the others as the reference's posclr
     * sets them, not as malloc left them */
    posclr(pos);
}

static void ref_free_pos(struct pos_t *pos)
{
    int n = pos->n;
    if (!pos->b) return;
    free_matrix(pos->b, -n, n, -n, n); free_matrix(pos->cosi, -n, n, -n, n);
    free_matrix(pos->cose, -n, n, -n, n); free_matrix(pos->z, -n, n, -n, n);
    free_imatrix(pos->body, -n, n, -n, n); free_imatrix(pos->comp, -n, n, -n, n);
    free_imatrix(pos->f, -n, n, -n, n); free_matrix(pos->cosill, -n, n, -n, n);
    free_matrix(pos->zill, -n, n, -n, n); free_imatrix(pos->bodyill, -n, n, -n, n);
    free_imatrix(pos->compill, -n, n, -n, n); free_imatrix(pos->fill, -n, n, -n, n);
}

void *ref_new(const shape_model_desc *m, const shape_eval_params *ep, int max_sets)
{
    ref_session *S = calloc(1, sizeof *S);
    struct par_t *par = &S->par;
    struct mod_t *mod = &S->mod;
    par->action = FIT;
    par->pos_smooth = (unsigned char)ep->pos_smooth;
    par->nsinc2 = ep->nsinc2;
    par->sinc2width = ep->sinc2width;
    par->mask_tol = ep->mask_tol;
    par->mincosine_seen = ep->mincosine_seen;
    par->exclude_seen = ep->mark_seen ? -1 : -2;
    par->dd_gamma = 1.0;
    par->bad_objfactor = 2.0;
    par->warn_badradar = 0;
    par->pos_scope = LOCAL;

    /* one VERTEX component, or m->ncomp of them back to back (model-wide
     * facet and attached-facet indices turned into the component's own) */
    const int nc = m->ncomp > 1 ? m->ncomp : 1;
    mod->shape.ncomp = nc;
    mod->shape.comp = calloc((size_t)nc, sizeof(struct comp_t));
    int v0 = 0, f0 = 0;
    for (int k = 0; k < nc; k++) {
        const int nvk = nc > 1 ? m->comp_nv[k] : m->nv, nfk = nc > 1 ? m->comp_nf[k] : m->nf;
        struct comp_t *c = &mod->shape.comp[k];
        c->type = VERTEX;
        struct vertices_t *real = &c->real;
        real->nv = c->desc.ver.nv = nvk;
        real->nf = c->desc.ver.nf = nfk;
        real->v = calloc((size_t)nvk, sizeof(struct vertex_t));
        real->f = calloc((size_t)nfk, sizeof(struct facet_t));
        for (int j = 0; j < 3; j++) {
            c->desc.ver.scalefactor[j].state = 'f';
            c->desc.ver.scalefactor[j].val = nc > 1 ? m->comp_scale[3 * k + j] : m->scale[j];
            real->scalefactor[j] = c->desc.ver.scalefactor[j];
            c->off[j].state = c->rot[j].state = 'c';
            c->off[j].val = nc > 1 ? m->comp_off[3 * k + j] : 0.0;
            c->rot[j].val = nc > 1 ? m->comp_rot[3 * k + j] : 0.0;
        }
        for (int i = 0; i < nvk; i++) {
            const int g = v0 + i;
            struct vertex_t *v = &real->v[i];
            for (int j = 0; j < 3; j++) { v->a[j] = m->a[3 * g + j]; v->u[j] = m->u[3 * g + j]; }
            v->r.state = 'f';
            v->r.val = m->r[g];
            v->naf = m->af_ptr[g + 1] - m->af_ptr[g];
            v->af = malloc(sizeof(int) * (size_t)(v->naf > 0 ? v->naf : 1));
            for (int q = 0; q < v->naf; q++) v->af[q] = m->af_idx[m->af_ptr[g] + q] - f0;
            v->act = 1;
            v->v_mirror = i;
        }
        for (int f = 0; f < nfk; f++) {
            for (int j = 0; j < 3; j++) real->f[f].v[j] = m->fv[3 * (f0 + f) + j] - v0;
            real->f[f].act = 1;
        }
        /* the vertex description shares the realization's arrays (VERTEX
         * type is its own realization, src/shape/realize_mod.c:455-458) */
        c->desc.ver.v = real->v;
        c->desc.ver.f = real->f;
        v0 += nvk;
        f0 += nfk;
    }

    S->dat.set = calloc((size_t)max_sets, sizeof(struct set_t));
    S->nsets_cap = max_sets;
    return S;
}

void ref_set_radar_law(void *h, const shape_radar_law *L)
{
    ref_session *S = h;
    struct photo_t *ph = &S->mod.photo;
    ph->nradlaws = 1;
    ph->radtype = calloc(1, 1);
    ph->radar = calloc(1, sizeof(union radscat_t));
    ph->radtype[0] = (unsigned char)L->type;
    switch (L->type) {
    case COSINELAW_DIFF:
        ph->radar[0].RC.R.val = L->diff_R; ph->radar[0].RC.C.val = L->diff_C; break;
    case GAUSSIANLAW: case HAGFORSLAW: case COSINELAW_QS:
        ph->radar[0].quasispec.R.val = L->qs_R; ph->radar[0].quasispec.C.val = L->qs_C;
        ph->radar[0].quasispec.cos_cutoff = L->qs_cos_cutoff; break;
    default:
        ph->radar[0].hybrid.diff.R.val = L->diff_R; ph->radar[0].hybrid.diff.C.val = L->diff_C;
        ph->radar[0].hybrid.qs.R.val = L->qs_R; ph->radar[0].hybrid.qs.C.val = L->qs_C;
        ph->radar[0].hybrid.qs.cos_cutoff = L->qs_cos_cutoff; break;
    }
}

void ref_set_optical_law(void *h, const shape_optical_law *L)
{
    ref_session *S = h;
    struct photo_t *ph = &S->mod.photo;
    ph->noptlaws = 1;
    ph->opttype = calloc(1, 1);
    ph->optical = calloc(1, sizeof(union optscat_t));
    ph->opttype[0] = (unsigned char)L->type;
    if (L->type == KAASALAINEN) {
        ph->optical[0].kaas.R.val = L->R; ph->optical[0].kaas.wt.val = L->wt;
        ph->optical[0].kaas.A0.val = L->A0; ph->optical[0].kaas.D.val = L->D;
        ph->optical[0].kaas.k.val = L->k;
    } else {
        ph->optical[0].R.R.val = L->R;
    }
}

static void ref_copy_rm(double out[3][3], const double *in)
{
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) out[i][j] = in[3 * i + j];
}

/* A delay-Doppler set with nviews views per frame (smearing): views[f *
 * nviews + k] is frame f's k-th view in rendering order, which calc_fits
 * walks as v = (v0 + 1 + k) % nviews (src/shape/calc_fits.c:489-490), so it
 * is stored at the reference's view index v; the frame-level fields come from
 * the last (epoch) view, index v0. */
int ref_add_deldop_set_views(void *h, const shape_deldop_set *ds, int nframes, int nviews, int v0,
                             const shape_deldop_frame *views, const double *obs_all,
                             const double *oov_all)
{
    ref_session *S = h;
    if (S->dat.nsets >= S->nsets_cap) return -1;
    struct set_t *set = &S->dat.set[S->dat.nsets++];
    set->type = DELAY;
    struct deldop_t *dd = &set->desc.deldop;
    dd->iradlaw = 0;
    dd->del_per_pixel = ds->del_per_pixel;
    dd->dop_per_pixel = ds->dop_per_pixel;
    dd->Ftx = ds->Ftx;
    dd->dopscale.val = ds->dopscale;
    dd->codemethod = ds->codemethod;
    dd->spb = ds->spb;
    dd->stride = ds->stride;
    dd->dopfftlen = ds->dopfftlen;
    if (nviews < 1 || v0 < 0 || v0 >= nviews) return -1;
    dd->nviews = nviews;
    dd->v0 = v0;
    dd->nframes = nframes;
    dd->frame = calloc((size_t)nframes, sizeof(struct deldopfrm_t));
    size_t off = 0;
    double dof = 0.0;
    for (int f = 0; f < nframes; f++) {
        const shape_deldop_frame *F = &views[(size_t)f * nviews + nviews - 1];
        struct deldopfrm_t *fr = &dd->frame[f];
        fr->ndel = F->ndel; fr->ndop = F->ndop;
        fr->delcom_vig = F->delcom_vig; fr->dopcom_vig = F->dopcom_vig;
        fr->dopDC_vig = F->dopDC_vig;
        fr->weight = F->weight; fr->dof = F->dof;
        fr->cal.state = F->cal_floating ? 'f' : 'c';
        fr->cal.val = F->cal;
        fr->sdev = 1.0;
        fr->obs = matrix(1, F->ndel, 1, F->ndop);
        fr->fit = matrix(1, F->ndel, 1, F->ndop);
        fr->oneovervar = matrix(1, F->ndel, 1, F->ndop);
        for (int i = 1; i <= F->ndel; i++)
            for (int j = 1; j <= F->ndop; j++) {
                size_t p = off + (size_t)(i - 1) * F->ndop + (size_t)(j - 1);
                fr->obs[i][j] = obs_all[p];
                fr->oneovervar[i][j] = oov_all[p];
                fr->fit[i][j] = 0.0;
            }
        off += (size_t)F->ndel * F->ndop;
        fr->view = calloc((size_t)nviews, sizeof(struct deldopview_t));
        for (int k = 0; k < nviews; k++) {
            const shape_deldop_frame *V = &views[(size_t)f * nviews + k];
            struct deldopview_t *w = &fr->view[(v0 + 1 + k) % nviews];
            ref_copy_rm(w->ae, V->ae);
            ref_copy_rm(w->oe, V->oe);
            for (int j = 0; j < 3; j++) w->spin[j] = V->spin[j];
            w->deloff = V->deloff;
            w->dopoff = V->dopoff;
        }
        ref_alloc_pos(&fr->pos, F->pos_n, F->km_per_pixel, 0);
        dof += F->dof;
    }
    dd->dof = dof;
    set->dof = dof;
    S->dat.dof_deldop += dof;
    S->dat.dof += dof;
    return S->dat.nsets - 1;
}

int ref_add_deldop_set(void *h, const shape_deldop_set *ds, int nframes,
                       const shape_deldop_frame *frames, const double *obs_all,
                       const double *oov_all)
{
    return ref_add_deldop_set_views(h, ds, nframes, 1, 0, frames, obs_all, oov_all);
}

/* A Doppler set (struct doppler_t, src/shape/shape2.h:1266-1287) with one
 * view per frame; obs_all / oov_all hold every frame's ndop bins back to back. */
int ref_add_doppler_set(void *h, const shape_doppler_set *ds, int nframes,
                        const shape_doppler_frame *frames, const double *obs_all,
                        const double *oov_all)
{
    ref_session *S = h;
    if (S->dat.nsets >= S->nsets_cap) return -1;
    struct set_t *set = &S->dat.set[S->dat.nsets++];
    set->type = DOPPLER;
    struct doppler_t *dp = &set->desc.doppler;
    dp->iradlaw = 0;
    dp->dop_per_bin = ds->dop_per_bin;
    dp->Ftx = ds->Ftx;
    dp->dopscale.val = ds->dopscale;
    dp->nviews = 1;
    dp->v0 = 0;
    dp->nframes = nframes;
    dp->frame = calloc((size_t)nframes, sizeof(struct dopfrm_t));
    size_t off = 0;
    double dof = 0.0;
    for (int f = 0; f < nframes; f++) {
        const shape_doppler_frame *F = &frames[f];
        struct dopfrm_t *fr = &dp->frame[f];
        fr->ndop = F->ndop;
        fr->dopcom_vig = F->dopcom_vig;
        fr->weight = F->weight;
        fr->dof = F->dof;
        fr->sdev = F->sdev;
        fr->cal.state = F->cal_floating ? 'f' : 'c';
        fr->cal.val = F->cal;
        fr->obs = vector(1, F->ndop);
        fr->fit = vector(1, F->ndop);
        fr->oneovervar = vector(1, F->ndop);
        for (int j = 1; j <= F->ndop; j++) {
            fr->obs[j] = obs_all[off + (size_t)(j - 1)];
            fr->oneovervar[j] = oov_all[off + (size_t)(j - 1)];
            fr->fit[j] = 0.0;
        }
        off += (size_t)F->ndop;
        fr->view = calloc(1, sizeof(struct dopview_t));
        ref_copy_rm(fr->view[0].ae, F->ae);
        ref_copy_rm(fr->view[0].oe, F->oe);
        for (int j = 0; j < 3; j++) fr->view[0].spin[j] = F->spin[j];
        fr->view[0].dopoff = F->dopoff;
        ref_alloc_pos(&fr->pos, F->pos_n, F->km_per_pixel, 0);
        dof += F->dof;
    }
    dp->dof = dof;
    set->dof = dof;
    S->dat.dof_doppler += dof;
    S->dat.dof += dof;
    return S->dat.nsets - 1;
}

int ref_add_lghtcrv_set(void *h, const shape_lghtcrv_set *ls, const shape_lghtcrv_point *pts)
{
    ref_session *S = h;
    if (S->dat.nsets >= S->nsets_cap) return -1;
    struct set_t *set = &S->dat.set[S->dat.nsets++];
    set->type = LGHTCRV;
    struct lghtcrv_t *lc = &set->desc.lghtcrv;
    int n = ls->n, ncalc = ls->ncalc;
    lc->ioptlaw = 0;
    lc->nviews = 1;
    lc->v0 = 0;
    lc->n = n;
    lc->ncalc = ncalc;
    lc->weight = ls->weight;
    lc->dof = ls->dof;
    lc->cal.state = ls->cal_floating ? 'f' : 'c';
    lc->cal.val = ls->cal;
    lc->t0 = vector(1, n);
    lc->t = matrix(1, n, 0, 0);
    lc->obs = vector(1, n);
    lc->oneovervar = vector(1, n);
    lc->fit = vector(1, n);
    lc->rotphase_calc = vector(1, ncalc);
    lc->rotphase_obs = vector(1, n);
    lc->x0 = vector(1, ncalc);
    lc->x = vector(1, ncalc);
    lc->y = vector(1, ncalc);
    lc->y2 = vector(1, ncalc);
    lc->solar_phase = vector(1, ncalc);
    lc->solar_azimuth = vector(1, ncalc);
    lc->rend = calloc((size_t)ncalc + 1, sizeof(struct crvrend_t));
    for (int i = 1; i <= n; i++) {
        lc->t0[i] = lc->t[i][0] = ls->t[i - 1];
        lc->obs[i] = ls->obs[i - 1];
        lc->oneovervar[i] = ls->oneovervar[i - 1];
        lc->fit[i] = 0.0;
    }
    for (int i = 1; i <= ncalc; i++) {
        const shape_lghtcrv_point *P = &pts[i - 1];
        lc->x0[i] = lc->x[i] = ls->x[i - 1];
        lc->y[i] = lc->y2[i] = 0.0;
        lc->solar_phase[i] = P->solar_phase;
        ref_copy_rm(lc->rend[i].ae, P->ae);
        ref_copy_rm(lc->rend[i].oe, P->oe);
        ref_copy_rm(lc->rend[i].se, P->se);
        ref_alloc_pos(&lc->rend[i].pos, P->pos_n, P->km_per_pixel, 1);
    }
    set->dof = ls->dof;
    S->dat.dof_lghtcrv += ls->dof;
    S->dat.dof += ls->dof;
    return S->dat.nsets - 1;
}

/* A plane-of-sky set (struct poset_t, src/shape/shape2.h:1290-1341) with one
 * view per frame, as read_poset and set_up_pos leave it: the sky rendering
 * (bistatic POS window), the observed and fit images [1..ncol][1..nrow],
 * 1/variance, COM offsets, north angle and the floating calibration; the
 * set's resampling mode and rebinning go to par (poset_resample,
 * image_rebin), its law is optical law 0. Returns the set index. */
int ref_add_poset_set(void *h, const shape_poset_set *ps, int nframes, const shape_poset_frame *frames,
                      const double *obs, const double *oov)
{
    ref_session *S = h;
    if (S->dat.nsets >= S->nsets_cap) return -1;
    struct set_t *set = &S->dat.set[S->dat.nsets++];
    set->type = POS;
    struct poset_t *po = &set->desc.poset;
    po->ioptlaw = 0;
    po->nviews = 1;
    po->v0 = 0;
    po->nframes = nframes;
    po->frame = calloc((size_t)nframes, sizeof(struct posetfrm_t));
    S->par.poset_resample = (unsigned char)ps->resample;
    S->par.image_rebin = (unsigned char)ps->rebin;
    size_t off = 0;
    double dof = 0.0;
    for (int f = 0; f < nframes; f++) {
        const shape_poset_frame *F = &frames[f];
        struct posetfrm_t *fr = &po->frame[f];
        fr->view = calloc(1, sizeof(struct posetview_t));
        ref_copy_rm(fr->view[0].ae, F->ae);
        ref_copy_rm(fr->view[0].oe, F->oe);
        ref_copy_rm(fr->view[0].se, F->se);
        fr->view[0].solar_phase = F->solar_phase;
        fr->ncol = F->ncol;
        fr->nrow = F->nrow;
        fr->colcom_vig = F->colcom_vig;
        fr->rowcom_vig = F->rowcom_vig;
        fr->off[0].state = fr->off[1].state = 'c';
        fr->off[0].val = F->xoff;
        fr->off[1].val = F->yoff;
        fr->northangle = F->northangle;
        fr->weight = F->weight;
        fr->dof = F->dof;
        fr->cal.state = 'f';
        fr->cal.val = 1.0;
        ref_alloc_pos(&fr->pos, F->pos_n, F->km_per_pixel, 1);
        fr->obs.b = matrix(1, F->ncol, 1, F->nrow);
        fr->fit.b = matrix(1, F->ncol, 1, F->nrow);
        fr->oneovervar = matrix(1, F->ncol, 1, F->nrow);
        fr->fit.km_per_pixel = F->fit_km_per_pixel;
        fr->obs.km_per_pixel = F->fit_km_per_pixel;
        for (int i = 1; i <= F->ncol; i++)
            for (int j = 1; j <= F->nrow; j++, off++) {
                fr->obs.b[i][j] = obs[off];
                fr->oneovervar[i][j] = oov[off];
                fr->fit.b[i][j] = 0.0;
            }
        dof += F->dof;
    }
    po->dof = dof;
    set->dof = dof;
    S->dat.dof_poset += dof;
    S->dat.dof += dof;
    return S->dat.nsets - 1;
}

/* A plane-of-sky frame after calc_fits + chi2: the fit image (layout of
 * the observed one), the sky rendering's brightness pos->b ((2n+1)^2, j
 * contiguous), cal and chi2 (out[0..1]); NULL skips. */
void ref_get_poset_frame(void *h, int s, int f, double *fit, double *b, double *out)
{
    ref_session *S = h;
    struct posetfrm_t *fr = &S->dat.set[s].desc.poset.frame[f];
    if (fit)
        for (int i = 1; i <= fr->ncol; i++)
            for (int j = 1; j <= fr->nrow; j++) fit[(size_t)(i - 1) * fr->nrow + (j - 1)] = fr->fit.b[i][j];
    if (b) {
        const int n = fr->pos.n, side = 2 * n + 1;
        for (int i = -n; i <= n; i++)
            for (int j = -n; j <= n; j++) b[(size_t)(i + n) * side + (j + n)] = fr->pos.b[i][j];
    }
    if (out) { out[0] = fr->cal.val; out[1] = fr->chi2; }
}

/* par's badposet flag and log factor after calc_fits (src/shape/calc_fits.c:408). */
void ref_get_badposet(void *h, double out[2])
{
    ref_session *S = h;
    out[0] = S->par.badposet;
    out[1] = S->par.badposet_logfactor;
}

/* Scale factor j of the component (a SIZEPAR free parameter, src/shape/mkparlist.c:219-226). */
void ref_set_scale(void *h, int j, double val)
{
    ref_session *S = h;
    S->mod.shape.comp[j / 3].desc.ver.scalefactor[j % 3].val = val;
}

/* Vertex deviation r of vertex i (a SHAPEPAR free parameter, src/shape/mkparlist.c:227-233). */
void ref_set_r(void *h, int i, double val)
{
    ref_session *S = h;
    int c = 0;
    while (i >= S->mod.shape.comp[c].real.nv) i -= S->mod.shape.comp[c++].real.nv;
    S->mod.shape.comp[c].real.v[i].r.val = val;
}

void ref_realize(void *h)
{
    ref_session *S = h;
    realize_mod(&S->par, &S->mod);
}

/* realize_mod + calc_fits + chi2(par, dat, 0): the evaluation inside
 * objective() (src/shape/bestfit.c:748-790) without penalties. Returns
 * dat->chi2. stdout carries chi2_lghtcrv's per-point prints (chi2.c:1147). */
double ref_evaluate(void *h)
{
    ref_session *S = h;
    realize_mod(&S->par, &S->mod);
    calc_fits(&S->par, &S->mod, &S->dat);
    return chi2(&S->par, &S->dat, 0);
}

/* The reference's vary_params (src/shape/vary_params.c:84-327) on the
 * session after ref_evaluate: flags = par->vary_delcor0, vary_radalb,
 * vary_optalb, vary_dopscale (0 = VARY_NONE); delcor0_free / dopscale_free
 * per dataset give the states of the 0th delay-correction coefficient and of
 * the Doppler scale factor ('f' when set, else 'c'). The datasets' and
 * dat's weight sums are formed as read_dat forms them
 * (src/shape/read_dat.c:421-501, 686-692, 1051-1056, 1900-1906). out = the
 * four means deldop_zmax, rad_xsec, opt_brightness, cos_subradarlat. */
void ref_vary_params(void *h, const int *flags, const int *delcor0_free, const int *dopscale_free, double *out)
{
    ref_session *S = h;
    struct dat_t *dat = &S->dat;
    S->par.vary_delcor0 = (unsigned char)flags[0];
    S->par.vary_radalb = (unsigned char)flags[1];
    S->par.vary_optalb = (unsigned char)flags[2];
    S->par.vary_dopscale = (unsigned char)flags[3];
    dat->sum_deldop_zmax_weights = dat->sum_rad_xsec_weights = 0.0;
    dat->sum_opt_brightness_weights = dat->sum_cos_subradarlat_weights = 0.0;
    for (int s = 0; s < dat->nsets; s++) {
        struct set_t *set = &dat->set[s];
        if (set->type == DELAY) {
            struct deldop_t *dd = &set->desc.deldop;
            if (!dd->delcor.a) {
                dd->delcor.n = 0;
                dd->delcor.a = calloc(1, sizeof(struct param_t));
            }
            dd->delcor.a[0].state = delcor0_free[s] ? 'f' : 'c';
            dd->dopscale.state = dopscale_free[s] ? 'f' : 'c';
            dd->sum_deldop_zmax_weights = dd->sum_rad_xsec_weights = dd->sum_cos_subradarlat_weights = 0.0;
            for (int f = 0; f < dd->nframes; f++) {
                const double w = dd->frame[f].weight;
                if (dd->delcor.a[0].state != 'c') dd->sum_deldop_zmax_weights += w;
                if (dd->frame[f].cal.state == 'c') dd->sum_rad_xsec_weights += w;
                if (dd->dopscale.state != 'c') dd->sum_cos_subradarlat_weights += w;
            }
            dat->sum_deldop_zmax_weights += dd->sum_deldop_zmax_weights;
            dat->sum_rad_xsec_weights += dd->sum_rad_xsec_weights;
            dat->sum_cos_subradarlat_weights += dd->sum_cos_subradarlat_weights;
        } else if (set->type == DOPPLER) {
            struct doppler_t *dp = &set->desc.doppler;
            dp->dopscale.state = dopscale_free[s] ? 'f' : 'c';
            dp->sum_rad_xsec_weights = dp->sum_cos_subradarlat_weights = 0.0;
            for (int f = 0; f < dp->nframes; f++) {
                const double w = dp->frame[f].weight;
                if (dp->frame[f].cal.state == 'c') dp->sum_rad_xsec_weights += w;
                if (dp->dopscale.state != 'c') dp->sum_cos_subradarlat_weights += w;
            }
            dat->sum_rad_xsec_weights += dp->sum_rad_xsec_weights;
            dat->sum_cos_subradarlat_weights += dp->sum_cos_subradarlat_weights;
        } else if (set->type == LGHTCRV) {
            struct lghtcrv_t *lc = &set->desc.lghtcrv;
            lc->sum_opt_brightness_weights = (lc->cal.state == 'c') ? lc->weight * lc->n : 0.0;
            dat->sum_opt_brightness_weights += lc->sum_opt_brightness_weights;
        }
    }
    vary_params(&S->par, &S->mod, dat, S->par.action, &out[0], &out[1], &out[2], &out[3]);
}

/* calc_fits + chi2 without re-realizing (model already realized). */
double ref_calc_chi2(void *h)
{
    ref_session *S = h;
    calc_fits(&S->par, &S->mod, &S->dat);
    return chi2(&S->par, &S->dat, 0);
}

void ref_get_realized(void *h, double *x, double *vn, double *fn, double *area)
{
    ref_session *S = h;
    int v0 = 0, f0 = 0;
    for (int c = 0; c < S->mod.shape.ncomp; c++) {
        struct vertices_t *real = &S->mod.shape.comp[c].real;
        for (int i = 0; i < real->nv; i++)
            for (int j = 0; j < 3; j++) {
                x[3 * (v0 + i) + j] = real->v[i].x[j];
                vn[3 * (v0 + i) + j] = real->v[i].n[j];
            }
        for (int f = 0; f < real->nf; f++) {
            for (int j = 0; j < 3; j++) fn[3 * (f0 + f) + j] = real->f[f].n[j];
            area[f0 + f] = real->f[f].area;
        }
        v0 += real->nv;
        f0 += real->nf;
    }
}

/* Flags of par after calc_fits: [posbnd, posbnd_logfactor, badradar, badradar_logfactor]. */
void ref_get_flags(void *h, double out[4])
{
    ref_session *S = h;
    out[0] = S->par.posbnd; out[1] = S->par.posbnd_logfactor;
    out[2] = S->par.badradar; out[3] = S->par.badradar_logfactor;
}

void ref_get_seen(void *h, unsigned char *seen)
{
    ref_session *S = h;
    int f0 = 0;
    for (int c = 0; c < S->mod.shape.ncomp; c++) {
        struct vertices_t *real = &S->mod.shape.comp[c].real;
        for (int f = 0; f < real->nf; f++) seen[f0 + f] = real->f[f].seen;
        f0 += real->nf;
    }
}

/* The model-wide index of component c's facet f (components back to back). */
static int ref_global_facet(const struct mod_t *mod, int c, int f)
{
    if (!mod || f < 0 || c < 0 || c >= mod->shape.ncomp) return f;
    for (int k = 0; k < c; k++) f += mod->shape.comp[k].real.nf;
    return f;
}

static void ref_copy_pos_out(const struct mod_t *mod, const struct pos_t *pos, double *z, double *cose,
                             double *cosi, int *f, double *zill, int *fill, int lims[8])
{
    int n = pos->n, side = 2 * n + 1;
    for (int i = -n; i <= n; i++)
        for (int j = -n; j <= n; j++) {
            size_t p = (size_t)(i + n) * side + (size_t)(j + n);
            if (z) z[p] = pos->z[i][j];
            if (cose) cose[p] = pos->cose[i][j];
            if (cosi) cosi[p] = pos->cosi[i][j];
            if (f) f[p] = ref_global_facet(mod, pos->comp[i][j], pos->f[i][j]);
            if (zill) zill[p] = pos->zill[i][j];
            if (fill) fill[p] = ref_global_facet(mod, pos->bistatic ? pos->compill[i][j] : 0, pos->fill[i][j]);
        }
    if (lims) {
        lims[0] = pos->xlim[0]; lims[1] = pos->xlim[1];
        lims[2] = pos->ylim[0]; lims[3] = pos->ylim[1];
        lims[4] = pos->xlim2[0]; lims[5] = pos->xlim2[1];
        lims[6] = pos->ylim2[0]; lims[7] = pos->ylim2[1];
    }
}

/* Outputs of one delay-Doppler frame after ref_evaluate. Any pointer may be NULL.
 * res receives xlim/ylim, idellim/idoplim, dellim/doplim, badradar_logfactor,
 * posbnd_logfactor (of the pos), cal and chi2. */
void ref_get_deldop_frame(void *h, int s, int f, double *fit, double *z, double *cose,
                          int *fac, shape_deldop_result *res)
{
    ref_session *S = h;
    struct deldopfrm_t *fr = &S->dat.set[s].desc.deldop.frame[f];
    if (fit)
        for (int i = 1; i <= fr->ndel; i++)
            for (int j = 1; j <= fr->ndop; j++)
                fit[(size_t)(i - 1) * fr->ndop + (size_t)(j - 1)] = fr->fit[i][j];
    int lims[8];
    ref_copy_pos_out(&S->mod, &fr->pos, z, cose, NULL, fac, NULL, NULL, lims);
    if (res) {
        memset(res, 0, sizeof *res);
        res->xlim[0] = lims[0]; res->xlim[1] = lims[1];
        res->ylim[0] = lims[2]; res->ylim[1] = lims[3];
        res->idellim[0] = fr->idellim[0]; res->idellim[1] = fr->idellim[1];
        res->idoplim[0] = fr->idoplim[0]; res->idoplim[1] = fr->idoplim[1];
        res->dellim[0] = fr->dellim[0]; res->dellim[1] = fr->dellim[1];
        res->doplim[0] = fr->doplim[0]; res->doplim[1] = fr->doplim[1];
        res->badradar_logfactor = fr->badradar_logfactor;
        res->posbnd_logfactor = fr->pos.posbnd_logfactor;
        res->cal = fr->cal.val;
        res->chi2 = fr->chi2;
    }
}

/* Outputs of one Doppler frame after ref_evaluate (delay fields blank). */
void ref_get_doppler_frame(void *h, int s, int f, double *fit, double *z, double *cose,
                           int *fac, shape_deldop_result *res)
{
    ref_session *S = h;
    struct dopfrm_t *fr = &S->dat.set[s].desc.doppler.frame[f];
    if (fit)
        for (int j = 1; j <= fr->ndop; j++) fit[j - 1] = fr->fit[j];
    int lims[8];
    ref_copy_pos_out(&S->mod, &fr->pos, z, cose, NULL, fac, NULL, NULL, lims);
    if (res) {
        memset(res, 0, sizeof *res);
        res->xlim[0] = lims[0]; res->xlim[1] = lims[1];
        res->ylim[0] = lims[2]; res->ylim[1] = lims[3];
        res->idoplim[0] = fr->idoplim[0]; res->idoplim[1] = fr->idoplim[1];
        res->doplim[0] = fr->doplim[0]; res->doplim[1] = fr->doplim[1];
        res->badradar_logfactor = fr->badradar_logfactor;
        res->posbnd_logfactor = fr->pos.posbnd_logfactor;
        res->o2 = fr->overflow_o2;     /* the overflow terms (chi2 sums are local to chi2_doppler) */
        res->m2 = fr->overflow_m2;
        res->cal = fr->cal.val;
        res->chi2 = fr->chi2;
    }
}

/* The reference's natural cubic spline as calc_lghtcrv uses it
 * (src/shape/calc_fits.c:1923-1933): spline() over the n knots (x, y) with
 * both end derivatives 2e30, then splint() at each of the m epochs t. */
void ref_spline_eval(const double *x, const double *y, int n, const double *t, int m, double *out)
{
    double *xv = vector(1, n), *yv = vector(1, n), *y2 = vector(1, n);
    for (int i = 1; i <= n; i++) { xv[i] = x[i - 1]; yv[i] = y[i - 1]; }
    spline(xv, yv, n, 2.0e30, 2.0e30, y2);
    for (int k = 0; k < m; k++) splint(xv, yv, y2, n, t[k], &out[k]);
    free_vector(xv, 1, n);
    free_vector(yv, 1, n);
    free_vector(y2, 1, n);
}

/* Outputs of a lightcurve set after ref_evaluate: y[ncalc], fit[n], [cal, chi2]. */
void ref_get_lghtcrv(void *h, int s, double *y, double *fit, double out[2])
{
    ref_session *S = h;
    struct lghtcrv_t *lc = &S->dat.set[s].desc.lghtcrv;
    for (int i = 1; i <= lc->ncalc; i++) y[i - 1] = lc->y[i];
    for (int i = 1; i <= lc->n; i++) fit[i - 1] = lc->fit[i];
    out[0] = lc->cal.val;
    out[1] = S->dat.set[s].chi2;
}

/* POS maps of one calculated lightcurve point (1-based i as in the reference). */
void ref_get_lghtcrv_pos(void *h, int s, int i, double *z, double *cose, double *cosi,
                         int *fac, double *zill, int *fill, int lims[8])
{
    ref_session *S = h;
    ref_copy_pos_out(&S->mod, &S->dat.set[s].desc.lghtcrv.rend[i].pos, z, cose, cosi, fac, zill, fill, lims);
}

double ref_set_chi2(void *h, int s)
{
    ref_session *S = h;
    return S->dat.set[s].chi2;
}

void ref_free(void *h)
{
    ref_session *S = h;
    if (!S) return;
    for (int s = 0; s < S->dat.nsets; s++) {
        struct set_t *set = &S->dat.set[s];
        if (set->type == DELAY) {
            struct deldop_t *dd = &set->desc.deldop;
            for (int f = 0; f < dd->nframes; f++) {
                struct deldopfrm_t *fr = &dd->frame[f];
                free_matrix(fr->obs, 1, fr->ndel, 1, fr->ndop);
                free_matrix(fr->fit, 1, fr->ndel, 1, fr->ndop);
                free_matrix(fr->oneovervar, 1, fr->ndel, 1, fr->ndop);
                ref_free_pos(&fr->pos);
                free(fr->view);
            }
            free(dd->frame);
        } else if (set->type == DOPPLER) {
            struct doppler_t *dp = &set->desc.doppler;
            for (int f = 0; f < dp->nframes; f++) {
                struct dopfrm_t *fr = &dp->frame[f];
                free_vector(fr->obs, 1, fr->ndop);
                free_vector(fr->fit, 1, fr->ndop);
                free_vector(fr->oneovervar, 1, fr->ndop);
                ref_free_pos(&fr->pos);
                free(fr->view);
            }
            free(dp->frame);
        } else if (set->type == LGHTCRV) {
            struct lghtcrv_t *lc = &set->desc.lghtcrv;
            for (int i = 1; i <= lc->ncalc; i++) ref_free_pos(&lc->rend[i].pos);
            free(lc->rend);
        } else if (set->type == POS) {
            struct poset_t *po = &set->desc.poset;
            for (int f = 0; f < po->nframes; f++) {
                struct posetfrm_t *fr = &po->frame[f];
                ref_free_pos(&fr->pos);
                free_matrix(fr->obs.b, 1, fr->ncol, 1, fr->nrow);
                free_matrix(fr->fit.b, 1, fr->ncol, 1, fr->nrow);
                free_matrix(fr->oneovervar, 1, fr->ncol, 1, fr->nrow);
                free(fr->view);
            }
            free(po->frame);
        }
    }
    free(S->dat.set);
    for (int c = 0; c < S->mod.shape.ncomp; c++) {
        struct vertices_t *real = &S->mod.shape.comp[c].real;
        for (int i = 0; i < real->nv; i++) free(real->v[i].af);
        free(real->v); free(real->f);
    }
    free(S->mod.shape.comp);
    free(S);
}

/* Multi-core evaluation in the reference's host-multithreading scheme: one
 * dataset (here: one session) per thread, as calc_fits_hmt assigns datasets
 * to threads (src/HostMultiThreading/calc_fits_hmt.c:134-160). */
typedef struct { void *h; double chi2; } ref_mt_job;
static void *ref_mt_worker(void *arg)
{
    ref_mt_job *j = arg;
    j->chi2 = ref_evaluate(j->h);
    return NULL;
}

double ref_evaluate_mt(void **sessions, int nsessions)
{
    pthread_t *th = calloc((size_t)nsessions, sizeof(pthread_t));
    ref_mt_job *jobs = calloc((size_t)nsessions, sizeof(ref_mt_job));
    for (int i = 0; i < nsessions; i++) {
        jobs[i].h = sessions[i];
        pthread_create(&th[i], NULL, ref_mt_worker, &jobs[i]);
    }
    double tot = 0.0;
    for (int i = 0; i < nsessions; i++) {
        pthread_join(th[i], NULL);
        tot += jobs[i].chi2;
    }
    free(th); free(jobs);
    return tot;
}

/* Line searches of the reference, for pinning the engine's own bracketing
 * and Brent minimiser: the objective is a plain C callback. */
typedef double (*ref_objfn)(double);
void ref_mnbrak(double *ax, double *bx, double *cx, double *fa, double *fb, double *fc, ref_objfn fn)
{
    mnbrak(ax, bx, cx, fa, fb, fc, fn);
}
double ref_brent_abs(double ax, double bx, double cx, ref_objfn fn, double tol, double abstol, double *xmin)
{
    return brent_abs(ax, bx, cx, fn, tol, abstol, xmin);
}


/* The reference's spin realization (realize_spin, src/shape/realize_spin.c)
 * for n one-view frames of a single delay-Doppler set with view epochs t[]
 * and orbital spin contributions orbspin[3n]: the check of
 * shape_realize_spin. Non-principal-axis states use the reference's
 * brute-force integration with tolerance int_abstol. Writes each view's ae
 * (row-major) and total spin. */
int ref_realize_spin_frames(const shape_spin_state *sp, const double angleoff[3], const double omegaoff[3],
                            int n, const double *t, const double *orbspin, double *ae, double *spin_out,
                            double int_abstol)
{
    if (sp->n_impulse < 0 || sp->n_impulse > MAXIMP) return -1;
    struct par_t *par = calloc(1, sizeof *par);
    struct mod_t *mod = calloc(1, sizeof *mod);
    struct dat_t *dat = calloc(1, sizeof *dat);
    par->int_method = BRUTE;
    par->int_abstol = int_abstol;
    mod->spin.pa = (unsigned char)sp->pa;
    mod->spin.t0 = sp->t0;
    for (int j = 0; j < 3; j++) {
        mod->spin.angle[j].val = sp->angle[j];
        mod->spin.omega[j].val = sp->omega[j];
        mod->spin.omegadot[j].val = sp->omegadot[j];
        mod->spin.inertia[j].val = sp->inertia[j] > 0.0 ? sp->inertia[j] : 1.0;
    }
    mod->spin.n_impulse = sp->n_impulse;
    for (int k = 0; k < sp->n_impulse; k++) {
        mod->spin.t_impulse[k] = sp->t_impulse[k];
        for (int j = 0; j < 3; j++) mod->spin.impulse[k][j].val = sp->impulse[k][j];
    }
    mod->spin.lib_amp.val = sp->lib_amp;
    mod->spin.lib_freq.val = sp->lib_freq;
    mod->spin.lib_phase.val = sp->lib_phase;
    dat->nsets = 1;
    dat->set = calloc(1, sizeof(struct set_t));
    struct set_t *set = &dat->set[0];
    set->type = DELAY;
    for (int j = 0; j < 3; j++) {
        set->angleoff[j].val = angleoff[j];
        set->angleoff[j].state = 'c';
        set->omegaoff[j].val = omegaoff[j];
        set->omegaoff[j].state = 'c';
    }
    struct deldop_t *dd = &set->desc.deldop;
    dd->nframes = n;
    dd->nviews = 1;
    dd->frame = calloc((size_t)(n > 0 ? n : 1), sizeof(struct deldopfrm_t));
    for (int f = 0; f < n; f++) {
        dd->frame[f].view = calloc(1, sizeof(struct deldopview_t));
        dd->frame[f].view[0].t = t[f];
        for (int j = 0; j < 3; j++) dd->frame[f].view[0].orbspin[j] = orbspin[3 * f + j];
    }
    realize_spin(par, mod, dat);
    for (int f = 0; f < n; f++) {
        for (int i = 0; i < 3; i++) {
            for (int j = 0; j < 3; j++) ae[9 * f + 3 * i + j] = dd->frame[f].view[0].ae[i][j];
            spin_out[3 * f + i] = dd->frame[f].view[0].spin[i];
        }
        free(dd->frame[f].view);
    }
    free(dd->frame);
    free(dat->set);
    free(dat);
    free(mod);
    free(par);
    return 0;
}


/* The reference's penalties(par, mod, dat) (src/shape/penalties.c:121-1236)
 * after realize_mod, for n penalties of the given types and weights: the
 * check of the engine's penalty terms. The model's edges come from the
 * reference's own setupsides (src/shape/read_mod.c:2386). sp (or NULL)
 * supplies spin.inertia and the spin impulses; angleoff / omegaoff (or
 * NULL) 3 doubles per dataset. Writes par->pen.base[1..n] to base and
 * returns the penalty sum. */
double ref_penalties(void *h, int n, const int *type, const double *weight, const shape_spin_state *sp,
                     const double *angleoff, const double *omegaoff, double *base)
{
    ref_session *S = h;
    for (int c = 0; c < S->mod.shape.ncomp; c++) {
        struct vertices_t *real = &S->mod.shape.comp[c].real;
        if (!real->s) setupsides(real);
    }
    if (sp) {
        S->mod.spin.n_impulse = sp->n_impulse;
        for (int j = 0; j < 3; j++) S->mod.spin.inertia[j].val = sp->inertia[j];
        for (int k = 0; k < sp->n_impulse; k++)
            for (int j = 0; j < 3; j++) S->mod.spin.impulse[k][j].val = sp->impulse[k][j];
    }
    for (int s = 0; s < S->dat.nsets; s++)
        for (int j = 0; j < 3; j++) {
            S->dat.set[s].angleoff[j].val = angleoff ? angleoff[3 * s + j] : 0.0;
            S->dat.set[s].omegaoff[j].val = omegaoff ? omegaoff[3 * s + j] : 0.0;
        }
    realize_mod(&S->par, &S->mod);
    struct par_t *par = &S->par;
    par->pen.n = n;
    par->pen.type = calloc((size_t)n + 1, sizeof(int));
    par->pen.weight = calloc((size_t)n + 1, sizeof(double));
    par->pen.base = calloc((size_t)n + 1, sizeof(double));
    for (int i = 0; i < n; i++) {
        par->pen.type[i + 1] = type[i];
        par->pen.weight[i + 1] = weight[i];
    }
    par->showstate = 0;
    double sum = penalties(par, &S->mod, &S->dat);
    for (int i = 0; i < n; i++) base[i] = par->pen.base[i + 1];
    free(par->pen.type);
    free(par->pen.weight);
    free(par->pen.base);
    par->pen.n = 0;
    par->pen.type = NULL;
    par->pen.weight = par->pen.base = NULL;
    return sum;
}


/* The act flags realize_mod's check_surface left (src/shape/realize_mod.c:
 * 572-756), model-wide: vertices, then facets, components back to back. */
void ref_get_active(void *h, unsigned char *vact, unsigned char *fact)
{
    ref_session *S = h;
    int v0 = 0, f0 = 0;
    for (int c = 0; c < S->mod.shape.ncomp; c++) {
        const struct vertices_t *real = &S->mod.shape.comp[c].real;
        for (int i = 0; i < real->nv; i++) vact[v0 + i] = (unsigned char)real->v[i].act;
        for (int f = 0; f < real->nf; f++) fact[f0 + f] = (unsigned char)real->f[f].act;
        v0 += real->nv;
        f0 += real->nf;
    }
}


/* The reference's read_mod (src/shape/read_mod.c:204-227) on a model file:
 * the check of shape_mod_read. The ref_mod_* getters copy the result into
 * the engine's descriptor types. */
typedef struct { struct par_t par; struct mod_t mod; } ref_modfile;

void *ref_mod_read(const char *path)
{
    ref_modfile *F = calloc(1, sizeof *F);
    F->par.action = FIT;
    snprintf(F->mod.name, sizeof F->mod.name, "%s", path);
    read_mod(&F->par, &F->mod);
    return F;
}

/* Sizes into nv / nf; the arrays (each may be NULL) as shape_model_desc
 * holds them. */
/* The model's vertex components back to back: vertex and facet indices made
 * model-wide (a component's local index plus the vertices or facets of the
 * components before it); scale holds component 0's factors. */
void ref_mod_shape(void *h, int *nv, int *nf, double *a, double *u, double *r, double *scale, int *fv,
                   int *af_ptr, int *af_idx)
{
    ref_modfile *F = h;
    int v0 = 0, f0 = 0, k = 0;
    for (int c = 0; c < F->mod.shape.ncomp; c++) {
        struct vertices_t *real = &F->mod.shape.comp[c].real;
        if (c == 0)
            for (int j = 0; j < 3 && scale; j++) scale[j] = real->scalefactor[j].val;
        for (int i = 0; i < real->nv; i++) {
            const int g = v0 + i;
            for (int j = 0; j < 3; j++) {
                if (a) a[3 * g + j] = real->v[i].a[j];
                if (u) u[3 * g + j] = real->v[i].u[j];
            }
            if (r) r[g] = real->v[i].r.val;
            if (af_ptr) af_ptr[g] = k;
            for (int q = 0; q < real->v[i].naf; q++, k++)
                if (af_idx) af_idx[k] = f0 + real->v[i].af[q];
        }
        for (int f = 0; f < real->nf && fv; f++)
            for (int j = 0; j < 3; j++) fv[3 * (f0 + f) + j] = v0 + real->f[f].v[j];
        v0 += real->nv;
        f0 += real->nf;
    }
    *nv = v0;
    *nf = f0;
    if (af_ptr) af_ptr[v0] = k;
}

/* Component c's vertex and facet counts, scale factors, linear offsets (km)
 * and rotation offsets (radians); returns the number of components. */
int ref_mod_comp(void *h, int c, int *nv, int *nf, double *scale, double *off, double *rot)
{
    ref_modfile *F = h;
    if (c < 0 || c >= F->mod.shape.ncomp) return F->mod.shape.ncomp;
    struct comp_t *cm = &F->mod.shape.comp[c];
    *nv = cm->real.nv;
    *nf = cm->real.nf;
    for (int j = 0; j < 3; j++) {
        scale[j] = cm->real.scalefactor[j].val;
        off[j] = cm->off[j].val;
        rot[j] = cm->rot[j].val;
    }
    return F->mod.shape.ncomp;
}

int ref_mod_radar(void *h, int i, shape_radar_law *L)
{
    ref_modfile *F = h;
    struct photo_t *ph = &F->mod.photo;
    memset(L, 0, sizeof *L);
    if (i < 0 || i >= ph->nradlaws) return ph->nradlaws;      /* count only */
    L->type = ph->radtype[i] == NOLAW ? 0 : ph->radtype[i];
    switch (ph->radtype[i]) {
    case COSINELAW_DIFF:
        L->diff_R = ph->radar[i].RC.R.val; L->diff_C = ph->radar[i].RC.C.val; break;
    case GAUSSIANLAW: case HAGFORSLAW: case COSINELAW_QS:
        L->qs_R = ph->radar[i].quasispec.R.val; L->qs_C = ph->radar[i].quasispec.C.val;
        L->qs_cos_cutoff = ph->radar[i].quasispec.cos_cutoff; break;
    case GAUSSIAN_COSINE: case HAGFORS_COSINE: case COSINE_COSINE:
        L->qs_R = ph->radar[i].hybrid.qs.R.val; L->qs_C = ph->radar[i].hybrid.qs.C.val;
        L->qs_cos_cutoff = ph->radar[i].hybrid.qs.cos_cutoff;
        L->diff_R = ph->radar[i].hybrid.diff.R.val; L->diff_C = ph->radar[i].hybrid.diff.C.val; break;
    default: break;
    }
    return ph->nradlaws;
}

int ref_mod_optical(void *h, int i, shape_optical_law *L)
{
    ref_modfile *F = h;
    struct photo_t *ph = &F->mod.photo;
    memset(L, 0, sizeof *L);
    if (i < 0 || i >= ph->noptlaws) return ph->noptlaws;      /* count only */
    L->type = ph->opttype[i] == NOLAW ? 0 : ph->opttype[i];
    if (ph->opttype[i] == KAASALAINEN) {
        L->R = ph->optical[i].kaas.R.val; L->wt = ph->optical[i].kaas.wt.val;
        L->A0 = ph->optical[i].kaas.A0.val; L->D = ph->optical[i].kaas.D.val;
        L->k = ph->optical[i].kaas.k.val;
    } else if (ph->opttype[i] == LAMBERTLAW || ph->opttype[i] == LOMMEL) {
        L->R = ph->optical[i].R.R.val;
    }
    return ph->noptlaws;
}

void ref_mod_spin(void *h, shape_spin_state *sp)
{
    ref_modfile *F = h;
    const struct spin_t *s = &F->mod.spin;
    memset(sp, 0, sizeof *sp);
    sp->pa = s->pa;
    sp->t0 = s->t0;
    for (int j = 0; j < 3; j++) {
        sp->angle[j] = s->angle[j].val;
        sp->omega[j] = s->omega[j].val;
        sp->omegadot[j] = s->omegadot[j].val;
        sp->inertia[j] = s->inertia[j].val;
    }
    sp->n_impulse = s->n_impulse;
    for (int n = 0; n < s->n_impulse && n < SHAPE_MAX_IMPULSES; n++) {
        sp->t_impulse[n] = s->t_impulse[n];
        for (int j = 0; j < 3; j++) sp->impulse[n][j] = s->impulse[n][j].val;
    }
    sp->lib_amp = s->lib_amp.val;
    sp->lib_freq = s->lib_freq.val;
    sp->lib_phase = s->lib_phase.val;
}


/* The reference's data-file readers (read_deldop_ascii / _binary / _rdf
 * and read_doppler_*, src/shape/read_dat.c:2074-2260) on one file: kind 0-2
 * delay-Doppler ascii / binary / rdf, 3-5 the Doppler ones (ndel = 1).
 * obs receives the window idel_use x idop_use, delay-major. */
void read_deldop_ascii(FILE *fin, struct deldop_t *deldop, int iframe, int idel_use[2], int idop_use[2]);
void read_deldop_binary(FILE *fin, struct deldop_t *deldop, int iframe, int idel_use[2], int idop_use[2],
                        int swap_bytes);
void read_deldop_rdf(FILE *fin, struct deldop_t *deldop, int iframe, int idel_use[2], int idop_use[2],
                     int swap_bytes);
void read_doppler_ascii(FILE *fin, struct doppler_t *doppler, int iframe, int idop_use[2]);
void read_doppler_binary(FILE *fin, struct doppler_t *doppler, int iframe, int idop_use[2], int swap_bytes);
void read_doppler_rdf(FILE *fin, struct doppler_t *doppler, int iframe, int idop_use[2], int swap_bytes);

int ref_read_radar_data(const char *path, int kind, int ndel, int ndop, const int *idel_in, const int *idop_in,
                        int swap, double sdev, double *obs)
{
    int idel_use[2] = {idel_in[0], idel_in[1]}, idop_use[2] = {idop_in[0], idop_in[1]};
    const int wdel = idel_use[1] - idel_use[0] + 1, wdop = idop_use[1] - idop_use[0] + 1;
    FILE *fin = fopen(path, "rb");
    if (!fin) return -1;
    if (kind < 3) {
        struct deldop_t *dd = calloc(1, sizeof *dd);      /* 32 MB: not on the stack */
        dd->ndel = ndel;
        dd->ndop = ndop;
        dd->frame = calloc(1, sizeof(struct deldopfrm_t));
        dd->frame[0].sdev = sdev;
        dd->frame[0].obs = matrix(1, wdel, 1, wdop);
        if (kind == 0) read_deldop_ascii(fin, dd, 0, idel_use, idop_use);
        else if (kind == 1) read_deldop_binary(fin, dd, 0, idel_use, idop_use, swap);
        else read_deldop_rdf(fin, dd, 0, idel_use, idop_use, swap);
        for (int j = 1; j <= wdel; j++)
            for (int k = 1; k <= wdop; k++) obs[(j - 1) * wdop + (k - 1)] = dd->frame[0].obs[j][k];
        free_matrix(dd->frame[0].obs, 1, wdel, 1, wdop);
        free(dd->frame);
        free(dd);
    } else {
        struct doppler_t *dp = calloc(1, sizeof *dp);
        dp->ndop = ndop;
        dp->frame = calloc(1, sizeof(struct dopfrm_t));
        dp->frame[0].sdev = sdev;
        dp->frame[0].obs = vector(1, wdop);
        if (kind == 3) read_doppler_ascii(fin, dp, 0, idop_use);
        else if (kind == 4) read_doppler_binary(fin, dp, 0, idop_use, swap);
        else read_doppler_rdf(fin, dp, 0, idop_use, swap);
        for (int k = 1; k <= wdop; k++) obs[k - 1] = dp->frame[0].obs[k];
        free_vector(dp->frame[0].obs, 1, wdop);
        free(dp->frame);
        free(dp);
    }
    fclose(fin);
    return 0;
}


/* The reference's ephem2mat (src/shape/ephem2mat.c:33-228) on ephemeris
 * tables given as (t, ra, dec, dist) quadruples: the check of
 * shape_ephem_view. nsun = 0: monostatic. */
double ref_ephem2mat(const double *ast, int nast, const double *sun, int nsun, double t, double *oe, double *se,
                     double *s, double *phase_az)
{
    struct ephem_t A, S;
    A.n = nast;
    A.pnt = (struct ephpnt_t *)ast;
    S.n = nsun;
    S.pnt = (struct ephpnt_t *)sun;
    double o[3][3], e[3][3];
    memset(e, 0, sizeof e);
    double dist = ephem2mat(A, S, t, o, e, s, &phase_az[0], &phase_az[1], nsun > 0);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) { oe[3 * i + j] = o[i][j]; se[3 * i + j] = e[i][j]; }
    return dist;
}


/* The reference's deldopoffs (src/shape/deldopoffs.c:17-42) for nv single-
 * view frames at epochs t[]: the check of shape_delcor_offsets. */
void deldopoffs(struct deldop_t *deldop);
void ref_deldopoffs(const double *a, int n, double t0, int nv, const double *t, double delpp, double doppp,
                    double Ftx, double *deloff, double *dopoff)
{
    struct deldop_t *dd = calloc(1, sizeof *dd);
    dd->nframes = nv;
    dd->nviews = 1;
    dd->del_per_pixel = delpp;
    dd->dop_per_pixel = doppp;
    dd->Ftx = Ftx;
    dd->delcor.t0 = t0;
    dd->delcor.n = n;
    dd->delcor.a = calloc((size_t)n + 1, sizeof(struct param_t));
    for (int i = 0; i <= n; i++) dd->delcor.a[i].val = a[i];
    dd->frame = calloc((size_t)nv, sizeof(struct deldopfrm_t));
    for (int f = 0; f < nv; f++) {
        dd->frame[f].view = calloc(1, sizeof(struct deldopview_t));
        dd->frame[f].view[0].t = t[f];
    }
    deldopoffs(dd);
    for (int f = 0; f < nv; f++) {
        deloff[f] = dd->frame[f].view[0].deloff;
        dopoff[f] = dd->frame[f].view[0].dopoff;
        free(dd->frame[f].view);
    }
    free(dd->frame);
    free(dd->delcor.a);
    free(dd);
}


/* The reference's read_mod + read_dat + realize_delcor + realize_spin on a
 * model file and an observation file (paths relative to the current
 * directory, as the reference opens them): the check of shape_obs_read /
 * shape_obs_frames. ref_obs_frame copies one delay-Doppler frame's view
 * and data out. */
typedef struct { struct par_t par; struct mod_t mod; struct dat_t dat; } ref_obsfile;

void *ref_obs_read(const char *modpath, const char *obspath, int perform_ltc, double dd_gamma, int speckle,
                   int big_endian)
{
    ref_obsfile *F = calloc(1, sizeof *F);
    F->par.action = FIT;
    F->par.perform_ltc = (unsigned char)perform_ltc;
    F->par.dd_gamma = dd_gamma;
    F->par.speckle = (unsigned char)speckle;
    F->par.endian = big_endian ? BIG_ENDIAN_DATA : LITTLE_ENDIAN_DATA;
    F->par.int_method = BRUTE;
    F->par.int_abstol = 1e-7;
    F->par.pos_scope = LOCAL;              /* POS sizing in read_dat (set_up_pos) */
    F->par.pos_pixels = 151;
    F->par.pos_width = 2.25;
    for (int k = 0; k < MAXSUNMAGS; k++) F->par.sun_appmag[k] = -26.75;
    snprintf(F->mod.name, sizeof F->mod.name, "%s", modpath);
    snprintf(F->dat.name, sizeof F->dat.name, "%s", obspath);
    read_mod(&F->par, &F->mod);
    read_dat(&F->par, &F->mod, &F->dat);
    realize_delcor(&F->dat, 0.0, 0);
    realize_spin(&F->par, &F->mod, &F->dat);
    return F;
}

/* geom: t, oe[9], orbspin[3], ae[9], spin[3], deloff, dopoff, delcom_vig,
 * dopcom_vig, dopDC_vig, weight, dof, cal, sdev (34 doubles); ndel/ndop of
 * the window; obs and oneovervar delay-major (either may be NULL). */
void ref_obs_frame_view(void *h, int s, int f, int k, double *geom, int *nd, double *obs, double *oov)
{
    ref_obsfile *F = h;
    struct deldop_t *dd = &F->dat.set[s].desc.deldop;
    struct deldopfrm_t *fr = &dd->frame[f];
    struct deldopview_t *v = &fr->view[k];
    double *g = geom;
    *g++ = v->t;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) *g++ = v->oe[i][j];
    for (int i = 0; i < 3; i++) *g++ = v->orbspin[i];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) *g++ = v->ae[i][j];
    for (int i = 0; i < 3; i++) *g++ = v->spin[i];
    *g++ = v->deloff; *g++ = v->dopoff;
    *g++ = fr->delcom_vig; *g++ = fr->dopcom_vig; *g++ = fr->dopDC_vig;
    *g++ = fr->weight; *g++ = fr->dof; *g++ = fr->cal.val; *g++ = fr->sdev;
    nd[0] = fr->ndel;
    nd[1] = fr->ndop;
    for (int j = 1; j <= fr->ndel; j++)
        for (int k = 1; k <= fr->ndop; k++) {
            if (obs) obs[(j - 1) * fr->ndop + (k - 1)] = fr->obs[j][k];
            if (oov) oov[(j - 1) * fr->ndop + (k - 1)] = fr->oneovervar[j][k];
        }
}

/* View 0 of a frame (the only one of an unsmeared set). */
void ref_obs_frame(void *h, int s, int f, double *geom, int *nd, double *obs, double *oov)
{
    ref_obs_frame_view(h, s, f, 0, geom, nd, obs, oov);
}

/* Views per frame and the epoch view's index of delay-Doppler set s. */
void ref_obs_views(void *h, int s, int *out)
{
    ref_obsfile *F = h;
    out[0] = F->dat.set[s].desc.deldop.nviews;
    out[1] = F->dat.set[s].desc.deldop.v0;
}

/* A lightcurve set of ref_obs_read's data: sizes = ioptlaw, ncalc, n (x
 * NULL: sizes only); x[ncalc]; per calculated point i, pt[28 i ..] =
 * oe[9], se[9], ae[9], solar_phase; t[n] (first view), obs[n], oov[n];
 * tail = weight, dof, cal. */
void ref_obs_lghtcrv(void *h, int s, int *sizes, double *x, double *pt, double *t, double *obs, double *oov,
                     double *tail)
{
    ref_obsfile *F = h;
    struct lghtcrv_t *lc = &F->dat.set[s].desc.lghtcrv;
    sizes[0] = lc->ioptlaw;
    sizes[1] = lc->ncalc;
    sizes[2] = lc->n;
    if (!x) return;
    for (int i = 1; i <= lc->ncalc; i++) {
        x[i - 1] = lc->x[i];
        double *g = pt + 28 * (size_t)(i - 1);
        for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) *g++ = lc->rend[i].oe[a][b];
        for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) *g++ = lc->rend[i].se[a][b];
        for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) *g++ = lc->rend[i].ae[a][b];
        *g++ = lc->solar_phase[i];
    }
    for (int i = 1; i <= lc->n; i++) {
        t[i - 1] = lc->t[i][0];
        obs[i - 1] = lc->obs[i];
        oov[i - 1] = lc->oneovervar[i];
    }
    tail[0] = lc->weight;
    tail[1] = lc->dof;
    tail[2] = lc->cal.val;
}

/* The asteroid (which = 0) or solar (1) ephemeris of lightcurve set s as
 * ref_obs_read's read_dat left it: per entry t, ra, dec, dist; returns n. */
int ref_obs_lghtcrv_ephem(void *h, int s, int which, double *out)
{
    ref_obsfile *F = h;
    struct lghtcrv_t *lc = &F->dat.set[s].desc.lghtcrv;
    struct ephem_t *e = which ? &lc->solephem : &lc->astephem;
    if (out)
        for (int i = 0; i < e->n; i++) {
            out[4 * i] = e->pnt[i].t; out[4 * i + 1] = e->pnt[i].ra;
            out[4 * i + 2] = e->pnt[i].dec; out[4 * i + 3] = e->pnt[i].dist;
        }
    return e->n;
}

/* A Doppler frame of ref_obs_read's data: geom = t, oe[9], orbspin[3],
 * ae[9], spin[3], dopoff, dopcom_vig, weight, dof, cal, sdev (31 doubles);
 * ndop of the window; the spectrum and its 1/variance. */
void ref_obs_doppler_frame(void *h, int s, int f, double *geom, int *ndop, double *obs, double *oov)
{
    ref_obsfile *F = h;
    struct doppler_t *dp = &F->dat.set[s].desc.doppler;
    struct dopfrm_t *fr = &dp->frame[f];
    struct dopview_t *v = &fr->view[0];
    double *g = geom;
    *g++ = v->t;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) *g++ = v->oe[i][j];
    for (int i = 0; i < 3; i++) *g++ = v->orbspin[i];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) *g++ = v->ae[i][j];
    for (int i = 0; i < 3; i++) *g++ = v->spin[i];
    *g++ = v->dopoff;
    *g++ = fr->dopcom_vig; *g++ = fr->weight; *g++ = fr->dof; *g++ = fr->cal.val; *g++ = fr->sdev;
    *ndop = fr->ndop;
    for (int k = 1; k <= fr->ndop; k++) {
        obs[k - 1] = fr->obs[k];
        oov[k - 1] = fr->oneovervar[k];
    }
}
