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
