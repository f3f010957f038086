/*
 * Helpers shared by the drop-in files (shape_b200_dropin.c,
 * shape_b200_pos.c), compiled inside the reference tree after its head.h:
 * the reference's error convention (bailout) for engine statuses and
 * unsupported inputs, and conversions of the reference's law unions and
 * matrices into the engine's plain descriptions.
 */
#ifndef SHAPE_B200_DROPIN_COMMON_H
#define SHAPE_B200_DROPIN_COMMON_H

#include <string.h>

#include "shape_b200.h"

static inline void b200_fail(const char *what)
{
    static char msg[600];
    snprintf(msg, sizeof msg, "shape_b200: %s: %s\n", what, shape_last_error());
    bailout(msg);
}

static inline void b200_check(int rc, const char *what)
{
    if (rc < 0) b200_fail(what);
}

static inline void b200_unsupported(const char *what)
{
    static char msg[600];
    snprintf(msg, sizeof msg, "shape_b200: unsupported input: %s\n", what);
    bailout(msg);
}

/* ------------------------------------------------------------ conversion */

static inline void rm9(double out[9], double in[3][3])
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) out[3 * i + j] = in[i][j];
}

static inline shape_radar_law radar_law_of(const struct photo_t *ph, int ilaw)
{
    shape_radar_law L;
    memset(&L, 0, sizeof L);
    if (ilaw < 0 || ilaw >= ph->nradlaws) b200_unsupported("radar law index out of range");
    L.type = ph->radtype[ilaw];
    const union radscat_t *r = &ph->radar[ilaw];
    switch (L.type) {
    case COSINELAW_DIFF:
        L.diff_R = r->RC.R.val; L.diff_C = r->RC.C.val; break;
    case GAUSSIANLAW: case HAGFORSLAW: case COSINELAW_QS:
        L.qs_R = r->quasispec.R.val; L.qs_C = r->quasispec.C.val;
        L.qs_cos_cutoff = r->quasispec.cos_cutoff; break;
    case GAUSSIAN_COSINE: case HAGFORS_COSINE: case COSINE_COSINE:
        L.qs_R = r->hybrid.qs.R.val; L.qs_C = r->hybrid.qs.C.val;
        L.qs_cos_cutoff = r->hybrid.qs.cos_cutoff;
        L.diff_R = r->hybrid.diff.R.val; L.diff_C = r->hybrid.diff.C.val; break;
    default:
        b200_unsupported("radar scattering law (facet-dependent or tabular)");
    }
    return L;
}

static inline shape_optical_law optical_law_of(const struct photo_t *ph, int ilaw)
{
    shape_optical_law L;
    memset(&L, 0, sizeof L);
    if (ilaw < 0 || ilaw >= ph->noptlaws) b200_unsupported("optical law index out of range");
    L.type = ph->opttype[ilaw];
    const union optscat_t *o = &ph->optical[ilaw];
    switch (L.type) {
    case LAMBERTLAW: case LOMMEL:
        L.R = o->R.R.val; break;
    case KAASALAINEN:
        L.R = o->kaas.R.val; L.wt = o->kaas.wt.val; L.A0 = o->kaas.A0.val;
        L.D = o->kaas.D.val; L.k = o->kaas.k.val; break;
    default:
        b200_unsupported("optical scattering law (Hapke or facet-dependent)");
    }
    return L;
}

#endif
