/*
 * CPU oracle for SHAPE's model-evaluation hot path. TEST INFRASTRUCTURE ONLY
 * (see shape_oracle.h): used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py, never by the product library.
 *
 * Build with -O2 -ffp-contract=off and no -march flags: the reference CPU
 * code is compiled the same way in oracle/_ref, and FP64 parity of z, facet
 * and cos(e) maps is bit-exact only when neither side contracts a*b+c into
 * an FMA. Expressions below keep the reference's association order; where
 * the reference adds to a literal 0.0 first (cotrans, mmmul, normalize) the
 * restatement does too, because 0.0 + (-0.0) is +0.0.
 */
#include "shape_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MIN(a, b) (((a) < (b)) ? (a) : (b))
#define ORC_MAX(a, b) (((a) > (b)) ? (a) : (b))

/* y = A x (cotrans dir=1, src/util/cotrans.c) with A row-major 3x3. */
static void orc_mv(double y[3], const double A[9], const double x[3])
{
    double t[3];
    for (int i = 0; i < 3; i++) {
        t[i] = 0.0;
        for (int k = 0; k < 3; k++)
            t[i] += A[3 * i + k] * x[k];
    }
    y[0] = t[0]; y[1] = t[1]; y[2] = t[2];
}

/* y = A^T x (cotrans dir=-1, src/util/cotrans.c). */
static void orc_mtv(double y[3], const double A[9], const double x[3])
{
    double t[3];
    for (int i = 0; i < 3; i++) {
        t[i] = 0.0;
        for (int k = 0; k < 3; k++)
            t[i] += A[3 * k + i] * x[k];
    }
    y[0] = t[0]; y[1] = t[1]; y[2] = t[2];
}

/* M = B * A^T: the "mtrnsps(oa, ae); mmmul(oa, B, oa)" idiom of
 * src/shape/posvis.c:101-122 and src/shape/posmask.c:70-71
 * (src/util/mmmul.c, src/util/mtrnsps.c). */
static void orc_mul_bt(double M[9], const double B[9], const double A[9])
{
    double t[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            t[3 * i + j] = 0.0;
            for (int k = 0; k < 3; k++)
                t[3 * i + j] += B[3 * i + k] * A[3 * j + k];
        }
    memcpy(M, t, sizeof t);
}

/* normalize (src/util/normalize.c). */
static double orc_normalize(double u[3])
{
    double norm = 0.0;
    for (int i = 0; i < 3; i++)
        norm += u[i] * u[i];
    norm = sqrt(norm);
    if (norm != 0.0)
        for (int i = 0; i < 3; i++)
            u[i] /= norm;
    return norm;
}

/* ------------------------------------------------------------------ realize */

/* realize_coordinates for a VERTEX component with no rotation/offset
 * (src/shape/realize_mod.c:471-479 vertex coordinates, :532-545 facnrm per
 * facet via src/shape/facnrm.c:13-25 and src/util/cross.c, :550-563 vertex
 * normals as the normalized sum of attached facet normals in af order). */
void orc_realize_vertex(const shape_model_desc *m, double *x, double *vn,
                        double *fn, double *area)
{
    for (int i = 0; i < m->nv; i++)
        for (int j = 0; j < 3; j++)
            x[3 * i + j] = m->scale[j] * (m->u[3 * i + j] * m->r[i] + m->a[3 * i + j]);

    for (int f = 0; f < m->nf; f++) {
        const double *p0 = x + 3 * m->fv[3 * f + 0];
        const double *p1 = x + 3 * m->fv[3 * f + 1];
        const double *p2 = x + 3 * m->fv[3 * f + 2];
        double a[3], b[3], c[3];
        for (int i = 0; i < 3; i++) {
            a[i] = p1[i] - p0[i];
            b[i] = p2[i] - p1[i];
        }
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
        double len = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        if (area) area[f] = 0.5 * len;
        orc_normalize(c);
        fn[3 * f + 0] = c[0]; fn[3 * f + 1] = c[1]; fn[3 * f + 2] = c[2];
    }

    for (int i = 0; i < m->nv; i++) {
        double n[3] = {0.0, 0.0, 0.0};
        for (int j = m->af_ptr[i]; j < m->af_ptr[i + 1]; j++) {
            int f = m->af_idx[j];
            for (int k = 0; k < 3; k++)
                n[k] += fn[3 * f + k];
        }
        orc_normalize(n);
        for (int k = 0; k < 3; k++)
            vn[3 * i + k] = n[k];
    }
}

/* ------------------------------------------------------------------- posclr */

int orc_pos_alloc(orc_pos *pos, int n, int bistatic)
{
    size_t np = (size_t)(2 * n + 1) * (size_t)(2 * n + 1);
    memset(pos, 0, sizeof *pos);
    pos->n = n;
    pos->bistatic = bistatic;
    pos->b = calloc(np, sizeof(double));
    pos->cose = calloc(np, sizeof(double));
    pos->cosi = calloc(np, sizeof(double));
    pos->z = calloc(np, sizeof(double));
    pos->f = calloc(np, sizeof(int));
    pos->cosill = calloc(np, sizeof(double));
    pos->zill = calloc(np, sizeof(double));
    pos->fill = calloc(np, sizeof(int));
    return (pos->b && pos->cose && pos->cosi && pos->z && pos->f && pos->cosill &&
            pos->zill && pos->fill) ? 0 : -1;
}

void orc_pos_free(orc_pos *pos)
{
    free(pos->b); free(pos->cose); free(pos->cosi); free(pos->z); free(pos->f);
    free(pos->cosill); free(pos->zill); free(pos->fill);
    memset(pos, 0, sizeof *pos);
}

/* posclr (src/shape/posclr.c:24-67). */
void orc_posclr(orc_pos *pos)
{
    int n = pos->n;
    size_t np = (size_t)(2 * n + 1) * (size_t)(2 * n + 1);
    for (size_t p = 0; p < np; p++) {
        pos->b[p] = pos->cose[p] = pos->cosi[p] = 0.0;
        pos->z[p] = -SHAPE_HUGENUMBER;
        pos->f[p] = -1;
    }
    pos->xlim[0] = pos->ylim[0] = n;
    pos->xlim[1] = pos->ylim[1] = -n;
    if (pos->bistatic) {
        for (size_t p = 0; p < np; p++) {
            pos->cosill[p] = 0.0;
            pos->zill[p] = -SHAPE_HUGENUMBER;
            pos->fill[p] = -1;
        }
        pos->xlim2[0] = pos->ylim2[0] = n;
        pos->xlim2[1] = pos->ylim2[1] = -n;
    }
}

/* ------------------------------------------------------------------- posvis */

typedef struct { double imin, imax, jmin, jmax; } orc_box;

static int orc_clamp_lo(double v) { return (v < INT_MIN) ? INT_MIN : (int)v; }
static int orc_clamp_hi(double v) { return (v > INT_MAX) ? INT_MAX : (int)v; }

/* POSrect (src/shape/posvis.c:322-364). */
static void orc_posrect(orc_pos *pos, int src, double imin_dbl, double imax_dbl,
                        double jmin_dbl, double jmax_dbl, orc_box *overall)
{
    overall->imin = ORC_MIN(overall->imin, imin_dbl);
    overall->imax = ORC_MAX(overall->imax, imax_dbl);
    overall->jmin = ORC_MIN(overall->jmin, jmin_dbl);
    overall->jmax = ORC_MAX(overall->jmax, jmax_dbl);
    int imin = orc_clamp_lo(imin_dbl), imax = orc_clamp_hi(imax_dbl);
    int jmin = orc_clamp_lo(jmin_dbl), jmax = orc_clamp_hi(jmax_dbl);
    int n = pos->n;
    int *xl = src ? pos->xlim2 : pos->xlim;
    int *yl = src ? pos->ylim2 : pos->ylim;
    if (imin < xl[0]) xl[0] = ORC_MAX(imin, -n);
    if (imax > xl[1]) xl[1] = ORC_MIN(imax, n);
    if (jmin < yl[0]) yl[0] = ORC_MAX(jmin, -n);
    if (jmax > yl[1]) yl[1] = ORC_MIN(jmax, n);
}

/* posvis (src/shape/posvis.c:84-317) for body 0, component 0. */
int orc_posvis(const orc_real *real, const double orbit_offset[3], orc_pos *pos,
               int smooth, int src)
{
    const int n = pos->n, side = 2 * n + 1;
    const double kmpp = pos->kmpp;
    double oa[9], usrc[3] = {0.0, 0.0, 1.0};
    double *cosa, *cosb, *zz;
    int *fac;
    int outbnd = 0;
    orc_box overall = {SHAPE_HUGENUMBER, -SHAPE_HUGENUMBER, SHAPE_HUGENUMBER, -SHAPE_HUGENUMBER};

    pos->posbnd_logfactor = 0.0;
    if (src) {
        orc_mul_bt(oa, pos->se, pos->ae);
        cosa = pos->cosill; cosb = NULL; zz = pos->zill; fac = pos->fill;
    } else {
        orc_mul_bt(oa, pos->oe, pos->ae);
        cosa = pos->cose; cosb = pos->cosi; zz = pos->z; fac = pos->f;
        if (pos->bistatic) {
            orc_mtv(usrc, pos->se, usrc);
            orc_mv(usrc, pos->oe, usrc);
        }
    }

    for (int f = 0; f < real->nf; f++) {
        double nrm[3], v0[3], v1[3], v2[3];
        const int *fv = real->fv + 3 * f;
        orc_mv(nrm, oa, real->fn + 3 * f);
        if (!(nrm[2] > 0.0))
            continue;
        orc_mv(v0, oa, real->x + 3 * fv[0]);
        orc_mv(v1, oa, real->x + 3 * fv[1]);
        orc_mv(v2, oa, real->x + 3 * fv[2]);
        for (int i = 0; i < 3; i++) {
            v0[i] += orbit_offset[i];
            v1[i] += orbit_offset[i];
            v2[i] += orbit_offset[i];
        }
        double imin_dbl = floor(ORC_MIN(v0[0], ORC_MIN(v1[0], v2[0])) / kmpp - SHAPE_SMALLVAL + 0.5);
        double imax_dbl = floor(ORC_MAX(v0[0], ORC_MAX(v1[0], v2[0])) / kmpp + SHAPE_SMALLVAL + 0.5);
        double jmin_dbl = floor(ORC_MIN(v0[1], ORC_MIN(v1[1], v2[1])) / kmpp - SHAPE_SMALLVAL + 0.5);
        double jmax_dbl = floor(ORC_MAX(v0[1], ORC_MAX(v1[1], v2[1])) / kmpp + SHAPE_SMALLVAL + 0.5);
        int imin = orc_clamp_lo(imin_dbl), imax = orc_clamp_hi(imax_dbl);
        int jmin = orc_clamp_lo(jmin_dbl), jmax = orc_clamp_hi(jmax_dbl);
        if (imin < -n || imax > n || jmin < -n || jmax > n)
            outbnd = 1;
        int i1 = ORC_MAX(imin, -n), i2 = ORC_MIN(imax, n);
        int j1 = ORC_MAX(jmin, -n), j2 = ORC_MIN(jmax, n);
        if (i1 > n || i2 < -n || j1 > n || j2 < -n) {
            orc_posrect(pos, src, imin_dbl, imax_dbl, jmin_dbl, jmax_dbl, &overall);
            continue;
        }
        for (int i = i1; i <= i2; i++) {
            double x0 = i * kmpp;
            for (int j = j1; j <= j2; j++) {
                double x1 = j * kmpp, den, s, t, z;
                s = ((x0 - v0[0]) * (v2[1] - v1[1]) - (v2[0] - v1[0]) * (x1 - v0[1]))
                    * (den = 1 / ((v1[0] - v0[0]) * (v2[1] - v1[1]) - (v2[0] - v1[0]) * (v1[1] - v0[1])));
                if (!((s >= -SHAPE_SMALLVAL) && (s <= 1.0 + SHAPE_SMALLVAL)))
                    continue;
                t = ((v1[0] - v0[0]) * (x1 - v0[1]) - (x0 - v0[0]) * (v1[1] - v0[1])) * den;
                if (!((t >= -SHAPE_SMALLVAL) && (t <= s + SHAPE_SMALLVAL)))
                    continue;
                z = v0[2] + s * (v1[2] - v0[2]) + t * (v2[2] - v1[2]);
                size_t p = (size_t)(i + n) * side + (size_t)(j + n);
                if (!((z > zz[p]) || (fac[p] < 0)))
                    continue;
                zz[p] = z;
                if (smooth) {
                    const double *n0 = real->vn + 3 * fv[0];
                    const double *n1 = real->vn + 3 * fv[1];
                    const double *n2 = real->vn + 3 * fv[2];
                    for (int k = 0; k < 3; k++)
                        nrm[k] = n0[k] + s * (n1[k] - n0[k]) + t * (n2[k] - n1[k]);
                    orc_mv(nrm, oa, nrm);
                    orc_normalize(nrm);
                }
                if (nrm[2] > 0.0) {
                    cosa[p] = nrm[2];
                    if (!src && pos->bistatic) {
                        cosb[p] = nrm[0] * usrc[0] + nrm[1] * usrc[1] + nrm[2] * usrc[2];
                        if (cosb[p] <= 0.0)
                            cosa[p] = 0.0;
                    }
                }
                orc_posrect(pos, src, (double)i, (double)i, (double)j, (double)j, &overall);
                fac[p] = f;
            }
        }
    }

    if (outbnd) {
        double xfactor = (ORC_MAX(overall.imax, n) - ORC_MIN(overall.imin, -n) + 1) / (2 * n + 1);
        double yfactor = (ORC_MAX(overall.jmax, n) - ORC_MIN(overall.jmin, -n) + 1) / (2 * n + 1);
        pos->posbnd_logfactor = log(xfactor * yfactor);
    }
    return outbnd;
}

/* ------------------------------------------------------------------ posmask */

/* iround (src/util/iround.c). */
static int orc_iround(double x) { return (x < 0.0) ? (int)(x - 0.5) : (int)(x + 0.5); }

/* posmask (src/shape/posmask.c:58-174), one body and one component. */
void orc_posmask(orc_pos *pos, double tol)
{
    const int n = pos->n, side = 2 * n + 1;
    const double bignum = 0.99 * SHAPE_HUGENUMBER;
    double so[9];
    orc_mul_bt(so, pos->se, pos->oe);
    const double pixels_per_km = 1 / pos->kmpp;
#define ZILL(a, b) pos->zill[(size_t)((a) + n) * side + (size_t)((b) + n)]
    for (int i = -n; i <= n; i++)
        for (int j = -n; j <= n; j++) {
            size_t p = (size_t)(i + n) * side + (size_t)(j + n);
            if (pos->cose[p] == 0.0)
                continue;
            double x[3] = {i * pos->kmpp, j * pos->kmpp, pos->z[p]};
            orc_mv(x, so, x);
            double i0 = x[0] * pixels_per_km, j0 = x[1] * pixels_per_km;
            int im = orc_iround(i0), jm = orc_iround(j0);
            if (!(fabs(i0) < n && fabs(j0) < n && ZILL(im, jm) > -bignum &&
                  pos->f[p] != pos->fill[(size_t)(im + n) * side + (size_t)(jm + n)]))
                continue;
            int i1 = (int)floor(i0), j1 = (int)floor(j0);
            double zill;
            if (ZILL(i1, j1) > -bignum && ZILL(i1 + 1, j1) > -bignum &&
                ZILL(i1, j1 + 1) > -bignum && ZILL(i1 + 1, j1 + 1) > -bignum) {
                double t = i0 - i1, u = j0 - j1;
                zill = (1 - t) * (1 - u) * ZILL(i1, j1) + t * (1 - u) * ZILL(i1 + 1, j1)
                       + t * u * ZILL(i1 + 1, j1 + 1) + (1 - t) * u * ZILL(i1, j1 + 1);
            } else {
                zill = ZILL(im, jm);
                int i_sign = (i0 >= im) ? 1 : -1;
                int i2 = im + i_sign;
                if (abs(i2) <= n && ZILL(i2, jm) > -bignum) {
                    zill += fabs(i0 - im) * (ZILL(i2, jm) - ZILL(im, jm));
                } else {
                    i2 = im - i_sign;
                    if (abs(i2) <= n && ZILL(i2, jm) > -bignum)
                        zill -= fabs(i0 - im) * (ZILL(i2, jm) - ZILL(im, jm));
                }
                int j_sign = (j0 >= jm) ? 1 : -1;
                int j2 = jm + j_sign;
                if (abs(j2) <= n && ZILL(im, j2) > -bignum) {
                    zill += fabs(j0 - jm) * (ZILL(im, j2) - ZILL(im, jm));
                } else {
                    j2 = jm - j_sign;
                    if (abs(j2) <= n && ZILL(im, j2) > -bignum)
                        zill -= fabs(j0 - jm) * (ZILL(im, j2) - ZILL(im, jm));
                }
            }
            if (zill - x[2] > tol)
                pos->cose[p] = 0.0;
        }
#undef ZILL
}

/* ------------------------------------------------------------------- radlaw */

/* radlaw (src/shape/radlaw.c:44-148) for the facet-independent laws. */
double orc_radlaw(const shape_radar_law *L, double c)
{
    double v = -9.99, tan2inc, sin2inc, arg;
    switch (L->type) {
    case SHAPE_RADLAW_COSINE_DIFF:
        v = L->diff_R * (L->diff_C + 1) * pow(c, 2 * L->diff_C - 1);
        break;
    case SHAPE_RADLAW_GAUSSIAN:
        if (c >= L->qs_cos_cutoff) {
            tan2inc = 1 / (c * c) - 1;
            v = L->qs_R * L->qs_C * exp(-L->qs_C * tan2inc) / (c * c * c * c * c);
        } else v = 0.0;
        break;
    case SHAPE_RADLAW_HAGFORS:
        if (c >= L->qs_cos_cutoff) {
            sin2inc = 1 - c * c;
            arg = c * c * c * c + L->qs_C * sin2inc;
            v = 0.5 * L->qs_R * L->qs_C * pow(arg, -1.5) / c;
        } else v = 0.0;
        break;
    case SHAPE_RADLAW_COSINE_QS:
        if (c >= L->qs_cos_cutoff)
            v = L->qs_R * (L->qs_C + 1) * pow(c, 2 * L->qs_C - 1);
        else v = 0.0;
        break;
    case SHAPE_RADLAW_GAUSSIAN_COSINE:
        v = L->diff_R * (L->diff_C + 1) * pow(c, 2 * L->diff_C - 1);
        if (c >= L->qs_cos_cutoff) {
            tan2inc = 1 / (c * c) - 1;
            v += L->qs_R * L->qs_C * exp(-L->qs_C * tan2inc) / (c * c * c * c * c);
        }
        break;
    case SHAPE_RADLAW_HAGFORS_COSINE:
        v = L->diff_R * (L->diff_C + 1) * pow(c, 2 * L->diff_C - 1);
        if (c >= L->qs_cos_cutoff) {
            sin2inc = 1 - c * c;
            arg = c * c * c * c + L->qs_C * sin2inc;
            v += 0.5 * L->qs_R * L->qs_C * pow(arg, -1.5) / c;
        }
        break;
    case SHAPE_RADLAW_COSINE_COSINE:
        v = L->diff_R * (L->diff_C + 1) * pow(c, 2 * L->diff_C - 1);
        if (c >= L->qs_cos_cutoff)
            v += L->qs_R * (L->qs_C + 1) * pow(c, 2 * L->qs_C - 1);
        break;
    default:
        break;
    }
    return v;
}

/* --------------------------------------------------------------- pos2deldop */

static double orc_sinc2(double x)
{
    double tmp = fabs(3.141592653589793 * x);
    if (tmp > 1.0e-4) {
        tmp = sin(tmp) / tmp;
        return tmp * tmp;
    }
    return 1.0;
}
static double orc_tri(double x) { double t = 1 - fabs(x); return t > 0.0 ? t : 0.0; }
static double orc_tri2(double x) { double t = 1 - fabs(x); return t > 0.0 ? t * t : 0.0; }

/* pos2deldop (src/shape/pos2deldop.c:176-581) for body 0, one view, no
 * orbital offsets. fit must be cleared by the caller (calc_fits.c:538). */
int orc_pos2deldop(const shape_eval_params *par, const shape_deldop_set *set,
                   const shape_deldop_frame *frm, const orc_pos *pos,
                   double *fit, shape_deldop_result *res)
{
    const int n = pos->n, side = 2 * n + 1;
    const int ndel = frm->ndel, ndop = frm->ndop;
    const int spb = set->spb, stride = set->stride, codemethod = set->codemethod;
    const int spb_over_stride = spb / stride;
    const double one_over_spb = 1.0 / spb;
    const int spb_sq = spb * spb;
    double const1, const2, w[3], del_c[SHAPE_MAXBINS], dop_c[SHAPE_MAXBINS + 1];
    int badradar = 0;

    res->idellim[0] = ndel + 999999; res->idellim[1] = -999999;
    res->idoplim[0] = ndop + 999999; res->idoplim[1] = -999999;
    res->dellim[0] = SHAPE_HUGENUMBER; res->dellim[1] = -SHAPE_HUGENUMBER;
    res->doplim[0] = SHAPE_HUGENUMBER; res->doplim[1] = -SHAPE_HUGENUMBER;
    res->badradar_logfactor = 0.0;

    if (codemethod != SHAPE_CODE_LONG_ORIG) {
        const1 = (3 * spb - 1) / (2.0 * stride);
        const2 = (spb - 1) / (2.0 * stride);
    } else {
        const1 = (double)spb_over_stride;
        const2 = 0.0;
    }
    const double delfact = -SHAPE_KM2US / set->del_per_pixel;
    orc_mv(w, frm->oe, frm->spin);
    const double dopfact = set->dopscale * SHAPE_KM2HZFACT * pos->kmpp * set->Ftx / set->dop_per_pixel;
    const double ax = -w[1] * dopfact;
    const double ay = w[0] * dopfact;
    const double km2Hz = sqrt(ax * ax + ay * ay) * set->dop_per_pixel / pos->kmpp;
    double dop_extra;
    if (w[0] != 0.0 || w[1] != 0.0)
        dop_extra = km2Hz * 0.5 * pos->kmpp * sqrt(w[0] * w[0] + w[1] * w[1]) / ORC_MAX(fabs(w[0]), fabs(w[1]));
    else
        dop_extra = 0.0;

    const int nsinc2 = par->nsinc2;
    const int nsinc2_sq = nsinc2 * nsinc2;
    const double xincr = ax / nsinc2, yincr = ay / nsinc2;
    const double dopdiff_bl = -(nsinc2 - 1) * (xincr + yincr) / 2;
    const double dopdiff_max = (nsinc2 - 1) * (fabs(xincr) + fabs(yincr)) / 2;
    if (2 * dopdiff_max + par->sinc2width + 1 > SHAPE_MAXBINS) {
        badradar = 1;
        res->badradar_logfactor += log((2 * dopdiff_max + par->sinc2width + 1) / SHAPE_MAXBINS);
    }
    const double delshift = frm->delcom_vig + frm->deloff;
    const double dopshift = frm->dopcom_vig + frm->dopoff;

    for (int x = pos->xlim[0]; x <= pos->xlim[1]; x++)
        for (int y = pos->ylim[0]; y <= pos->ylim[1]; y++) {
            size_t p = (size_t)(x + n) * side + (size_t)(y + n);
            if (!(pos->cose[p] > 0.0 && pos->f[p] >= 0 && pos->z[p] != -1e20))
                continue;
            double delPOS = pos->z[p] * delfact + delshift;
            int idel_min = (int)floor(delPOS - const1) + 1;
            int idel_max = (int)ceil(delPOS + const1) - 1;
            double dopPOS = ax * (x - 0.0) + ay * (y - 0.0) + dopshift;
            int idop_min = (int)floor(dopPOS - dopdiff_max + 1 - par->sinc2width / 2.0);
            int idop_max = (int)floor(dopPOS + dopdiff_max + par->sinc2width / 2.0);
            double codefactor = (codemethod == SHAPE_CODE_SHORT)
                                    ? orc_sinc2((dopPOS - frm->dopDC_vig) / set->dopfftlen) : 1.0;
            if (idel_min < res->idellim[0]) res->idellim[0] = idel_min;
            if (idel_max > res->idellim[1]) res->idellim[1] = idel_max;
            if (idop_min < res->idoplim[0]) res->idoplim[0] = idop_min;
            if (idop_max > res->idoplim[1]) res->idoplim[1] = idop_max;
            res->dellim[0] = ORC_MIN(res->dellim[0], delPOS);
            res->dellim[1] = ORC_MAX(res->dellim[1], delPOS);
            res->doplim[0] = ORC_MIN(res->doplim[0], dopPOS);
            res->doplim[1] = ORC_MAX(res->doplim[1], dopPOS);
            int in_bounds = (idel_min >= 1) && (idel_max <= ndel) && (idop_min >= 1) && (idop_max <= ndop);

            for (int idel = idel_min; idel <= idel_max; idel++) {
                double dc;
                if (codemethod != SHAPE_CODE_LONG_ORIG) {
                    if (spb == 1) {
                        dc = orc_tri2(delPOS - idel);
                    } else if (spb == 2) {
                        double arg = (delPOS - (idel - const2)) / spb_over_stride;
                        dc = orc_tri(arg) + orc_tri(arg - 0.5);
                        dc *= dc / 4;
                    } else {
                        dc = 0.0;
                        int m_min = ORC_MAX((int)floor((delPOS - idel - const2) * stride), 0);
                        int m_max = ORC_MIN((int)ceil((delPOS - idel + const1) * stride), spb) - 1;
                        double arg = (delPOS - (idel - const2)) / spb_over_stride - m_min * one_over_spb;
                        for (int m = m_min; m <= m_max; m++) {
                            dc += orc_tri(arg);
                            arg -= one_over_spb;
                        }
                        dc *= dc / spb_sq;
                    }
                } else {
                    dc = orc_tri2((delPOS - idel) / spb_over_stride);
                }
                del_c[idel - idel_min] = dc;
            }
            for (int idop = idop_min; idop <= idop_max; idop++) {
                double sm;
                if (nsinc2 == 1) {
                    sm = orc_sinc2(dopPOS - idop);
                } else if (nsinc2 == 2) {
                    double bl = dopPOS + dopdiff_bl - idop;
                    sm = (orc_sinc2(bl) + orc_sinc2(bl + xincr) + orc_sinc2(bl + yincr) +
                          orc_sinc2(bl + xincr + yincr)) / 4;
                } else {
                    double left = dopPOS + dopdiff_bl - idop;
                    sm = 0.0;
                    for (int i = 0; i < nsinc2; i++) {
                        double arg = left;
                        for (int j = 0; j < nsinc2; j++) {
                            sm += orc_sinc2(arg);
                            arg += xincr;
                        }
                        left += yincr;
                    }
                    sm /= nsinc2_sq;
                }
                dop_c[ORC_MIN(idop - idop_min, SHAPE_MAXBINS)] = sm;
            }
            double sumweights = 0.0;
            for (int idel = idel_min; idel <= idel_max; idel++)
                for (int idop = idop_min; idop <= idop_max; idop++)
                    sumweights += del_c[idel - idel_min] * dop_c[ORC_MIN(idop - idop_min, SHAPE_MAXBINS)];
            double amp = orc_radlaw(&set->law, pos->cose[p]) * pos->kmpp * pos->kmpp * codefactor / sumweights;
            if (in_bounds) {
                for (int idel = idel_min; idel <= idel_max; idel++)
                    for (int idop = idop_min; idop <= idop_max; idop++) {
                        double c = amp * del_c[idel - idel_min] * dop_c[ORC_MIN(idop - idop_min, SHAPE_MAXBINS)];
                        fit[(size_t)(idel - 1) * ndop + (size_t)(idop - 1)] += c;
                    }
            }
        }

    res->dellim[0] = (res->dellim[0] - delshift) * set->del_per_pixel;
    res->dellim[1] = (res->dellim[1] - delshift) * set->del_per_pixel;
    res->doplim[0] = (res->doplim[0] - dopshift) * set->dop_per_pixel - dop_extra;
    res->doplim[1] = (res->doplim[1] - dopshift) * set->dop_per_pixel + dop_extra;
    res->badradar = badradar;
    return badradar;
}

/* --------------------------------------------------------------- pos2doppler */

/* pos2doppler (src/shape/pos2doppler.c:149-501) for body 0, one view, no
 * orbital offsets, speckle off. fit (ndop) must be cleared by the caller
 * (src/shape/calc_fits.c:914). Pixels whose sinc^2 footprint leaves the
 * spectrum go to an overflow spectrum of ORC_MAXOVERFLOW bins centred on the
 * COM; ovf receives its chi-square terms {o2, m2, xsec, dopmean}
 * (pos2doppler.c:451-499). Returns badradar. */
#define ORC_MAXOVERFLOW 2000
int orc_pos2doppler(const shape_eval_params *par, const shape_doppler_set *set,
                    const shape_doppler_frame *frm, const orc_pos *pos, double *fit,
                    shape_deldop_result *res, double ovf[4])
{
    const int n = pos->n, side = 2 * n + 1, ndop = frm->ndop;
    double w[3], dop_c[SHAPE_MAXBINS + 1];
    int badradar = 0, any_overflow = 0, idop0 = 0;
    double *overflow = calloc(ORC_MAXOVERFLOW, sizeof(double));

    res->idellim[0] = res->idellim[1] = 0;
    res->dellim[0] = res->dellim[1] = 0.0;
    res->idoplim[0] = ndop + 999999; res->idoplim[1] = -999999;
    res->doplim[0] = SHAPE_HUGENUMBER; res->doplim[1] = -SHAPE_HUGENUMBER;
    res->badradar_logfactor = 0.0;

    orc_mv(w, frm->oe, frm->spin);
    const double dopfact = set->dopscale * SHAPE_KM2HZFACT * pos->kmpp * set->Ftx / set->dop_per_bin;
    const double ax = -w[1] * dopfact;
    const double ay = w[0] * dopfact;
    const double km2Hz = sqrt(ax * ax + ay * ay) * set->dop_per_bin / pos->kmpp;
    double dop_extra;
    if (w[0] != 0.0 || w[1] != 0.0)
        dop_extra = km2Hz * 0.5 * pos->kmpp * sqrt(w[0] * w[0] + w[1] * w[1]) / ORC_MAX(fabs(w[0]), fabs(w[1]));
    else
        dop_extra = 0.0;
    const int nsinc2 = par->nsinc2;
    const int nsinc2_sq = nsinc2 * nsinc2;
    const double xincr = ax / nsinc2, yincr = ay / nsinc2;
    const double dopdiff_bl = -(nsinc2 - 1) * (xincr + yincr) / 2;
    const double dopdiff_max = (nsinc2 - 1) * (fabs(xincr) + fabs(yincr)) / 2;
    if (2 * dopdiff_max + par->sinc2width + 1 > SHAPE_MAXBINS) {
        badradar = 1;
        res->badradar_logfactor += log((2 * dopdiff_max + par->sinc2width + 1) / SHAPE_MAXBINS);
    }
    const double dopshift = frm->dopcom_vig + frm->dopoff + 0.0;

    for (int x = pos->xlim[0]; x <= pos->xlim[1]; x++)
        for (int y = pos->ylim[0]; y <= pos->ylim[1]; y++) {
            size_t p = (size_t)(x + n) * side + (size_t)(y + n);
            if (!(pos->cose[p] > 0.0 && pos->f[p] >= 0))
                continue;
            double dopPOS = ax * (x - 0.0) + ay * (y - 0.0) + dopshift;
            int idop_min = (int)floor(dopPOS - dopdiff_max + 1 - par->sinc2width / 2.0);
            int idop_max = (int)floor(dopPOS + dopdiff_max + par->sinc2width / 2.0);
            if (idop_min < res->idoplim[0]) res->idoplim[0] = idop_min;
            if (idop_max > res->idoplim[1]) res->idoplim[1] = idop_max;
            res->doplim[0] = ORC_MIN(res->doplim[0], dopPOS);
            res->doplim[1] = ORC_MAX(res->doplim[1], dopPOS);
            int in_bounds = (idop_min >= 1) && (idop_max <= ndop);
            if (!in_bounds && !any_overflow) {
                any_overflow = 1;
                memset(overflow, 0, sizeof(double) * ORC_MAXOVERFLOW);
                idop0 = ORC_MAXOVERFLOW / 2 - (int)floor(dopshift + 0.5);
            }
            for (int idop = idop_min; idop <= idop_max; idop++) {
                double sm;
                if (nsinc2 == 1) {
                    sm = orc_sinc2(dopPOS - idop);
                } else if (nsinc2 == 2) {
                    double bl = dopPOS + dopdiff_bl - idop;
                    sm = (orc_sinc2(bl) + orc_sinc2(bl + xincr) + orc_sinc2(bl + yincr) +
                          orc_sinc2(bl + xincr + yincr)) / 4;
                } else {
                    double left = dopPOS + dopdiff_bl - idop;
                    sm = 0.0;
                    for (int i = 0; i < nsinc2; i++) {
                        double arg = left;
                        for (int j = 0; j < nsinc2; j++) {
                            sm += orc_sinc2(arg);
                            arg += xincr;
                        }
                        left += yincr;
                    }
                    sm /= nsinc2_sq;
                }
                dop_c[ORC_MIN(idop - idop_min, SHAPE_MAXBINS)] = sm;
            }
            double sumweights = 0.0;
            for (int idop = idop_min; idop <= idop_max; idop++)
                sumweights += dop_c[ORC_MIN(idop - idop_min, SHAPE_MAXBINS)];
            double amp = orc_radlaw(&set->law, pos->cose[p]) * pos->kmpp * pos->kmpp / sumweights;
            if (in_bounds) {
                for (int idop = idop_min; idop <= idop_max; idop++)
                    fit[idop - 1] += amp * dop_c[ORC_MIN(idop - idop_min, SHAPE_MAXBINS)];
            } else {
                int idop1 = ORC_MAX(idop_min, -idop0);
                int idop2 = ORC_MIN(idop_max, -idop0 + ORC_MAXOVERFLOW - 1);
                for (int idop = idop1; idop <= idop2; idop++)
                    overflow[idop + idop0] += amp * dop_c[ORC_MIN(idop - idop_min, SHAPE_MAXBINS)];
            }
        }

    res->doplim[0] = (res->doplim[0] - dopshift) * set->dop_per_bin - dop_extra;
    res->doplim[1] = (res->doplim[1] - dopshift) * set->dop_per_bin + dop_extra;

    const double variance = frm->sdev * frm->sdev;
    ovf[0] = ovf[1] = ovf[2] = ovf[3] = 0.0;
    if (any_overflow) {
        int j1 = ORC_MAX(res->idoplim[0] + idop0, 0);
        int j2 = ORC_MIN(res->idoplim[1] + idop0, ORC_MAXOVERFLOW - 1);
        for (int j = j1; j <= j2; j++)
            if (overflow[j] != 0.0) {
                ovf[0] += 1.0;
                ovf[1] += overflow[j] * overflow[j] / variance;
                ovf[2] += overflow[j];
                ovf[3] += (j - idop0) * overflow[j];
            }
        if (ovf[2] != 0.0)
            ovf[3] /= ovf[2];
        if ((res->idoplim[0] + idop0) < 0 || (res->idoplim[1] + idop0) >= ORC_MAXOVERFLOW) {
            badradar = 1;
            double dopfactor = (ORC_MAX(res->idoplim[1] + idop0, ORC_MAXOVERFLOW) -
                                ORC_MIN(res->idoplim[0] + idop0, 0)) / (1.0 * ORC_MAXOVERFLOW);
            res->badradar_logfactor += log(dopfactor);
        }
    }
    free(overflow);
    res->badradar = badradar;
    return badradar;
}

/* -------------------------------------------------------------- apply_photo */

/* apply_photo (src/shape/apply_photo.c:78-309) for the Lambert, Lommel and
 * Kaasalainen laws, body 0. */
double orc_apply_photo(const shape_optical_law *law, double phase,
                       double intensityfactor, orc_pos *pos)
{
    const int n = pos->n, side = 2 * n + 1;
    double sum = 0.0, scale = 0.0, s_ls = 0.0, s_l = 0.0;
    if (law->type == SHAPE_OPTLAW_LAMBERT) {
        scale = law->R / SHAPE_PIE;
    } else if (law->type == SHAPE_OPTLAW_LOMMEL) {
        scale = law->R / (4 * SHAPE_PIE);
    } else {
        double phasefunc = law->A0 * exp(-phase / law->D) + law->k * phase + 1;
        s_ls = (1 - law->wt) * phasefunc * law->R / (4 * SHAPE_PIE);
        s_l = law->wt * phasefunc * law->R / SHAPE_PIE;
    }
    for (int i = pos->xlim[0]; i <= pos->xlim[1]; i++)
        for (int j = pos->ylim[0]; j <= pos->ylim[1]; j++) {
            size_t p = (size_t)(i + n) * side + (size_t)(j + n);
            if (!(pos->cose[p] > 0.0 && pos->cosi[p] > 0.0 && pos->f[p] >= 0))
                continue;
            double b;
            if (law->type == SHAPE_OPTLAW_LAMBERT)
                b = intensityfactor * scale * pos->cosi[p];
            else if (law->type == SHAPE_OPTLAW_LOMMEL)
                b = intensityfactor * scale * pos->cosi[p] / (pos->cosi[p] + pos->cose[p]);
            else
                b = intensityfactor * pos->cosi[p] * (s_ls / (pos->cosi[p] + pos->cose[p]) + s_l);
            pos->b[p] = b;
            sum += b;
        }
    if (sum == 0.0)
        sum = 1.0e-40;
    return sum;
}

/* --------------------------------------------------------------------- chi2 */

/* One frame of chi2_deldop (src/shape/chi2.c:405-460), overflow terms zero
 * (pos2deldop.c:551-555); the same sums serve chi2_lghtcrv (chi2.c:1125-1170). */
void orc_chi2_frame(const double *obs, const double *oneovervar, const double *fit,
                    int npix, double weight, int cal_floating, double cal_in,
                    double *o2, double *m2, double *om, double *cal, double *chi2)
{
    double so2 = 0.0, sm2 = 0.0, som = 0.0;
    for (int p = 0; p < npix; p++) {
        so2 += obs[p] * obs[p] * oneovervar[p];
        sm2 += fit[p] * fit[p] * oneovervar[p];
        som += fit[p] * obs[p] * oneovervar[p];
    }
    double c = cal_in;
    if (cal_floating)
        c = (som > 0.0) ? som / sm2 : SHAPE_TINYCALFACT;
    *o2 = so2; *m2 = sm2; *om = som; *cal = c;
    *chi2 = weight * (so2 - 2 * c * som + c * c * sm2);
}

/* One frame of chi2_doppler (src/shape/chi2.c:722-780): the sums start from
 * the overflow spectrum's o2 and m2 (pos2doppler.c:451-499). */
void orc_chi2_doppler_frame(const double *obs, const double *oneovervar, const double *fit,
                            int ndop, double ovf_o2, double ovf_m2, double weight,
                            int cal_floating, double cal_in, double *o2, double *m2,
                            double *om, double *cal, double *chi2)
{
    double so2 = ovf_o2, sm2 = ovf_m2, som = 0.0;
    for (int j = 0; j < ndop; j++) {
        so2 += obs[j] * obs[j] * oneovervar[j];
        sm2 += fit[j] * fit[j] * oneovervar[j];
        som += fit[j] * obs[j] * oneovervar[j];
    }
    double c = cal_in;
    if (cal_floating)
        c = (som > 0.0) ? som / sm2 : SHAPE_TINYCALFACT;
    *o2 = so2; *m2 = sm2; *om = som; *cal = c;
    *chi2 = weight * (so2 - 2 * c * som + c * c * sm2);
}

/* --------------------------------------------------------------- composites */

void orc_deldop_frame(const shape_eval_params *par, const orc_real *real,
                      const shape_deldop_set *set, const shape_deldop_frame *frm,
                      const double *obs, const double *oneovervar,
                      orc_pos *pos, double *fit, unsigned char *seen,
                      shape_deldop_result *res)
{
    const double zero3[3] = {0.0, 0.0, 0.0};
    memcpy(pos->ae, frm->ae, sizeof pos->ae);
    memcpy(pos->oe, frm->oe, sizeof pos->oe);
    pos->kmpp = frm->km_per_pixel;
    pos->bistatic = 0;
    orc_posclr(pos);
    res->outbnd = orc_posvis(real, zero3, pos, par->pos_smooth, 0);
    res->posbnd_logfactor = pos->posbnd_logfactor;
    const int n = pos->n, side = 2 * n + 1;
    if (seen && par->mark_seen)
        for (int k = pos->xlim[0]; k <= pos->xlim[1]; k++)
            for (int l = pos->ylim[0]; l <= pos->ylim[1]; l++) {
                size_t p = (size_t)(k + n) * side + (size_t)(l + n);
                if (pos->cose[p] > par->mincosine_seen && pos->f[p] >= 0)
                    seen[pos->f[p]] = 1;
            }
    memset(fit, 0, sizeof(double) * (size_t)frm->ndel * (size_t)frm->ndop);
    orc_pos2deldop(par, set, frm, pos, fit, res);
    res->xlim[0] = pos->xlim[0]; res->xlim[1] = pos->xlim[1];
    res->ylim[0] = pos->ylim[0]; res->ylim[1] = pos->ylim[1];
    orc_chi2_frame(obs, oneovervar, fit, frm->ndel * frm->ndop, frm->weight,
                   frm->cal_floating, frm->cal, &res->o2, &res->m2, &res->om,
                   &res->cal, &res->chi2);
}

/* A smeared frame (src/shape/calc_fits.c:475-594): views[0..nviews-1] in
 * rendering order (v0+1 .. v0+nviews modulo nviews, the epoch view last),
 * each cleared, rendered by posvis and mapped by pos2deldop into its own fit;
 * the frame's fit is the sum over views divided by nviews (summed in view
 * order). posbnd, the seen marks and the limits are the epoch view's; each
 * view whose footprint is too wide adds dof * log-factor / nviews to
 * *badradar_term in view order, and sets *badradar_any. res holds the epoch
 * view's own flags and the chi-square of the mean fit. */
void orc_deldop_frame_views(const shape_eval_params *par, const orc_real *real,
                            const shape_deldop_set *set, int nviews, const shape_deldop_frame *views,
                            const double *obs, const double *oneovervar,
                            orc_pos *pos, double *fit, unsigned char *seen,
                            shape_deldop_result *res, int *badradar_any, double *badradar_term)
{
    const double zero3[3] = {0.0, 0.0, 0.0};
    const shape_deldop_frame *ep = &views[nviews - 1];
    const size_t D = (size_t)ep->ndel * (size_t)ep->ndop;
    double *store = calloc(D, sizeof(double));
    *badradar_any = 0;
    *badradar_term = 0.0;
    for (int k = 0; k < nviews; k++) {
        const shape_deldop_frame *V = &views[k];
        const int epoch = (k == nviews - 1);
        memcpy(pos->ae, V->ae, sizeof pos->ae);
        memcpy(pos->oe, V->oe, sizeof pos->oe);
        pos->kmpp = ep->km_per_pixel;
        pos->bistatic = 0;
        orc_posclr(pos);
        int ob = orc_posvis(real, zero3, pos, par->pos_smooth, 0);
        if (epoch) {
            res->outbnd = ob;
            res->posbnd_logfactor = pos->posbnd_logfactor;
        }
        const int n = pos->n, side = 2 * n + 1;
        if (epoch && seen && par->mark_seen)
            for (int i = pos->xlim[0]; i <= pos->xlim[1]; i++)
                for (int l = pos->ylim[0]; l <= pos->ylim[1]; l++) {
                    size_t p = (size_t)(i + n) * side + (size_t)(l + n);
                    if (pos->cose[p] > par->mincosine_seen && pos->f[p] >= 0)
                        seen[pos->f[p]] = 1;
                }
        /* the view's own fields with the frame's sizes and COM bins */
        shape_deldop_frame fv = *ep;
        memcpy(fv.ae, V->ae, sizeof fv.ae);
        memcpy(fv.oe, V->oe, sizeof fv.oe);
        memcpy(fv.spin, V->spin, sizeof fv.spin);
        fv.deloff = V->deloff;
        fv.dopoff = V->dopoff;
        shape_deldop_result rv = *res;
        memset(fit, 0, sizeof(double) * D);
        orc_pos2deldop(par, set, &fv, pos, fit, &rv);
        if (rv.badradar) {
            *badradar_any = 1;
            *badradar_term += ep->dof * rv.badradar_logfactor / nviews;
        }
        res->badradar = rv.badradar;
        res->badradar_logfactor = rv.badradar_logfactor;
        for (size_t i = 0; i < D; i++) store[i] += fit[i];
        if (epoch) {
            res->xlim[0] = pos->xlim[0]; res->xlim[1] = pos->xlim[1];
            res->ylim[0] = pos->ylim[0]; res->ylim[1] = pos->ylim[1];
            memcpy(res->idellim, rv.idellim, sizeof res->idellim);
            memcpy(res->idoplim, rv.idoplim, sizeof res->idoplim);
            memcpy(res->dellim, rv.dellim, sizeof res->dellim);
            memcpy(res->doplim, rv.doplim, sizeof res->doplim);
        }
    }
    for (size_t i = 0; i < D; i++) fit[i] = store[i] / nviews;
    free(store);
    orc_chi2_frame(obs, oneovervar, fit, ep->ndel * ep->ndop, ep->weight,
                   ep->cal_floating, ep->cal, &res->o2, &res->m2, &res->om,
                   &res->cal, &res->chi2);
}

/* calc_doppler for one frame (src/shape/calc_fits.c:860-935) then its chi2. */
void orc_doppler_frame(const shape_eval_params *par, const orc_real *real,
                       const shape_doppler_set *set, const shape_doppler_frame *frm,
                       const double *obs, const double *oneovervar,
                       orc_pos *pos, double *fit, unsigned char *seen,
                       shape_deldop_result *res)
{
    const double zero3[3] = {0.0, 0.0, 0.0};
    memcpy(pos->ae, frm->ae, sizeof pos->ae);
    memcpy(pos->oe, frm->oe, sizeof pos->oe);
    pos->kmpp = frm->km_per_pixel;
    pos->bistatic = 0;
    orc_posclr(pos);
    res->outbnd = orc_posvis(real, zero3, pos, par->pos_smooth, 0);
    res->posbnd_logfactor = pos->posbnd_logfactor;
    const int n = pos->n, side = 2 * n + 1;
    if (seen && par->mark_seen)
        for (int k = pos->xlim[0]; k <= pos->xlim[1]; k++)
            for (int l = pos->ylim[0]; l <= pos->ylim[1]; l++) {
                size_t p = (size_t)(k + n) * side + (size_t)(l + n);
                if (pos->cose[p] > par->mincosine_seen && pos->f[p] >= 0)
                    seen[pos->f[p]] = 1;
            }
    memset(fit, 0, sizeof(double) * (size_t)frm->ndop);
    double ovf[4];
    orc_pos2doppler(par, set, frm, pos, fit, res, ovf);
    res->xlim[0] = pos->xlim[0]; res->xlim[1] = pos->xlim[1];
    res->ylim[0] = pos->ylim[0]; res->ylim[1] = pos->ylim[1];
    orc_chi2_doppler_frame(obs, oneovervar, fit, frm->ndop, ovf[0], ovf[1], frm->weight,
                           frm->cal_floating, frm->cal, &res->o2, &res->m2, &res->om,
                           &res->cal, &res->chi2);
}

double orc_lghtcrv_point(const shape_eval_params *par, const orc_real *real,
                         const shape_optical_law *law, const shape_lghtcrv_point *pt,
                         orc_pos *pos, unsigned char *seen, int *outbnd,
                         double *outbnd_logsum)
{
    const double zero3[3] = {0.0, 0.0, 0.0};
    memcpy(pos->ae, pt->ae, sizeof pos->ae);
    memcpy(pos->oe, pt->oe, sizeof pos->oe);
    memcpy(pos->se, pt->se, sizeof pos->se);
    pos->kmpp = pt->km_per_pixel;
    pos->bistatic = 1;
    orc_posclr(pos);
    *outbnd = 0;
    *outbnd_logsum = 0.0;
    if (orc_posvis(real, zero3, pos, par->pos_smooth, 0)) {
        *outbnd = 1;
        *outbnd_logsum += 0.5 * pos->posbnd_logfactor;
    }
    if (orc_posvis(real, zero3, pos, 0, 1)) {
        *outbnd = 1;
        *outbnd_logsum += 0.5 * pos->posbnd_logfactor;
    }
    orc_posmask(pos, par->mask_tol);
    const int n = pos->n, side = 2 * n + 1;
    if (seen && par->mark_seen)
        for (int k = pos->xlim[0]; k <= pos->xlim[1]; k++)
            for (int l = pos->ylim[0]; l <= pos->ylim[1]; l++) {
                size_t p = (size_t)(k + n) * side + (size_t)(l + n);
                if (pos->cose[p] > par->mincosine_seen && pos->cosi[p] > par->mincosine_seen &&
                    pos->f[p] >= 0)
                    seen[pos->f[p]] = 1;
            }
    double intensityfactor = pow(pos->kmpp / SHAPE_AU, 2.0);
    return orc_apply_photo(law, pt->solar_phase, intensityfactor, pos);
}

/* ------------------------------------------------------------------- spline */

/* Natural cubic spline through (x[i], y[i]), i = 0..n-1: second derivatives
 * y2 with y2[0] = y2[n-1] = 0, from the tridiagonal system
 *   h[i-1] y2[i-1] + 2 (h[i-1] + h[i]) y2[i] + h[i] y2[i+1]
 *     = 6 ((y[i+1]-y[i])/h[i] - (y[i]-y[i-1])/h[i-1])
 * with each row divided by its span x[i+1] - x[i-1]: lower coefficient
 * w = h[i-1] / span, diagonal 2, upper 1 - w. Forward elimination keeps,
 * per row, the multiplier of y2[i+1] (stored in y2[i]) and the eliminated
 * right-hand side r[i]; back substitution then gives y2[i] = m[i] y2[i+1]
 * + r[i]. Solving the span-scaled rows in this order is how the reference
 * solves the system (spline(x, y, n, 2e30, 2e30, y2),
 * src/shape/calc_fits.c:1923), so the second derivatives and every fit
 * value are bit-identical to it. */
void orc_spline_natural(const double *x, const double *y, int n, double *y2)
{
    if (n < 1) return;
    double *r = malloc(sizeof(double) * (size_t)n);
    y2[0] = r[0] = 0.0;
    for (int i = 1; i < n - 1; i++) {
        const double span = x[i + 1] - x[i - 1];
        const double w = (x[i] - x[i - 1]) / span;
        const double piv = w * y2[i - 1] + 2.0;
        y2[i] = (w - 1.0) / piv;
        const double dslope = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
        r[i] = (6.0 * dslope / span - w * r[i - 1]) / piv;
    }
    if (n > 1) y2[n - 1] = 0.0;
    for (int i = n - 2; i >= 0; i--) y2[i] = y2[i] * y2[i + 1] + r[i];
    free(r);
}

/* Cubic spline evaluation at t: locate the bracketing knots by bisection
 * (a knot equal to t lands on the lower index, so t at a knot returns that
 * knot's y exactly) and evaluate the cubic in terms of the normalised
 * distances to both knots. This is the role of splint in
 * src/shape/calc_fits.c:1925-1933. */
double orc_splint(const double *x, const double *y, const double *y2, int n, double t)
{
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (x[mid] > t) hi = mid; else lo = mid;
    }
    double h = x[hi] - x[lo];
    double wl = (x[hi] - t) / h, wh = (t - x[lo]) / h;
    return wl * y[lo] + wh * y[hi] +
           ((wl * wl * wl - wl) * y2[lo] + (wh * wh * wh - wh) * y2[hi]) * (h * h) / 6.0;
}
