// View geometry shared by the host (engine setup, the one-view operations)
// and the device (spin realization inside the evaluation graph): FP64 in
// the reference's operation order, so both give the same values (square
// roots are correctly rounded on both; the one log of a badradar view may
// differ in its last bit). Compile with FMA contraction off.
#pragma once

#include <cmath>
#include <cstring>

#include "engine_internal.h"
#include "kernels.h"

namespace shape {

// y = A x with A row-major (cotrans dir=1, src/util/cotrans.c)
__host__ __device__ inline void mv(double y[3], const double *A, const double x[3])
{
    double t[3];
    for (int i = 0; i < 3; i++) {
        t[i] = 0.0;
        for (int k = 0; k < 3; k++) t[i] += A[3 * i + k] * x[k];
    }
    y[0] = t[0]; y[1] = t[1]; y[2] = t[2];
}
// y = A^T x (cotrans dir=-1)
__host__ __device__ inline void mtv(double y[3], const double *A, const double x[3])
{
    double t[3];
    for (int i = 0; i < 3; i++) {
        t[i] = 0.0;
        for (int k = 0; k < 3; k++) t[i] += A[3 * k + i] * x[k];
    }
    y[0] = t[0]; y[1] = t[1]; y[2] = t[2];
}
// M = B * A^T (mtrnsps + mmmul as in src/shape/posvis.c:101-122)
__host__ __device__ inline void mul_bt(double *M, const double *B, const double *A)
{
    double t[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            t[3 * i + j] = 0.0;
            for (int k = 0; k < 3; k++) t[3 * i + j] += B[3 * i + k] * A[3 * j + k];
        }
    memcpy(M, t, sizeof t);
}

// View-dependent constants of radar frame F (src/shape/pos2deldop.c:218-275,
// src/shape/posvis.c:101-122): the observer <- body matrix, the Doppler
// axes and footprint extents, the delay and Doppler shifts and a Doppler
// spectrum's overflow origin; dx = the Doppler extent term of the frame's
// bin limits; the badradar flag and log-factor of a footprint wider than
// MAXBINS. g.nsinc2, g.sinc2width and g.dop1d must be set.
__host__ __device__ inline void radar_view_geom(FrameGeom &g, FrameHost &h, double &dx, const shape_deldop_frame &F,
                     const shape_deldop_set &S)
{
    mul_bt(g.oa, F.oe, F.ae);
    double w[3];
    mv(w, F.oe, F.spin);
    double dopfact = S.dopscale * SHAPE_KM2HZFACT * F.km_per_pixel * S.Ftx / S.dop_per_pixel;
    g.ax = -w[1] * dopfact;
    g.ay = w[0] * dopfact;
    double km2Hz = sqrt(g.ax * g.ax + g.ay * g.ay) * S.dop_per_pixel / F.km_per_pixel;
    dx = 0.0;
    if (w[0] != 0.0 || w[1] != 0.0)
        dx = km2Hz * 0.5 * F.km_per_pixel * sqrt(w[0] * w[0] + w[1] * w[1]) /
             (fabs(w[0]) < fabs(w[1]) ? fabs(w[1]) : fabs(w[0]));
    g.xincr = g.ax / g.nsinc2;
    g.yincr = g.ay / g.nsinc2;
    g.dopdiff_bl = -(g.nsinc2 - 1) * (g.xincr + g.yincr) / 2;
    g.dopdiff_max = (g.nsinc2 - 1) * (fabs(g.xincr) + fabs(g.yincr)) / 2;
    g.delshift = F.delcom_vig + F.deloff;
    g.dopshift = F.dopcom_vig + F.dopoff + 0.0;
    g.dopDC_vig = F.dopDC_vig;
    if (g.dop1d) g.idop0 = DOP_MAXOVERFLOW / 2 - (int)floor(g.dopshift + 0.5);
    h.badradar = 0;
    h.badradar_logfactor = 0.0;
    if (2 * g.dopdiff_max + g.sinc2width + 1 > SHAPE_MAXBINS) {
        h.badradar = 1;
        h.badradar_logfactor = log((2 * g.dopdiff_max + g.sinc2width + 1) / SHAPE_MAXBINS);
    }
}

// View-dependent constants of lightcurve point P (src/shape/calc_fits.c:
// 1634-1716): the observer and sun views' body matrices, the sun direction
// in observer coordinates and the observer -> sun transform of posmask.
__host__ __device__ inline void lc_view_geom(FrameGeom &go, FrameGeom &gs, LcPointDev &pd, const shape_lghtcrv_point &P)
{
    mul_bt(go.oa, P.oe, P.ae);
    double us[3] = {0.0, 0.0, 1.0};
    mtv(us, P.se, us);
    mv(us, P.oe, us);
    go.usrc[0] = us[0]; go.usrc[1] = us[1]; go.usrc[2] = us[2];
    mul_bt(gs.oa, P.se, P.ae);
    mul_bt(pd.so, P.se, P.oe);
}

// The float copies of a view's constants that the FP32 raster reads.
__host__ __device__ inline void view_float_consts(FrameGeom &g)
{
    const double fv[FDD_N] = {g.delfact, g.delshift, g.ax, g.ay, g.dopshift, g.const1, g.const2,
                              g.one_over_spb, g.xincr, g.yincr, g.dopdiff_bl, g.dopdiff_max,
                              g.dopDC_vig, g.dopfftlen, g.kmpp, g.sinc2width / 2.0,
                              (double)g.spb_over_stride, (double)g.stride, (double)g.spb_sq,
                              (double)g.nsinc2_sq};
    for (int k = 0; k < FDD_N; k++) g.fdd[k] = (float)fv[k];
    for (int k = 0; k < 9; k++) g.foa[k] = (float)g.oa[k];
    for (int k = 0; k < 3; k++) g.foa[9 + k] = (float)g.usrc[k];
}

}  // namespace shape
