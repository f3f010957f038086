// Spin realization on the host: the per-view steps of realize_spin
// (src/shape/realize_spin.c:41-285) with inteuler (src/shape/inteuler.c) and
// euler2mat (src/util/euler.c). Principal-axis rotators: each quantity is
// computed with the reference's operations in the reference's order, so the
// matrices and spin vectors are the reference's to the last bit.
// Non-principal-axis rotators: Euler's equations for the body-frame spin
// vector and the body-frame motion of the ecliptic axes, integrated between
// impulse epochs with an adaptive Dormand-Prince 5(4) method (Dormand and
// Prince 1980) to a relative error of 1e-13; the reference integrates the
// same equations with its own stepper, so values agree to that accuracy.
#include <cmath>

#include "engine_impl.h"
#include "spin_impl.cuh"

using shape::euler_zxz;
using shape::impulse_path;
using shape::spin_pa_body;
using shape::spin_to_ecliptic;

namespace {

// Torque-free rotation: y = (w in body coordinates, then the three ecliptic
// axes in body coordinates, the columns of ae). Euler's equations for w;
// each fixed axis a moves in the body frame as da/dt = a x w.
void npa_rhs(const double I[3], const double *y, double *dy)
{
    dy[0] = ((I[1] - I[2]) / I[0]) * y[1] * y[2];
    dy[1] = ((I[2] - I[0]) / I[1]) * y[2] * y[0];
    dy[2] = ((I[0] - I[1]) / I[2]) * y[0] * y[1];
    for (int c = 3; c < 12; c += 3) {
        dy[c + 0] = y[c + 1] * y[2] - y[c + 2] * y[1];
        dy[c + 1] = y[c + 2] * y[0] - y[c + 0] * y[2];
        dy[c + 2] = y[c + 0] * y[1] - y[c + 1] * y[0];
    }
}

// Integrates y from ta to tb (either direction) with the Dormand-Prince
// 5(4) pair and step-size control on the local error estimate. Time runs
// from 0 to tb - ta (exact for epochs within a factor of two of each
// other): stepping the absolute epoch (~2.5e6 days, ulp ~5e-10 day) would
// drift the integrated span by the rounding of every step. Returns false if
// it takes more than a bounded number of steps.
bool npa_integrate(const double I[3], double *y, double ta, double tb)
{
    // stage weights (the right-hand side does not depend on time, so the
    // stage nodes are not needed)
    static const double a21 = 1.0 / 5;
    static const double a31 = 3.0 / 40, a32 = 9.0 / 40;
    static const double a41 = 44.0 / 45, a42 = -56.0 / 15, a43 = 32.0 / 9;
    static const double a51 = 19372.0 / 6561, a52 = -25360.0 / 2187, a53 = 64448.0 / 6561, a54 = -212.0 / 729;
    static const double a61 = 9017.0 / 3168, a62 = -355.0 / 33, a63 = 46732.0 / 5247, a64 = 49.0 / 176,
                        a65 = -5103.0 / 18656;
    static const double b1 = 35.0 / 384, b3 = 500.0 / 1113, b4 = 125.0 / 192, b5 = -2187.0 / 6784,
                        b6 = 11.0 / 84;
    // differences of the fifth- and fourth-order weights (error estimate)
    static const double e1 = 35.0 / 384 - 5179.0 / 57600, e3 = 500.0 / 1113 - 7571.0 / 16695,
                        e4 = 125.0 / 192 - 393.0 / 640, e5 = -2187.0 / 6784 + 92097.0 / 339200,
                        e6 = 11.0 / 84 - 187.0 / 2100, e7 = -1.0 / 40;
    const double tol = 1e-13, span = tb - ta;
    if (span == 0.0) return true;
    const double dir = span > 0 ? 1.0 : -1.0;
    double t = 0.0, h = dir * std::fmin(std::fabs(span), 1e-3);
    double k1[12], k2[12], k3[12], k4[12], k5[12], k6[12], k7[12], yt[12], yn[12];
    npa_rhs(I, y, k1);
    for (long it = 0; it < 50000000L; it++) {
        if (dir * (t + h - span) > 0) h = span - t;
        for (int i = 0; i < 12; i++) yt[i] = y[i] + h * a21 * k1[i];
        npa_rhs(I, yt, k2);
        for (int i = 0; i < 12; i++) yt[i] = y[i] + h * (a31 * k1[i] + a32 * k2[i]);
        npa_rhs(I, yt, k3);
        for (int i = 0; i < 12; i++) yt[i] = y[i] + h * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
        npa_rhs(I, yt, k4);
        for (int i = 0; i < 12; i++) yt[i] = y[i] + h * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
        npa_rhs(I, yt, k5);
        for (int i = 0; i < 12; i++)
            yt[i] = y[i] + h * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
        npa_rhs(I, yt, k6);
        for (int i = 0; i < 12; i++)
            yn[i] = y[i] + h * (b1 * k1[i] + b3 * k3[i] + b4 * k4[i] + b5 * k5[i] + b6 * k6[i]);
        npa_rhs(I, yn, k7);
        // error relative to the spin magnitude (w) and to 1 (unit axes)
        const double wmag = std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]) + 1e-300;
        double err = 0.0;
        for (int i = 0; i < 12; i++) {
            const double ei = h * (e1 * k1[i] + e3 * k3[i] + e4 * k4[i] + e5 * k5[i] + e6 * k6[i] + e7 * k7[i]);
            const double sc = tol * (i < 3 ? wmag : 1.0);
            err = std::fmax(err, std::fabs(ei) / sc);
        }
        if (err <= 1.0) {
            t += h;
            for (int i = 0; i < 12; i++) { y[i] = yn[i]; k1[i] = k7[i]; }
            if (dir * (t - span) >= 0) return true;
        }
        const double f = (err == 0.0) ? 5.0 : std::fmin(5.0, std::fmax(0.2, 0.9 * std::pow(err, -0.2)));
        h *= f;
    }
    return false;
}

}  // namespace

extern "C" int shape_realize_spin(const shape_spin_state *spin, const double angleoff[3], const double omegaoff[3],
                                  int n, const double *t, const double *orbspin, double *ae, double *spin_out)
{
    if (!spin || !angleoff || !omegaoff || n < 0 || (n > 0 && (!t || !orbspin || !ae || !spin_out)))
        return shape::report_error(SHAPE_E_ARG, "realize_spin: null argument");
    if (spin->n_impulse < 0 || spin->n_impulse > SHAPE_MAX_IMPULSES)
        return shape::report_error(SHAPE_E_ARG, "realize_spin: more than SHAPE_MAX_IMPULSES impulses");
    if (!spin->pa && !(spin->inertia[0] > 0.0 && spin->inertia[1] > 0.0 && spin->inertia[2] > 0.0))
        return shape::report_error(SHAPE_E_ARG, "realize_spin: non-positive moment of inertia");
    // the dataset's angle offsets are added to the model's Euler angles
    const double phi = spin->angle[0] + angleoff[0], theta = spin->angle[1] + angleoff[1];
    const double psi0 = spin->angle[2] + angleoff[2];
    for (int v = 0; v < n; v++) {
        double te[SHAPE_MAX_IMPULSES + 2], imp[SHAPE_MAX_IMPULSES + 2][3];
        const int ne = impulse_path(*spin, t[v], te, imp);
        double m[3][3], w[3];
        if (!spin->pa) {
            // non-principal-axis: integrate from t0 one impulse interval at a
            // time (intervals shorter than 1e-6 day are skipped, as the
            // reference does), adding each impulse after its interval
            euler_zxz(m, phi, theta, psi0);
            double y[12];
            for (int j = 0; j < 3; j++) y[j] = spin->omega[j];
            for (int j = 0; j < 3; j++)
                for (int i = 0; i < 3; i++) y[3 + 3 * j + i] = m[i][j];
            for (int k = 0; k + 1 < ne; k++) {
                if (std::fabs(te[k + 1] - te[k]) >= 1.0e-6 &&
                    !npa_integrate(spin->inertia, y, te[k], te[k + 1]))
                    return shape::report_error(SHAPE_E_STATE, "realize_spin: integration did not converge");
                for (int j = 0; j < 3; j++) y[j] += imp[k + 1][j];
            }
            for (int j = 0; j < 3; j++) w[j] = y[j];
            for (int j = 0; j < 3; j++)
                for (int i = 0; i < 3; i++) m[i][j] = y[3 + 3 * j + i];
        } else {
            spin_pa_body(*spin, phi, theta, psi0, te, imp, ne, m, w);
        }
        spin_to_ecliptic(m, w, omegaoff, &orbspin[3 * (size_t)v], &ae[9 * (size_t)v], &spin_out[3 * (size_t)v]);
    }
    return SHAPE_OK;
}

namespace {

// Unit vector in place (normalize, src/util/normalize.c): divided by its
// length unless that is zero.
void unit(double u[3])
{
    double norm = 0.0;
    for (int i = 0; i < 3; i++) norm += u[i] * u[i];
    norm = std::sqrt(norm);
    if (norm != 0.0)
        for (int i = 0; i < 3; i++) u[i] /= norm;
}

void cross3(double z[3], const double x[3], const double y[3])
{
    const double a = x[1] * y[2] - x[2] * y[1], b = x[2] * y[0] - x[0] * y[2], c = x[0] * y[1] - x[1] * y[0];
    z[0] = a; z[1] = b; z[2] = c;
}

// Equatorial -> ecliptic (J2000 obliquity; the cosine and sine of
// src/astro/eq2ec.c).
void eq_to_ecl(double u[3])
{
    const double COSEPS = 0.9174821430652418, SINEPS = 0.3977769691126060;
    const double tmp = u[1] * COSEPS + u[2] * SINEPS;
    u[2] = u[2] * COSEPS - u[1] * SINEPS;
    u[1] = tmp;
}

// Linear interpolation of an ephemeris at t: RA (across the 0/360 line),
// Dec and distance with their rates; false if t is outside the table.
bool interpolate(const shape_ephem_point *e, int n, double t, double *ra, double *dec, double *dist,
                 double *rarate, double *decrate)
{
    const double PIE = 3.141592653589793;
    if (n < 2 || e[0].t > t) return false;
    int i = 0;
    while (e[i + 1].t < t) {
        ++i;
        if (i == n - 1) return false;
    }
    const double Dt = e[i + 1].t - e[i].t, dt = t - e[i].t;
    const double delta_ra = e[i + 1].ra - e[i].ra, twopi = 2 * PIE;
    if (delta_ra > PIE)
        *rarate = (e[i + 1].ra - (e[i].ra + twopi)) / Dt;
    else if (delta_ra < -PIE)
        *rarate = ((e[i + 1].ra + twopi) - e[i].ra) / Dt;
    else
        *rarate = (e[i + 1].ra - e[i].ra) / Dt;
    *ra = e[i].ra + *rarate * dt;
    *ra = *ra - twopi * floor(*ra / twopi);
    *decrate = (e[i + 1].dec - e[i].dec) / Dt;
    *dec = e[i].dec + *decrate * dt;
    const double distrate = (e[i + 1].dist - e[i].dist) / Dt;
    *dist = e[i].dist + distrate * dt;
    return true;
}

}  // namespace

extern "C" int shape_ephem_view(const shape_ephem_point *ast, int nast, const shape_ephem_point *sun, int nsun,
                                double t, double oe_out[9], double se_out[9], double s[3], double *solar_phase,
                                double *solar_azimuth, double *dist)
{
    const double PIE = 3.141592653589793;
    if (!ast || !oe_out || !s || !solar_phase || !solar_azimuth || !dist || (sun && !se_out))
        return shape::report_error(SHAPE_E_ARG, "ephem_view: null argument");
    double ra, dec, rarate, decrate;
    if (!interpolate(ast, nast, t, &ra, &dec, dist, &rarate, &decrate))
        return shape::report_error(SHAPE_E_ARG, "ephem_view: epoch outside the asteroid ephemeris");
    // observer axes: z toward the observer, x along -RA (pole x z), y = z x x
    double oe[3][3], ee[3], edot[3];
    oe[2][0] = -cos(dec) * cos(ra);
    oe[2][1] = -cos(dec) * sin(ra);
    oe[2][2] = -sin(dec);
    for (int i = 0; i < 3; i++) ee[i] = oe[2][i] * *dist;
    oe[0][0] = -oe[2][1];
    oe[0][1] = oe[2][0];
    oe[0][2] = 0.0;
    unit(oe[0]);
    cross3(oe[1], oe[2], oe[0]);
    for (int i = 0; i < 3; i++) eq_to_ecl(oe[i]);
    // plane-of-sky motion's contribution to the apparent spin: edot x z
    edot[0] = decrate * sin(dec) * cos(ra) + rarate * cos(dec) * sin(ra);
    edot[1] = decrate * sin(dec) * sin(ra) - rarate * cos(dec) * cos(ra);
    edot[2] = -decrate * cos(dec);
    eq_to_ecl(edot);
    cross3(s, edot, oe[2]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) oe_out[3 * i + j] = oe[i][j];
    if (!sun) {
        *solar_phase = 0.0;
        *solar_azimuth = 0.0;
        return SHAPE_OK;
    }
    double ra_s, dec_s, dist_s, rr, dr;
    if (!interpolate(sun, nsun, t, &ra_s, &dec_s, &dist_s, &rr, &dr))
        return shape::report_error(SHAPE_E_ARG, "ephem_view: epoch outside the solar ephemeris");
    double ss[3] = {cos(dec_s) * cos(ra_s) * dist_s, cos(dec_s) * sin(ra_s) * dist_s, sin(dec_s) * dist_s};
    for (int i = 0; i < 3; i++) ss[i] = ss[i] + ee[i];   // asteroid -> Sun
    eq_to_ecl(ss);
    unit(ss);
    const double theta = acos(ss[2]), phi = atan2(ss[1], ss[0]) + PIE / 2;
    double se[3][3];
    euler_zxz(se, phi, theta, 0.0);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) se_out[3 * i + j] = se[i][j];
    double so[3];
    for (int i = 0; i < 3; i++) {
        so[i] = 0.0;
        for (int j = 0; j < 3; j++) so[i] += oe[i][j] * ss[j];
    }
    unit(so);
    *solar_phase = acos(so[2]);
    if (so[0] == 0.0 && so[1] == 0.0) {
        *solar_azimuth = 0.0;
    } else {
        *solar_azimuth = atan2(so[1], so[0]) - PIE / 2;
        if (*solar_azimuth < 0.0) *solar_azimuth += 2 * PIE;
    }
    return SHAPE_OK;
}

// A radar view's epoch and geometry as read_deldop / read_doppler set them
// (src/shape/read_dat.c:866-900): the ephemeris at the uncorrected epoch
// gives the distance; with light-time correction the one-way light time
// (DAYSPERAU = 5.775518328e-3 day per AU, src/shape/const.h) is taken off
// the epoch and the ephemeris evaluated again there.
extern "C" int shape_ephem_radar_view(const shape_ephem_point *ast, int nast, double t_obs, int perform_ltc,
                                      double *t_view, double oe[9], double orbspin[3])
{
    if (!t_view) return shape::report_error(SHAPE_E_ARG, "ephem_radar_view: null argument");
    double ph, az, dist;
    *t_view = t_obs;
    int rc = shape_ephem_view(ast, nast, nullptr, 0, *t_view, oe, nullptr, orbspin, &ph, &az, &dist);
    if (rc || !perform_ltc) return rc;
    *t_view -= 5.775518328e-3 * dist;
    return shape_ephem_view(ast, nast, nullptr, 0, *t_view, oe, nullptr, orbspin, &ph, &az, &dist);
}

// Delay and Doppler offsets of a view from its dataset's delay-correction
// polynomial (deldopoffs, src/shape/deldopoffs.c:17-42): delay (usec)
// a0 + sum a_n (t - t0)^n in bins of del_per_pixel, and its rate (usec/day)
// as a Doppler offset -rate Ftx / (dop_per_pixel 86400) in bins.
extern "C" int shape_delcor_offsets(const double *a, int n, double t0, double t_view, double del_per_pixel,
                                    double dop_per_pixel, double Ftx, double *deloff, double *dopoff)
{
    if (!a || n < 0 || !deloff || !dopoff || !(del_per_pixel != 0.0) || !(dop_per_pixel != 0.0))
        return shape::report_error(SHAPE_E_ARG, "delcor_offsets: invalid argument");
    double x = 1.0, dop = 0.0, del = a[0];
    const double arg = t_view - t0;
    for (int k = 1; k <= n; k++) {
        dop += k * a[k] * x;
        del += a[k] * (x *= arg);
    }
    *deloff = del / del_per_pixel;
    *dopoff = -dop * Ftx / (dop_per_pixel * 86400.0);
    return SHAPE_OK;
}

namespace shape {

__global__ void k_realize_views(SpinRealizeArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const SpinViewSrc v = a.src[i];
    const double *ao = a.off + 6 * (size_t)v.rec, *oo = ao + 3;
    if (v.kind == 0) {
        shape_deldop_frame F = a.frames[v.index];
        realize_spin_pa(*a.spin, ao, oo, v.t, v.orb, F.ae, F.spin);
        for (int k = 0; k < 9; k++) a.frames[v.index].ae[k] = F.ae[k];
        for (int k = 0; k < 3; k++) a.frames[v.index].spin[k] = F.spin[k];
        FrameHost h = a.fh[v.index];
        FrameGeom g = a.geoms[h.view];
        double dx;
        radar_view_geom(g, h, dx, F, a.ddsets[v.dd]);
        view_float_consts(g);
        a.geoms[h.view] = g;
        a.fh[v.index] = h;
        a.dop_extra[v.index] = dx;
    } else {
        shape_lghtcrv_point P = a.points[v.index];
        const double zero[3] = {0.0, 0.0, 0.0};
        double unused[3];
        realize_spin_pa(*a.spin, ao, oo, v.t, zero, P.ae, unused);
        for (int k = 0; k < 9; k++) a.points[v.index].ae[k] = P.ae[k];
        LcPointDev pd = a.lcpts[v.index];
        FrameGeom go = a.geoms[pd.obs_view], gs = a.geoms[pd.sun_view];
        lc_view_geom(go, gs, pd, P);
        view_float_consts(go);
        view_float_consts(gs);
        a.geoms[pd.obs_view] = go;
        a.geoms[pd.sun_view] = gs;
        a.lcpts[v.index] = pd;
    }
}

void launch_realize_views(const SpinRealizeArgs &a, cudaStream_t s)
{
    if (a.n <= 0) return;
    k_realize_views<<<(a.n + 63) / 64, 64, 0, s>>>(a);
}

}  // namespace shape
