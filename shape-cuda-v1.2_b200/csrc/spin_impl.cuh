// Principal-axis spin realization shared by the host (shape_realize_spin)
// and the device (the evaluation graph's view realization): realize_spin's
// per-view steps (src/shape/realize_spin.c:41-285) with inteuler's
// principal-axis branch (src/shape/inteuler.c) and euler2mat
// (src/util/euler.c), in the reference's operation order. The host's sin
// and cos are the C library's, as the reference's are; the device's are
// CUDA's (within a few units in the last place), so a device-realized view
// matches the host's to that rounding. Compile with FMA contraction off.
#pragma once

#include <cmath>

#include "shape_types.h"

namespace shape {

// Rotation from ecliptic to body axes for z-x-z Euler angles (phi, theta,
// psi): rows are the body axes in ecliptic coordinates.
__host__ __device__ inline void euler_zxz(double m[3][3], double phi, double theta, double psi)
{
    const double ct = cos(theta), st = sin(theta);
    const double cf = cos(phi), sf = sin(phi);
    const double cp = cos(psi), sp = sin(psi);
    m[0][0] = cp * cf - ct * sf * sp;
    m[1][0] = -sp * cf - ct * sf * cp;
    m[2][0] = st * sf;
    m[0][1] = cp * sf + ct * cf * sp;
    m[1][1] = -sp * sf + ct * cf * cp;
    m[2][1] = -st * cf;
    m[0][2] = sp * st;
    m[1][2] = cp * st;
    m[2][2] = ct;
}

// Epochs from t0 to t with the impulses met on the way (negated when t is
// before t0), as the reference lists them (realize_impulse).
__host__ __device__ inline int impulse_path(const shape_spin_state &sp, double t, double *te, double (*imp)[3])
{
    int k = 0;
    te[0] = sp.t0;
    imp[0][0] = imp[0][1] = imp[0][2] = 0.0;
    if (t >= sp.t0) {
        for (int n = 0; n < sp.n_impulse; n++)
            if (sp.t_impulse[n] > sp.t0 && sp.t_impulse[n] <= t) {
                k++;
                te[k] = sp.t_impulse[n];
                for (int j = 0; j < 3; j++) imp[k][j] = sp.impulse[n][j];
            }
        if (te[k] < t) {
            k++;
            te[k] = t;
            imp[k][0] = imp[k][1] = imp[k][2] = 0.0;
        }
    } else {
        for (int n = sp.n_impulse - 1; n >= 0; n--)
            if (sp.t_impulse[n] < sp.t0 && sp.t_impulse[n] >= t) {
                k++;
                te[k] = sp.t_impulse[n];
                for (int j = 0; j < 3; j++) imp[k][j] = -sp.impulse[n][j];
            }
        if (te[k] > t) {
            k++;
            te[k] = t;
            imp[k][0] = imp[k][1] = imp[k][2] = 0.0;
        }
    }
    return k + 1;
}

// Principal-axis kinematics from t0 to the last epoch of the impulse path:
// psi advances with the z spin, its drift and the libration; z impulses add
// to the rate from their epochs. m receives the ecliptic -> body matrix, w
// the body-frame spin.
__host__ __device__ inline void spin_pa_body(const shape_spin_state &sp, double phi, double theta, double psi0,
                                             const double *te, const double (*imp)[3], int ne, double m[3][3],
                                             double w[3])
{
    const double dt = te[ne - 1] - te[0];
    double psi = psi0 + sp.omega[2] * dt + 0.5 * sp.omegadot[2] * dt * dt +
                 sp.lib_amp * sin(sp.lib_freq * dt + sp.lib_phase);
    for (int i = 0; i < 2; i++) w[i] = sp.omega[i] + sp.omegadot[i] * dt;
    w[2] = sp.omega[2] + sp.omegadot[2] * dt + sp.lib_amp * sp.lib_freq * cos(sp.lib_freq * dt + sp.lib_phase);
    for (int k = 0; k < ne; k++) {
        psi += imp[k][2] * (te[ne - 1] - te[k]);
        w[2] += imp[k][2];
    }
    euler_zxz(m, phi, theta, psi);
}

// The dataset's spin offsets (body frame) added to w, then body -> ecliptic
// (the transpose of ae) plus the orbital contribution: ae (row-major) and
// the view's spin vector.
__host__ __device__ inline void spin_to_ecliptic(const double m[3][3], double w[3], const double omegaoff[3],
                                                 const double orbspin[3], double *ae, double *spin)
{
    for (int j = 0; j < 3; j++) w[j] += omegaoff[j];
    double e[3];
    for (int i = 0; i < 3; i++) {
        e[i] = 0.0;
        for (int j = 0; j < 3; j++) e[i] += m[j][i] * w[j];
    }
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) ae[3 * i + j] = m[i][j];
        spin[i] = orbspin[i] + e[i];
    }
}

// One view of a principal-axis rotator at epoch t: ae and the spin vector.
__host__ __device__ inline void realize_spin_pa(const shape_spin_state &sp, const double angleoff[3],
                                                const double omegaoff[3], double t, const double orbspin[3],
                                                double *ae, double *spin)
{
    const double phi = sp.angle[0] + angleoff[0], theta = sp.angle[1] + angleoff[1];
    const double psi0 = sp.angle[2] + angleoff[2];
    double te[SHAPE_MAX_IMPULSES + 2], imp[SHAPE_MAX_IMPULSES + 2][3];
    const int ne = impulse_path(sp, t, te, imp);
    double m[3][3], w[3];
    spin_pa_body(sp, phi, theta, psi0, te, imp, ne, m, w);
    spin_to_ecliptic(m, w, omegaoff, orbspin, ae, spin);
}

}  // namespace shape
