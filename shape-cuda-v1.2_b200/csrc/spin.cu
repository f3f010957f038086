// Spin realization of principal-axis rotators on the host: the per-view
// steps of realize_spin (src/shape/realize_spin.c:41-285) with inteuler's
// principal-axis branch (src/shape/inteuler.c:85-117) and euler2mat
// (src/util/euler.c). Each quantity is computed with the reference's
// operations in the reference's order, so the matrices and spin vectors
// are the reference's to the last bit.
#include <cmath>

#include "engine_impl.h"

namespace {

// Rotation from ecliptic to body axes for z-x-z Euler angles (phi, theta,
// psi): rows are the body axes in ecliptic coordinates.
void euler_zxz(double m[3][3], double phi, double theta, double psi)
{
    const double ct = std::cos(theta), st = std::sin(theta);
    const double cf = std::cos(phi), sf = std::sin(phi);
    const double cp = std::cos(psi), sp = std::sin(psi);
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
int impulse_path(const shape_spin_state &sp, double t, double *te, double (*imp)[3])
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

}  // namespace

extern "C" int shape_realize_spin(const shape_spin_state *spin, const double angleoff[3], const double omegaoff[3],
                                  int n, const double *t, const double *orbspin, double *ae, double *spin_out)
{
    if (!spin || !angleoff || !omegaoff || n < 0 || (n > 0 && (!t || !orbspin || !ae || !spin_out)))
        return shape::report_error(SHAPE_E_ARG, "realize_spin: null argument");
    if (spin->n_impulse < 0 || spin->n_impulse > SHAPE_MAX_IMPULSES)
        return shape::report_error(SHAPE_E_ARG, "realize_spin: more than SHAPE_MAX_IMPULSES impulses");
    if (!spin->pa)
        return shape::report_error(SHAPE_E_UNSUPPORTED, "realize_spin: non-principal-axis rotation");
    // the dataset's angle offsets are added to the model's Euler angles
    const double phi = spin->angle[0] + angleoff[0], theta = spin->angle[1] + angleoff[1];
    const double psi0 = spin->angle[2] + angleoff[2];
    for (int v = 0; v < n; v++) {
        double te[SHAPE_MAX_IMPULSES + 2], imp[SHAPE_MAX_IMPULSES + 2][3];
        const int ne = impulse_path(*spin, t[v], te, imp);
        const double dt = te[ne - 1] - te[0];
        // principal-axis kinematics: psi advances with the z spin, its drift
        // and the libration; z impulses add to the rate from their epochs
        double psi = psi0 + spin->omega[2] * dt + 0.5 * spin->omegadot[2] * dt * dt +
                     spin->lib_amp * std::sin(spin->lib_freq * dt + spin->lib_phase);
        double w[3];
        for (int i = 0; i < 2; i++) w[i] = spin->omega[i] + spin->omegadot[i] * dt;
        w[2] = spin->omega[2] + spin->omegadot[2] * dt +
               spin->lib_amp * spin->lib_freq * std::cos(spin->lib_freq * dt + spin->lib_phase);
        for (int k = 0; k < ne; k++) {
            psi += imp[k][2] * (te[ne - 1] - te[k]);
            w[2] += imp[k][2];
        }
        double m[3][3];
        euler_zxz(m, phi, theta, psi);
        // the dataset's spin offsets (body frame), then body -> ecliptic
        // (transpose of ae), plus the orbital contribution
        for (int j = 0; j < 3; j++) w[j] += omegaoff[j];
        double e[3];
        for (int i = 0; i < 3; i++) {
            e[i] = 0.0;
            for (int j = 0; j < 3; j++) e[i] += m[j][i] * w[j];
        }
        for (int i = 0; i < 3; i++) {
            for (int j = 0; j < 3; j++) ae[9 * (size_t)v + 3 * i + j] = m[i][j];
            spin_out[3 * (size_t)v + i] = orbspin[3 * (size_t)v + i] + e[i];
        }
    }
    return SHAPE_OK;
}
