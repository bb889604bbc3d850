// dsmc_adjoint.h -- the smoothed timestep used for gradients and its hand-written adjoint.
//
// Gradient model.  The physical run (engine, hard energy knife) fixes every random choice: the
// collision events of each step (pair of atoms by id, scattering direction n^) are recorded and
// replayed.  In the smoothed model no atom is removed: each atom carries a survival weight w,
// multiplied every step by s = sigmoid((cut - e) / width), where e = v^2 + kappa (|B| - B_floor)
// is the knife energy in units of m/2, cut = 2 eta(step) kB T0 / m and width = 2 (width_kT) kB T0 / m.
// One step of one atom (after the recorded collisions of the step are applied):
//     v1 = v + dt/2 a(x),  x1 = x + dt v1,  v2 = v1 + dt/2 a(x1),  a = -(mu/m) grad|B|
//     e = |v2|^2 + kappa (|B(x1)| - B_floor),  w' = w sigmoid((cut - e)/width)
// Loss after the last step: L = (m/2) (sum w e / sum w) / (kB T0) + sum w / N0
// (final mean energy per retained atom in units of kB T0, plus the retained fraction).
// Parameters: B' (gradient), B0 (bias along z) of the linear trap B = (B'x/2, B'y/2, B0 - B'z),
// and the knot heights eta_k of the knife ramp.
//
// The adjoint is written out by hand: for the field of the linear trap, with J = diag(h, h, -B'),
// h = B'/2, b = B^/|B| the unit field:  grad|B| = J b,  Hessian H = J (I - b b^T) J / |B|,
// d|B|/dB' = b . (x/2, y/2, -z),  d|B|/dB0 = b_z,  d(grad|B|)/dtheta = dJ/dtheta b + J (I - b b^T) dB/dtheta / |B|.
// A collision with fixed n^ maps (vi, vj) to (c + r n^/2, c - r n^/2), c = (vi + vj)/2, r = |vi - vj|;
// its adjoint is  vi_bar = c_bar/2 + r_bar u/r,  vj_bar = c_bar/2 - r_bar u/r,  with
// c_bar = vi'_bar + vj'_bar, r_bar = n^ . (vi'_bar - vj'_bar)/2, u = vi - vj.
#ifndef DSMC_ADJOINT_H
#define DSMC_ADJOINT_H

#include "dsmc_physics.h"

namespace dsmc {

// number of differentiable parameters: B', B0, then the knife knots
constexpr int ADJ_NPARAM = 2 + 9;

template <class R> struct SmoothConsts {
    R Bp, B0, B_floor;
    R dt, half_dt, accel_scale, kappa;  // accel_scale = mu / m
    R inv_width;                        // 1 / width (v^2 units)
    double cut_scale;                   // d cut / d eta = 2 kB T0 / m
};

// field of the linear trap with its derivatives
template <class R> struct QuadField {
    R b[3];      // unit field
    R absB;
    R g[3];      // grad |B|
    R H[3][3];   // Hessian of |B|
    R dabs_dBp, dabs_dB0;
    R dg_dBp[3], dg_dB0[3];
};

template <class R>
DSMC_HD void quad_field(R Bp, R B0, R x, R y, R z, bool derivs, QuadField<R>& f) {
    const R h = R(0.5) * Bp;
    const R B[3] = {h * x, h * y, B0 - Bp * z};
    const R b2 = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
    R inv = R(0);
    if (b2 > R(0)) {
        inv = xrsqrt(b2);
        f.absB = b2 * inv;
        for (int i = 0; i < 3; ++i) f.b[i] = B[i] * inv;
    } else {
        f.absB = R(0);
        f.b[0] = R(0); f.b[1] = R(0); f.b[2] = R(1);
    }
    const R J[3] = {h, h, -Bp};
    for (int i = 0; i < 3; ++i) f.g[i] = J[i] * f.b[i];
    if (!derivs) return;
    // (I - b b^T) / |B|, zero where the field vanishes
    R P[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) P[i][j] = ((i == j ? R(1) : R(0)) - f.b[i] * f.b[j]) * inv;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) f.H[i][j] = J[i] * P[i][j] * J[j];
    const R q[3] = {R(0.5) * x, R(0.5) * y, -z};  // dB/dB'
    f.dabs_dBp = f.b[0] * q[0] + f.b[1] * q[1] + f.b[2] * q[2];
    f.dabs_dB0 = f.b[2];
    const R dJ[3] = {R(0.5), R(0.5), R(-1)};
    for (int i = 0; i < 3; ++i) {
        const R dbBp = P[i][0] * q[0] + P[i][1] * q[1] + P[i][2] * q[2];
        const R dbB0 = P[i][2];
        f.dg_dBp[i] = dJ[i] * f.b[i] + J[i] * dbBp;
        f.dg_dB0[i] = J[i] * dbB0;
    }
}

template <class R> DSMC_HD R sigmoid(R z) { return R(1) / (R(1) + xexp(-z)); }

// one smoothed step of one atom (collisions already applied to v); returns e
template <class R>
DSMC_HD R smooth_step(const SmoothConsts<R>& C, R cut, R* x, R* v, R& w) {
    QuadField<R> f0, f1;
    quad_field(C.Bp, C.B0, x[0], x[1], x[2], false, f0);
    const R as = -C.accel_scale;
    for (int i = 0; i < 3; ++i) v[i] = v[i] + C.half_dt * (as * f0.g[i]);
    for (int i = 0; i < 3; ++i) x[i] = x[i] + C.dt * v[i];
    quad_field(C.Bp, C.B0, x[0], x[1], x[2], false, f1);
    for (int i = 0; i < 3; ++i) v[i] = v[i] + C.half_dt * (as * f1.g[i]);
    const R e = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + C.kappa * (f1.absB - C.B_floor);
    w = w * sigmoid((cut - e) * C.inv_width);
    return e;
}

// Adjoint of smooth_step.  In: the state (x, v, w) the step started from (v after collisions),
// the adjoints xb, vb, wb of its outputs.  Out: xb, vb, wb overwritten with the adjoints of the
// inputs; theta_b[0..1] (B', B0) incremented; cut_b receives d/d cut.
template <class R>
DSMC_HD void smooth_step_adjoint(const SmoothConsts<R>& C, R cut, const R* x0, const R* v0, R w0, R* xb, R* vb,
                                 R& wb, R* theta_b, R& cut_b) {
    // recompute the forward intermediates
    QuadField<R> f0, f1;
    quad_field(C.Bp, C.B0, x0[0], x0[1], x0[2], true, f0);
    const R as = -C.accel_scale;
    R v1[3], x1[3], v2[3];
    for (int i = 0; i < 3; ++i) v1[i] = v0[i] + C.half_dt * (as * f0.g[i]);
    for (int i = 0; i < 3; ++i) x1[i] = x0[i] + C.dt * v1[i];
    quad_field(C.Bp, C.B0, x1[0], x1[1], x1[2], true, f1);
    for (int i = 0; i < 3; ++i) v2[i] = v1[i] + C.half_dt * (as * f1.g[i]);
    const R e = v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2] + C.kappa * (f1.absB - C.B_floor);
    const R s = sigmoid((cut - e) * C.inv_width);
    // w' = w s
    const R sb = wb * w0;
    wb = wb * s;
    const R zb = sb * s * (R(1) - s);
    const R eb = -zb * C.inv_width;
    cut_b = zb * C.inv_width;
    // e = |v2|^2 + kappa (|B(x1)| - B_floor)
    R v2b[3], x1b[3];
    for (int i = 0; i < 3; ++i) {
        v2b[i] = vb[i] + R(2) * eb * v2[i];
        x1b[i] = xb[i] + eb * C.kappa * f1.g[i];
    }
    theta_b[0] += eb * C.kappa * f1.dabs_dBp;
    theta_b[1] += eb * C.kappa * f1.dabs_dB0;
    // v2 = v1 + hdt as g(x1)
    R g1b[3];
    for (int i = 0; i < 3; ++i) g1b[i] = C.half_dt * as * v2b[i];
    for (int i = 0; i < 3; ++i) x1b[i] += f1.H[i][0] * g1b[0] + f1.H[i][1] * g1b[1] + f1.H[i][2] * g1b[2];
    theta_b[0] += f1.dg_dBp[0] * g1b[0] + f1.dg_dBp[1] * g1b[1] + f1.dg_dBp[2] * g1b[2];
    theta_b[1] += f1.dg_dB0[0] * g1b[0] + f1.dg_dB0[1] * g1b[1] + f1.dg_dB0[2] * g1b[2];
    // x1 = x0 + dt v1 ; v1 = v0 + hdt as g(x0)
    R v1b[3];
    for (int i = 0; i < 3; ++i) v1b[i] = v2b[i] + C.dt * x1b[i];
    R g0b[3];
    for (int i = 0; i < 3; ++i) g0b[i] = C.half_dt * as * v1b[i];
    for (int i = 0; i < 3; ++i) {
        xb[i] = x1b[i] + f0.H[i][0] * g0b[0] + f0.H[i][1] * g0b[1] + f0.H[i][2] * g0b[2];
        vb[i] = v1b[i];
    }
    theta_b[0] += f0.dg_dBp[0] * g0b[0] + f0.dg_dBp[1] * g0b[1] + f0.dg_dBp[2] * g0b[2];
    theta_b[1] += f0.dg_dB0[0] * g0b[0] + f0.dg_dB0[1] * g0b[1] + f0.dg_dB0[2] * g0b[2];
}

// collision of a recorded pair with fixed direction n (in place)
template <class R> DSMC_HD void collide_fixed(R* vi, R* vj, const R* n) {
    const R u0 = vi[0] - vj[0], u1 = vi[1] - vj[1], u2 = vi[2] - vj[2];
    const R r = xsqrt(u0 * u0 + u1 * u1 + u2 * u2);
    const R hr = R(0.5) * r;
    for (int k = 0; k < 3; ++k) {
        const R c = R(0.5) * (vi[k] + vj[k]);
        vi[k] = c + hr * n[k];
        vj[k] = c - hr * n[k];
    }
}

// adjoint of collide_fixed: pre-collision velocities vi, vj; adjoints of the outputs in vib, vjb,
// replaced by the adjoints of the inputs
template <class R> DSMC_HD void collide_fixed_adjoint(const R* vi, const R* vj, const R* n, R* vib, R* vjb) {
    const R u[3] = {vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]};
    const R r = xsqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const R rb = R(0.5) * (n[0] * (vib[0] - vjb[0]) + n[1] * (vib[1] - vjb[1]) + n[2] * (vib[2] - vjb[2]));
    const R k = r > R(0) ? rb / r : R(0);
    for (int a = 0; a < 3; ++a) {
        const R cb = vib[a] + vjb[a];
        vib[a] = R(0.5) * cb + k * u[a];
        vjb[a] = R(0.5) * cb - k * u[a];
    }
}

// knife ramp: eta(step) and the weights of the knots it interpolates
DSMC_HD double knot_weights(int nk, const double* ks, double step, int* k0, double* f) {
    if (nk <= 1 || step <= ks[0]) { *k0 = 0; *f = 0.0; return 0.0; }
    for (int i = 1; i < nk; ++i) {
        if (step <= ks[i]) {
            *k0 = i - 1;
            *f = (step - ks[i - 1]) / (ks[i] - ks[i - 1]);
            return *f;
        }
    }
    *k0 = nk - 1;
    *f = 0.0;
    return 0.0;
}

}  // namespace dsmc

#endif  // DSMC_ADJOINT_H
