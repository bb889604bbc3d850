// dsmc_adjoint.h -- the smoothed timestep used for gradients and its hand-written adjoint.
//
// Gradient model.  The physical run (engine, hard Majorana and energy cuts) fixes every random
// choice: the collision events of each step (pair of atoms by id, scattering direction n^) are
// recorded and replayed.  In the smoothed model no atom is removed: each atom carries a survival
// weight w, multiplied every step by the knife's s_K = sigmoid((cut - e) / width) -- e = v^2 +
// kappa (|B| - B_floor) the knife energy in units of m/2, cut = 2 eta(step) kB T0 / m, width =
// 2 (width_kT) kB T0 / m -- and, when the run has Majorana loss, by s_M = sigmoid(<s.B^> / width_M)
// in place of the hard test <s.B^> < 0 (evaporation.cu:86-95).  One step of one atom (after the
// recorded collisions of the step are applied), in the order of the engine's step:
//     psi1 = [cos t - i sin t (s.B^(x))] psi,  t = (mu dt / hbar) |B(x)|   (wavefunction.cu:39-73)
//     v1 = v + dt/2 a(x),  x1 = x + dt v1,  v2 = v1 + dt/2 a(x1),  a = -(mu/m) grad|B|
//     e = |v2|^2 + kappa (|B(x1)| - B_floor),  w' = w s_K(e) s_M(<s.B^(x1)>_psi1)
// (the rotation is unitary, so the engine's renormalisation, which only removes rounding, is left
// out).  Loss after the last step: L = L_E + L_N with L_E = (m/2) (sum w e / sum w) / (kB T0) (the
// final mean energy per retained atom in units of kB T0) and L_N = sum w / N0 (the retained
// fraction); the adjoint carries both seeds at once and returns dL_E/dtheta and dL_N/dtheta.
// Parameters: B' (gradient), B0 (bias along z) of the linear trap B = (B'x/2, B'y/2, B0 - B'z),
// and the knot heights eta_k of the knife ramp.
//
// The adjoint is written out by hand: for the field of the linear trap, with J = diag(h, h, -B'),
// h = B'/2, b = B^/|B| the unit field:  grad|B| = J b,  Hessian H = J (I - b b^T) J / |B|,
// d|B|/dB' = b . (x/2, y/2, -z),  d|B|/dB0 = b_z,  d(grad|B|)/dtheta = dJ/dtheta b + J (I - b b^T) dB/dtheta / |B|;
// an adjoint (b_bar, |B|_bar) of the unit field and the magnitude pulls back to the field vector as
// B_bar = (I - b b^T) b_bar / |B| + b |B|_bar, then to x (J B_bar), B' ((x/2, y/2, -z) . B_bar) and
// B0 (B_bar_z).  The rotation psi1 = c psi + s T(b) psi (T linear in b and in psi) has the adjoint
// psi_bar = c psi1_bar + s T(b)^T psi1_bar, t_bar = -s (psi1_bar . psi) + c (psi1_bar . T(b) psi),
// b_bar_k = s psi1_bar . T(e_k) psi.  A collision with fixed n^ maps (vi, vj) to
// (c + r n^/2, c - r n^/2), c = (vi + vj)/2, r = |vi - vj|; its adjoint is
// vi_bar = c_bar/2 + r_bar u/r,  vj_bar = c_bar/2 - r_bar u/r,  with
// c_bar = vi'_bar + vj'_bar, r_bar = n^ . (vi'_bar - vj'_bar)/2, u = vi - vj.
#ifndef DSMC_ADJOINT_H
#define DSMC_ADJOINT_H

#include "dsmc_physics.h"

namespace dsmc {

// number of differentiable parameters: B', B0, then the knife knots
constexpr int ADJ_NPARAM = 2 + 9;

// adjoint seeds carried together: 0 = the mean energy term L_E, 1 = the retained fraction L_N
constexpr int ADJ_SEEDS = 2;

template <class R> struct SmoothConsts {
    R Bp, B0, B_floor;
    R dt, half_dt, accel_scale, kappa;  // accel_scale = mu / m
    R inv_width;                        // 1 / width (v^2 units)
    R theta_per_B;                      // Larmor angle per tesla, mu dt / hbar (0: no precession)
    R inv_width_maj;                    // 1 / width of the Majorana sigmoid in <s.B^> (0: no Majorana weight)
    double cut_scale;                   // d cut / d eta = 2 kB T0 / m
};

// field of the linear trap: B = (h x, h y, B0 - B' z), h = B'/2, written B = J x + B0 e_z with
// J = diag(h, h, -B'); its unit vector, |B|, grad |B| = J b^ and (derivs) d|B|/dB', d|B|/dB0.  The
// second derivatives are never formed: the adjoints apply them through P = (I - b^ b^T) / |B|
// (field_grad_adjoint).
template <class R> struct QuadField {
    R b[3];      // unit field
    R absB;
    R inv;       // 1 / |B| (0 where the field vanishes)
    R g[3];      // grad |B|
    R dabs_dBp, dabs_dB0;
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
    f.inv = inv;
    const R J[3] = {h, h, -Bp};
    for (int i = 0; i < 3; ++i) f.g[i] = J[i] * f.b[i];
    if (!derivs) return;
    const R q[3] = {R(0.5) * x, R(0.5) * y, -z};  // dB/dB'
    f.dabs_dBp = f.b[0] * q[0] + f.b[1] * q[1] + f.b[2] * q[2];
    f.dabs_dB0 = f.b[2];
}

// adjoint of g = grad |B| = J b^ at x: with an adjoint gb of g, accumulates into xb (3) and tb
// (B', B0).  dg/dx = J P J (the Hessian of |B|); dg_i/dB' = dJ_i b_i + J_i (P q)_i with q = dB/dB' =
// (x/2, y/2, -z) and dJ = (1/2, 1/2, -1); dg_i/dB0 = J_i P_i2.  With u = J gb and r = P u (P is
// symmetric): xb += J r, tb[0] += sum dJ_i b_i gb_i + q . r, tb[1] += r_2.
template <class R>
DSMC_HD void field_grad_adjoint(R Bp, const R* x, const QuadField<R>& f, const R* gb, R* xb, R* tb) {
    const R h = R(0.5) * Bp;
    const R u[3] = {h * gb[0], h * gb[1], -Bp * gb[2]};
    const R d = f.b[0] * u[0] + f.b[1] * u[1] + f.b[2] * u[2];
    R r[3];
    for (int i = 0; i < 3; ++i) r[i] = (u[i] - f.b[i] * d) * f.inv;
    xb[0] += h * r[0];
    xb[1] += h * r[1];
    xb[2] += -Bp * r[2];
    tb[0] += R(0.5) * (f.b[0] * gb[0] + f.b[1] * gb[1]) - f.b[2] * gb[2]
             + (R(0.5) * x[0] * r[0] + R(0.5) * x[1] * r[1] - x[2] * r[2]);
    tb[1] += r[2];
}

template <class R> DSMC_HD R sigmoid(R z) { return R(1) / (R(1) + xexp(-z)); }

// psi1 = c psi + s T(b) psi: the Larmor rotation of the spinor p = (Re u, Im u, Re d, Im d) by the
// angle with cos c, sin s about the unit field b (the rows of wavefunction.cu:51-70)
template <class R> DSMC_HD void larmor_apply(R c, R s, const R* b, const R* p, R* q) {
    q[0] = p[0] * c + (b[0] * p[3] - b[1] * p[2] + b[2] * p[1]) * s;
    q[1] = p[1] * c + (-b[0] * p[2] - b[1] * p[3] - b[2] * p[0]) * s;
    q[2] = p[2] * c + (b[0] * p[1] + b[1] * p[0] - b[2] * p[3]) * s;
    q[3] = p[3] * c + (-b[0] * p[0] + b[1] * p[1] + b[2] * p[2]) * s;
}
// <s.B^> = 2 bx Re(u* d) + 2 by Im(u* d) + bz (|u|^2 - |d|^2)   (evaporation.cu:88-90)
template <class R> DSMC_HD R spin_projection(const R* b, const R* p) {
    const R re = p[0] * p[2] + p[1] * p[3];
    const R im = p[0] * p[3] - p[1] * p[2];
    const R dz = p[0] * p[0] + p[1] * p[1] - p[2] * p[2] - p[3] * p[3];
    return R(2) * (b[0] * re + b[1] * im) + b[2] * dz;
}

// one smoothed step of one atom (collisions already applied to v); returns e
template <class R>
DSMC_HD R smooth_step(const SmoothConsts<R>& C, R cut, R* x, R* v, R* psi, R& w) {
    QuadField<R> f0, f1;
    quad_field(C.Bp, C.B0, x[0], x[1], x[2], false, f0);
    if (C.theta_per_B != R(0)) {
        R s, c;
        xsincos(C.theta_per_B * f0.absB, &s, &c);
        R q[4];
        larmor_apply(c, s, f0.b, psi, q);
        for (int k = 0; k < 4; ++k) psi[k] = q[k];
    }
    const R as = -C.accel_scale;
    for (int i = 0; i < 3; ++i) v[i] = v[i] + C.half_dt * (as * f0.g[i]);
    for (int i = 0; i < 3; ++i) x[i] = x[i] + C.dt * v[i];
    quad_field(C.Bp, C.B0, x[0], x[1], x[2], false, f1);
    for (int i = 0; i < 3; ++i) v[i] = v[i] + C.half_dt * (as * f1.g[i]);
    const R e = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + C.kappa * (f1.absB - C.B_floor);
    R sw = sigmoid((cut - e) * C.inv_width);
    if (C.inv_width_maj != R(0)) sw = sw * sigmoid(spin_projection(f1.b, psi) * C.inv_width_maj);
    w = w * sw;
    return e;
}

// adjoint of (b, |B|) at x through the field vector: accumulates into xb (3) and tb (B', B0)
template <class R>
DSMC_HD void field_vec_adjoint(R Bp, const R* x, const QuadField<R>& f, const R* bb, R absBb, R* xb, R* tb) {
    const R d = f.b[0] * bb[0] + f.b[1] * bb[1] + f.b[2] * bb[2];
    R Bb[3];
    for (int i = 0; i < 3; ++i) Bb[i] = (bb[i] - f.b[i] * d) * f.inv + f.b[i] * absBb;
    const R h = R(0.5) * Bp;
    xb[0] += h * Bb[0];
    xb[1] += h * Bb[1];
    xb[2] += -Bp * Bb[2];
    tb[0] += R(0.5) * x[0] * Bb[0] + R(0.5) * x[1] * Bb[1] - x[2] * Bb[2];
    tb[1] += Bb[2];
}

// Adjoint of smooth_step for ADJ_SEEDS seeds at once.  In: the state (x, v, psi, w) the step
// started from (v after collisions), the adjoints xb, vb, pb, wb of its outputs (per seed).  Out:
// xb, vb, pb, wb overwritten with the adjoints of the inputs; theta_b[seed][0..1] (B', B0)
// incremented; cut_b[seed] receives d/d cut.
template <class R>
DSMC_HD void smooth_step_adjoint(const SmoothConsts<R>& C, R cut, const R* x0, const R* v0, const R* p0, R w0,
                                 R (*xb)[3], R (*vb)[3], R (*pb)[4], R* wb, R (*theta_b)[2], R* cut_b) {
    // recompute the forward intermediates
    QuadField<R> f0, f1;
    quad_field(C.Bp, C.B0, x0[0], x0[1], x0[2], true, f0);
    const bool larmor = C.theta_per_B != R(0);
    R sn = R(0), cs = R(1), p1[4];
    if (larmor) {
        xsincos(C.theta_per_B * f0.absB, &sn, &cs);
        larmor_apply(cs, sn, f0.b, p0, p1);
    } else {
        for (int k = 0; k < 4; ++k) p1[k] = p0[k];
    }
    const R as = -C.accel_scale;
    R v1[3], x1[3], v2[3];
    for (int i = 0; i < 3; ++i) v1[i] = v0[i] + C.half_dt * (as * f0.g[i]);
    for (int i = 0; i < 3; ++i) x1[i] = x0[i] + C.dt * v1[i];
    quad_field(C.Bp, C.B0, x1[0], x1[1], x1[2], true, f1);
    for (int i = 0; i < 3; ++i) v2[i] = v1[i] + C.half_dt * (as * f1.g[i]);
    const R e = v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2] + C.kappa * (f1.absB - C.B_floor);
    const R sK = sigmoid((cut - e) * C.inv_width);
    const bool maj = C.inv_width_maj != R(0);
    const R sM = maj ? sigmoid(spin_projection(f1.b, p1) * C.inv_width_maj) : R(1);
    const R re = p1[0] * p1[2] + p1[1] * p1[3];
    const R im = p1[0] * p1[3] - p1[1] * p1[2];
    const R dz = p1[0] * p1[0] + p1[1] * p1[1] - p1[2] * p1[2] - p1[3] * p1[3];
    for (int q = 0; q < ADJ_SEEDS; ++q) {
        // w' = w sK sM
        const R wo = wb[q];
        wb[q] = wo * (sK * sM);
        const R zKb = wo * w0 * sM * sK * (R(1) - sK);
        const R eb = -zKb * C.inv_width;
        cut_b[q] = zKb * C.inv_width;
        // the Majorana weight: <s.B^> of psi1 at x1
        R p1b[4] = {pb[q][0], pb[q][1], pb[q][2], pb[q][3]};
        R b1b[3] = {R(0), R(0), R(0)};
        if (maj) {
            const R projb = wo * w0 * sK * sM * (R(1) - sM) * C.inv_width_maj;
            b1b[0] = projb * (R(2) * re);
            b1b[1] = projb * (R(2) * im);
            b1b[2] = projb * dz;
            const R reb = R(2) * f1.b[0] * projb, imb = R(2) * f1.b[1] * projb, dzb = f1.b[2] * projb;
            p1b[0] += reb * p1[2] + imb * p1[3] + R(2) * dzb * p1[0];
            p1b[1] += reb * p1[3] - imb * p1[2] + R(2) * dzb * p1[1];
            p1b[2] += reb * p1[0] - imb * p1[1] - R(2) * dzb * p1[2];
            p1b[3] += reb * p1[1] + imb * p1[0] - R(2) * dzb * p1[3];
        }
        // e = |v2|^2 + kappa (|B(x1)| - B_floor), and the unit field at x1
        R v2b[3], x1b[3];
        for (int i = 0; i < 3; ++i) {
            v2b[i] = vb[q][i] + R(2) * eb * v2[i];
            x1b[i] = xb[q][i];
        }
        field_vec_adjoint(C.Bp, x1, f1, b1b, eb * C.kappa, x1b, theta_b[q]);
        // v2 = v1 + hdt as g(x1)
        R g1b[3];
        for (int i = 0; i < 3; ++i) g1b[i] = C.half_dt * as * v2b[i];
        field_grad_adjoint(C.Bp, x1, f1, g1b, x1b, theta_b[q]);
        // x1 = x0 + dt v1 ; v1 = v0 + hdt as g(x0)
        R v1b[3];
        for (int i = 0; i < 3; ++i) v1b[i] = v2b[i] + C.dt * x1b[i];
        R g0b[3];
        for (int i = 0; i < 3; ++i) g0b[i] = C.half_dt * as * v1b[i];
        for (int i = 0; i < 3; ++i) {
            xb[q][i] = x1b[i];
            vb[q][i] = v1b[i];
        }
        field_grad_adjoint(C.Bp, x0, f0, g0b, xb[q], theta_b[q]);
        // psi1 = c psi0 + s T(b0) psi0, angle t = theta_per_B |B(x0)|
        if (larmor) {
            R tp[4];  // T(b0)^T psi1_bar
            tp[0] = -f0.b[2] * p1b[1] + f0.b[1] * p1b[2] - f0.b[0] * p1b[3];
            tp[1] = f0.b[2] * p1b[0] + f0.b[0] * p1b[2] + f0.b[1] * p1b[3];
            tp[2] = -f0.b[1] * p1b[0] - f0.b[0] * p1b[1] + f0.b[2] * p1b[3];
            tp[3] = f0.b[0] * p1b[0] - f0.b[1] * p1b[1] - f0.b[2] * p1b[2];
            R cb = R(0), sb = R(0);
            for (int k = 0; k < 4; ++k) {
                cb += p1b[k] * p0[k];
                sb += tp[k] * p0[k];  // psi1_bar . T(b0) psi0
            }
            R b0b[3];
            b0b[0] = sn * (p1b[0] * p0[3] - p1b[1] * p0[2] + p1b[2] * p0[1] - p1b[3] * p0[0]);
            b0b[1] = sn * (-p1b[0] * p0[2] - p1b[1] * p0[3] + p1b[2] * p0[0] + p1b[3] * p0[1]);
            b0b[2] = sn * (p1b[0] * p0[1] - p1b[1] * p0[0] - p1b[2] * p0[3] + p1b[3] * p0[2]);
            const R tb_ = -sn * cb + cs * sb;
            field_vec_adjoint(C.Bp, x0, f0, b0b, C.theta_per_B * tb_, xb[q], theta_b[q]);
            for (int k = 0; k < 4; ++k) pb[q][k] = cs * p1b[k] + sn * tp[k];
        } else {
            for (int k = 0; k < 4; ++k) pb[q][k] = p1b[k];
        }
    }
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
