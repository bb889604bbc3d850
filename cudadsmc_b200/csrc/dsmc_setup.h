// dsmc_setup.h -- host-side derivation of the per-cloud kernel constants (CloudPhys) from the
// C-ABI parameter structs, and the named workloads.  Shared by the GPU engine and the CPU
// oracle so both start from bit-identical constants.
#ifndef DSMC_SETUP_H
#define DSMC_SETUP_H

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "dsmc.h"
#include "dsmc_physics.h"

namespace dsmc {

// reference constants (CUDADSMC/include/deviceSystemParameters.cuh:12-31,
// CUDADSMC/include/initialSystemParameters.cuh:27-34)
constexpr double kRefMuB = 9.27400915e-24;
constexpr double kRefMassRb = 1.443160648e-25;
constexpr double kRefKB = 1.3806503e-23;
constexpr double kRefHbar = 1.05457148e-34;
constexpr double kRefA = 5.3e-9;
constexpr double kPi = 3.14159265358979323846;

inline double run_kB(const dsmc_params& r) { return r.kB > 0 ? r.kB : kRefKB; }
inline double run_hbar(const dsmc_params& r) { return r.hbar > 0 ? r.hbar : kRefHbar; }

// Validates one cloud; returns an empty string when it is usable.
inline std::string validate_cloud(const dsmc_params& run, const dsmc_cloud_params& c, int k) {
    const std::string w = "cloud " + std::to_string(k) + ": ";
    if (!(run.dt > 0)) return "dt must be > 0";
    if (run.collide_every < 1) return "collide_every must be >= 1";
    if (c.n_atoms < 0) return w + "n_atoms < 0";
    if (c.cells[0] < 1 || c.cells[1] < 1 || c.cells[2] < 1) return w + "cells must be >= 1";
    if (!(c.mass > 0)) return w + "mass must be > 0";
    if (!(c.temperature > 0)) return w + "temperature must be > 0";
    if (c.trap < 0 || c.trap > 2) return w + "unknown trap";
    for (int a = 0; a < 3; ++a)
        if (!(c.grid_max[a] > c.grid_min[a])) return w + "grid_max must exceed grid_min";
    if (c.knife_nknots < 0 || c.knife_nknots > DSMC_MAX_KNOTS) return w + "knife_nknots out of range";
    if ((c.flags & DSMC_F_KNIFE) && c.knife_nknots < 1) return w + "knife enabled without knots";
    if (c.capacity > 0 && c.capacity < c.n_atoms) return w + "capacity below n_atoms";
    return std::string();
}

template <class R>
inline void make_cloud_phys(const dsmc_params& run, const dsmc_cloud_params& c, int k, int cell_base,
                            CloudPhys<R>& P) {
    const double kB = run_kB(run);
    const double hbar = run_hbar(run);
    const int64_t nc = (int64_t)c.cells[0] * c.cells[1] * c.cells[2];
    memset(&P, 0, sizeof(P));
    P.trap = c.trap;
    P.flags = c.flags;
    P.nx = c.cells[0]; P.ny = c.cells[1]; P.nz = c.cells[2];
    P.cell_base = cell_base;
    P.ovf_cell = (int32_t)(cell_base + nc);
    P.cloud_id = c.stream_id & 0xFFFFFF;
    (void)k;
    const double Lx = c.grid_max[0] - c.grid_min[0];
    const double Ly = c.grid_max[1] - c.grid_min[1];
    const double Lz = c.grid_max[2] - c.grid_min[2];
    const double dx = Lx / c.cells[0], dy = Ly / c.cells[1], dz = Lz / c.cells[2];
    P.gmin_x = (R)c.grid_min[0]; P.gmin_y = (R)c.grid_min[1]; P.gmin_z = (R)c.grid_min[2];
    P.inv_dx = (R)(1.0 / dx); P.inv_dy = (R)(1.0 / dy); P.inv_dz = (R)(1.0 / dz);
    P.fnx = (R)P.nx; P.fny = (R)P.ny; P.fnz = (R)P.nz;
    P.box_x = (R)Lx; P.box_y = (R)Ly; P.box_z = (R)Lz;
    P.inv_box_x = (R)(1.0 / Lx); P.inv_box_y = (R)(1.0 / Ly); P.inv_box_z = (R)(1.0 / Lz);
    P.Bp = (R)c.dBdz; P.Bpp = (R)c.d2Bdz2; P.B0 = (R)c.B0;
    P.B_floor = (R)(c.trap == DSMC_TRAP_IOFFE_PRITCHARD ? std::fabs(c.B0) : 0.0);
    P.dt = (R)run.dt; P.half_dt = (R)(0.5 * run.dt);
    P.accel_scale = (R)(c.moment / c.mass);
    P.theta_per_B = (R)(c.moment * run.dt / hbar);
    P.kappa = (R)(2.0 * c.moment / c.mass);
    P.sigma = (R)c.sigma;
    P.mcwf_cp = (R)(1.163 * std::sqrt(c.sigma));
    P.mcwf_cv = (R)(std::sqrt(2.0 / 3.14159265358979323846) * hbar / (c.mass * c.sigma));
    P.dt_period = (R)(run.collide_every * run.dt);
    P.cand_pref = (R)(c.alpha * run.dt * run.collide_every / (dx * dy * dz));
    P.v_init = (R)std::sqrt(kB * c.temperature / c.mass);
    P.r0_init = (R)((c.moment > 0 && c.dBdz != 0) ? kB * c.temperature / (c.moment * std::fabs(c.dBdz)) : 0.0);
    P.inv_kT_over_mu = (R)(c.moment / (kB * c.temperature));
    // proposal box of the rejection sampler: along each axis, 1.25 x the distance at which
    // mu (|B| - B_floor) reaches 40 kB T (bisection on the field), clipped to the grid box; the
    // Boltzmann weight left outside is below exp(-40)
    {
        double lo[3] = {c.grid_min[0], c.grid_min[1], c.grid_min[2]};
        double hi[3] = {c.grid_max[0], c.grid_max[1], c.grid_max[2]};
        if (c.trap == DSMC_TRAP_IOFFE_PRITCHARD && c.moment > 0) {
            CloudPhys<double> Q;
            memset(&Q, 0, sizeof(Q));
            Q.trap = TRAP_IOFFE_PRITCHARD;
            Q.Bp = c.dBdz; Q.Bpp = c.d2Bdz2; Q.B0 = c.B0;
            const double target = 40.0 * kB * c.temperature / c.moment + std::fabs(c.B0);
            for (int axis = 0; axis < 3; ++axis) {
                for (int side = -1; side <= 1; side += 2) {
                    const double lim = side < 0 ? -c.grid_min[axis] : c.grid_max[axis];
                    if (!(lim > 0)) continue;
                    double a0 = 0.0, a1 = lim;
                    double pt[3] = {0, 0, 0};
                    pt[axis] = side * a1;
                    Field<double> f;
                    trap_field(Q, pt[0], pt[1], pt[2], f);
                    if (f.absB < target) continue;  // the grid box is the bound
                    for (int it = 0; it < 200; ++it) {
                        const double m = 0.5 * (a0 + a1);
                        pt[axis] = side * m;
                        trap_field(Q, pt[0], pt[1], pt[2], f);
                        if (f.absB < target) a0 = m; else a1 = m;
                    }
                    const double w = std::min(1.25 * a1, lim);
                    if (side < 0) lo[axis] = -w; else hi[axis] = w;
                }
            }
        }
        P.prop_min_x = (R)lo[0]; P.prop_min_y = (R)lo[1]; P.prop_min_z = (R)lo[2];
        P.prop_len_x = (R)(hi[0] - lo[0]); P.prop_len_y = (R)(hi[1] - lo[1]); P.prop_len_z = (R)(hi[2] - lo[2]);
    }
    P.knife_nknots = c.knife_nknots;
    P.id_base = 0;  // set by the owner of the by-id records, which knows every cloud's capacity
    P.id_cap = (int32_t)c.capacity;
    P.pad0 = 0;
    for (int i = 0; i < DSMC_MAX_KNOTS; ++i) {
        P.knife_step[i] = c.knife_step[i];
        P.knife_eta[i] = c.knife_eta[i];
    }
    P.mass = c.mass; P.moment = c.moment; P.kB = kB; P.T0 = c.temperature;
}

// initial (sigma v_r)_max of every cell: sigma sqrt(16 kB T / (pi m))  (CUDADSMC/src/setUp.cu:287-292)
inline double default_sigvrmax(const dsmc_params& run, const dsmc_cloud_params& c) {
    if (c.sigvrmax_init > 0) return c.sigvrmax_init;
    return c.sigma * std::sqrt(16.0 * run_kB(run) * c.temperature / (kPi * c.mass));
}

inline int64_t cloud_cells(const dsmc_cloud_params& c) {
    return (int64_t)c.cells[0] * c.cells[1] * c.cells[2] + 1;  // + overflow cell
}

inline void fill_cloud_defaults(dsmc_cloud_params* c) {
    memset(c, 0, sizeof(*c));
    c->mass = kRefMassRb;
    c->moment = 0.5 * kRefMuB;  // |F=1, mF=-1>, g_F = -1/2: mu = g_F mF muB
    c->sigma = 8.0 * kPi * kRefA * kRefA;  // 8 pi a^2, CUDADSMC/src/collisions.cu:312
    c->alpha = 1.0;
    c->init_mode = DSMC_INIT_THERMAL;
    c->trap = DSMC_TRAP_QUADRUPOLE;
    c->flags = DSMC_F_COLLIDE | DSMC_F_LARMOR | DSMC_F_NORMALISE;
}

// grid spanning +-radii thermal lengths of the linear trap: r_z = kT/(mu B'), r_x = r_y = 2 r_z
inline void grid_around_quadrupole(dsmc_cloud_params* c, double radii, int nc) {
    const double rz = kRefKB * c->temperature / (c->moment * c->dBdz);
    const double rx = 2.0 * rz;
    const double z0 = c->B0 / c->dBdz;
    c->grid_min[0] = -radii * rx; c->grid_max[0] = radii * rx;
    c->grid_min[1] = -radii * rx; c->grid_max[1] = radii * rx;
    c->grid_min[2] = z0 - radii * rz; c->grid_max[2] = z0 + radii * rz;
    c->cells[0] = c->cells[1] = c->cells[2] = nc;
}

inline dsmc_status fill_preset(int which, dsmc_params* run, dsmc_cloud_params* c) {
    memset(run, 0, sizeof(*run));
    run->precision = DSMC_FP32;
    run->collide_every = 1;
    run->dt = 1e-6;
    run->seed = 1234;  // the reference's curand_init seed, CUDADSMC/src/setUp.cu:71
    run->use_graphs = 1;
    fill_cloud_defaults(c);
    switch (which) {
    case 0:  // small trapped cloud, FP64, no evaporation
        run->precision = DSMC_FP64;
        c->n_atoms = 10000;
        c->temperature = 20e-6;
        c->dBdz = 2.5;
        c->alpha = 3e6 / 1e4;  // h_N / N, CUDADSMC/src/main.cu:53
        grid_around_quadrupole(c, 5.0, 50);
        break;
    case 1:  // homogeneous periodic box
        run->dt = 5e-6;
        c->n_atoms = 1000000;
        c->temperature = 10e-6;
        c->trap = DSMC_TRAP_BOX;
        c->init_mode = DSMC_INIT_UNIFORM;
        c->flags = DSMC_F_COLLIDE;
        c->alpha = 1e4;
        c->dBdz = 0.0;
        for (int a = 0; a < 3; ++a) { c->grid_min[a] = -0.5e-3; c->grid_max[a] = 0.5e-3; }
        c->cells[0] = c->cells[1] = c->cells[2] = 100;
        break;
    case 2:  // full trapped step at scale
        c->n_atoms = 10000000;
        c->temperature = 50e-6;
        c->dBdz = 2.5;
        // the knife ramps eta against the initial temperature (an absolute energy ramp): a cut
        // that follows the running T of the just-truncated cloud moves down every step and
        // evaporates everything
        c->flags = DSMC_F_COLLIDE | DSMC_F_LARMOR | DSMC_F_NORMALISE | DSMC_F_MAJORANA | DSMC_F_KNIFE |
                   DSMC_F_KNIFE_FIXED_T;
        c->knife_nknots = 2;
        c->knife_step[0] = 0; c->knife_eta[0] = 6.0;
        c->knife_step[1] = 1e5; c->knife_eta[1] = 4.0;
        grid_around_quadrupole(c, 5.0, 128);
        break;
    case 4:  // adjoint workload
        c->n_atoms = 1000000;
        c->temperature = 30e-6;
        c->dBdz = 2.5;
        c->B0 = 1e-4;
        c->flags = DSMC_F_COLLIDE | DSMC_F_LARMOR | DSMC_F_NORMALISE | DSMC_F_KNIFE | DSMC_F_KNIFE_FIXED_T;
        c->knife_nknots = 9;
        for (int i = 0; i < 9; ++i) {
            c->knife_step[i] = 250.0 * i;
            c->knife_eta[i] = 8.0 - 0.5 * i;
        }
        grid_around_quadrupole(c, 5.0, 100);
        break;
    default:
        return DSMC_ERR_INVALID;
    }
    c->capacity = c->n_atoms;
    return DSMC_OK;
}

}  // namespace dsmc

#endif  // DSMC_SETUP_H
