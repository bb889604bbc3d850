// dsmc_oracle.cpp -- CPU restatement of the CUDADSMC timestep.  TEST INFRASTRUCTURE ONLY:
// used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the checker and the
// timed host-core baseline; the product (cudadsmc_b200) never links or calls it.
//
// What it restates (paths inside the CUDADSMC project):
//   main loop order            src/main.cu:410-524 (index/sort, collide, spin, move, evaporate)
//   initial cloud              src/setUp.cu:129-252 (exact Gamma(3) sampler for the linear trap)
//   (sigma v_r)max init        src/setUp.cu:287-292
//   cell index                 src/collisions.cu:163-226
//   sort by cell               src/collisions.cu:275-287 (thrust::sort_by_key, stable)
//   NTC collisions             src/collisions.cu:291-437, 529-546
//   Larmor + normalise         src/wavefunction.cu:11-73, 279-299
//   Verlet motion              src/moveAtoms.cu:23-157
//   evaporation tag + compact  src/evaporation.cu:68-106, src/main.cu:493-498
//   temperature                src/evaporation.cu:108-128
// with the intended semantics where the reference has defects: the sort pairs each atom with
// its own cell (collisions.cu:181 vs 282-284), candidate pairs are uniform over all distinct
// pairs (collisions.cu:407 never picks the last atom), dt is the run's dt everywhere
// (collisions.cu:314, wavefunction.cu:45,63 hard-code 1e-7).
//
// The per-atom and per-cell arithmetic is the shared header dsmc_physics.h (IEEE-exact
// operations only), so results are bit-identical to the GPU for the same inputs.  The
// serial path (fast = 0) defines the sorted order directly as a stable sort of the survivors
// by (new cell, moved); the OpenMP path (fast = 1) builds the same order in parallel and is
// the timed CPU baseline.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "dsmc.h"
#include "dsmc_physics.h"
#include "dsmc_setup.h"

using namespace dsmc;

namespace {

template <class R> struct Q4 { R x, y, z, w; };

struct CloudAcc {
    long long step = 0, n_alive = 0;
    i128 sum_v2 = 0, sum_B = 0, cum_evap_v2 = 0, cum_evap_B = 0;
    long long cum_evap = 0, cum_maj = 0, cum_knife = 0, cum_coll = 0, cum_cand = 0, cum_atom_steps = 0;
    double T_knife = 0;
};

struct OracleBase {
    std::string err;
    virtual ~OracleBase() {}
    virtual void init(uint64_t seed) = 0;
    virtual void step(int n) = 0;
    virtual void diag(int cloud, dsmc_diag* out) = 0;
    virtual void get_state(dsmc_state_buffers* o) = 0;
    virtual void set_state(const dsmc_state_buffers* in) = 0;
    virtual void cell_starts(int32_t* st, int64_t cap, int64_t* total) = 0;
    virtual void get_sigvrmax(void* out, int64_t cap) = 0;
    virtual void set_sigvrmax(const void* in, int64_t n) = 0;
    virtual void set_recording(int flags) = 0;
    virtual void get_evaporated(int k, double* p3, double* v3, int32_t* st, int32_t* fa, int64_t cap) = 0;
    virtual void get_cell_collisions(int32_t* counts, int64_t cap) = 0;
};

struct OFail { std::string msg; };

template <class R> struct Oracle final : OracleBase {
    typedef Q4<R> V;
    dsmc_params run;
    std::vector<dsmc_cloud_params> cp;
    std::vector<CloudPhys<R>> phys;
    int nclouds = 0, total_cells = 0;
    bool fast = false;
    std::vector<int> cell_base;           // nclouds + 1
    std::vector<int> natoms;              // atoms per cloud (current)
    std::vector<V> pos, vel, psi;         // current state, sorted
    std::vector<int> start;               // total_cells + 1
    std::vector<R> sigvrmax;
    std::vector<CloudAcc> acc;
    int step_no = 0;
    bool ready = false;
    // snapshot records (DSMC_REC_* flags): lost atoms by id slot, collisions per cell and step
    int rec_flags = 0;
    std::vector<V> rec_pos, rec_vel;
    std::vector<int> rec_step, rec_fate;
    std::vector<int> rec_coll_step, rec_coll_count;
    int64_t id_slots = 0;

    Oracle(const dsmc_params& r, const dsmc_cloud_params* c, int n, bool f) : run(r), cp(c, c + n), nclouds(n), fast(f) {
        phys.resize(n);
        cell_base.resize(n + 1);
        int cells = 0;
        for (int k = 0; k < n; ++k) {
            std::string bad = validate_cloud(run, cp[k], k);
            if (!bad.empty()) throw OFail{bad};
            make_cloud_phys<R>(run, cp[k], k, cells, phys[k]);
            cell_base[k] = cells;
            cells += (int)cloud_cells(cp[k]);
            const int64_t ck = cp[k].capacity > 0 ? cp[k].capacity : cp[k].n_atoms;
            phys[k].id_base = (int32_t)id_slots;
            phys[k].id_cap = (int32_t)ck;
            id_slots += ck;
        }
        cell_base[n] = cells;
        total_cells = cells;
        start.assign(total_cells + 1, 0);
        sigvrmax.resize(total_cells);
        for (int k = 0; k < n; ++k)
            for (int c = cell_base[k]; c < cell_base[k + 1]; ++c) sigvrmax[c] = (R)default_sigvrmax(run, cp[k]);
        acc.resize(n);
        natoms.assign(n, 0);
    }

    int cloud_begin(int k) const {
        int s = 0;
        for (int j = 0; j < k; ++j) s += natoms[j];
        return s;
    }

    // --------------------------------------------------------------- full sort + measure
    void sort_by_cell_and_measure(std::vector<V>& P, std::vector<V>& Vv, std::vector<V>& S) {
        const int n = (int)P.size();
        std::vector<int> cell(n), order(n);
        int i0 = 0;
        for (int k = 0; k < nclouds; ++k) {
            const CloudPhys<R>& C = phys[k];
            for (int i = i0; i < i0 + natoms[k]; ++i)
                cell[i] = cell_of(C, P[i].x, P[i].y, P[i].z, C.trap == TRAP_BOX);
            i0 += natoms[k];
        }
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cell[a] < cell[b]; });
        pos.resize(n); vel.resize(n); psi.resize(n);
        for (int j = 0; j < n; ++j) {
            pos[j] = P[order[j]]; vel[j] = Vv[order[j]]; psi[j] = S[order[j]];
        }
        std::fill(start.begin(), start.end(), 0);
        for (int j = 0; j < n; ++j) start[cell[order[j]] + 1]++;
        for (int c = 0; c < total_cells; ++c) start[c + 1] += start[c];
        step_no = 0;
        for (int k = 0; k < nclouds; ++k) {
            CloudAcc& a = acc[k];
            a = CloudAcc();
            const CloudPhys<R>& C = phys[k];
            const int b = cloud_begin(k);
            for (int i = b; i < b + natoms[k]; ++i) {
                Field<R> f;
                trap_field(C, pos[i].x, pos[i].y, pos[i].z, f);
                const R v2 = vel[i].x * vel[i].x + vel[i].y * vel[i].y + vel[i].z * vel[i].z;
                a.sum_v2 += fx_from((double)v2);
                const R sb = (lane_to_u32(vel[i].w) & 1u) ? -f.absB : f.absB;  // anti-trapped: -|B|
                a.sum_B += fx_from((double)sb);
            }
            a.n_alive = natoms[k];
            a.T_knife = knife_temperature(C.mass, C.kB, C.T0, (C.flags & F_KNIFE_FIXED_T) != 0, a.sum_v2, a.n_alive);
        }
        ready = true;
    }

    void init(uint64_t seed) override {
        run.seed = seed;
        int n = 0;
        for (int k = 0; k < nclouds; ++k) { natoms[k] = (int)cp[k].n_atoms; n += natoms[k]; }
        std::vector<V> P(n), Vv(n), S(n);
        int i0 = 0;
        for (int k = 0; k < nclouds; ++k) {
            const CloudPhys<R>& C = phys[k];
#pragma omp parallel for schedule(static) if (fast)
            for (int j = 0; j < natoms[k]; ++j) {
                Atom<R> a;
                init_atom(C, cp[k].init_mode, (uint32_t)j, seed, a);
                const int i = i0 + j;
                P[i] = V{a.x, a.y, a.z, lane_from_u32((uint32_t)j, R(0))};
                Vv[i] = V{a.vx, a.vy, a.vz, lane_from_u32(a.flags, R(0))};
                S[i] = V{a.ur, a.ui, a.dr, a.di};
            }
            i0 += natoms[k];
        }
        sort_by_cell_and_measure(P, Vv, S);
    }

    void set_state(const dsmc_state_buffers* in) override {
        int n = 0;
        for (int k = 0; k < nclouds; ++k) { natoms[k] = (int)in->cloud_counts[k]; n += natoms[k]; }
        if (n != in->n) throw OFail{"cloud_counts do not add up to n"};
        std::vector<V> P(n), Vv(n), S(n);
        memcpy(P.data(), in->pos, n * sizeof(V));
        memcpy(Vv.data(), in->vel, n * sizeof(V));
        memcpy(S.data(), in->psi, n * sizeof(V));
        sort_by_cell_and_measure(P, Vv, S);
    }

    // --------------------------------------------------------------- one timestep
    void step(int nsteps) override {
        if (!ready) throw OFail{"step before init"};
        for (int s = 0; s < nsteps; ++s) step_once();
    }

    void step_once() {
        const int n = (int)pos.size();
        const uint32_t st = (uint32_t)step_no;
        std::vector<long long> coll(nclouds, 0), cand(nclouds, 0);
        // 1. collisions, cell by cell (the cells of the current sorted order)
        if (step_no % run.collide_every == 0) {
            for (int k = 0; k < nclouds; ++k) {
                const CloudPhys<R>& C = phys[k];
                if (!(C.flags & F_COLLIDE)) continue;
                long long ca = 0, cc = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : ca, cc) if (fast)
                for (int c = C.cell_base; c < C.ovf_cell; ++c) {
                    const int m = start[c + 1] - start[c];
                    if (m < 2) continue;
                    R svm = sigvrmax[c];
                    CollideResult<R> r =
                        collide_cell<R>(&vel[start[c]], m, svm, C, (uint32_t)(c - C.cell_base), st, run.seed);
                    sigvrmax[c] = svm;
                    ca += r.accepted;
                    cc += r.candidates;
                    if (rec_flags & DSMC_REC_CELL_COLLISIONS) {
                        rec_coll_step[c] = step_no;
                        rec_coll_count[c] = r.accepted;
                    }
                }
                coll[k] = ca;
                cand[k] = cc;
            }
        }
        // 2. spin + motion + evaporation tests, atom by atom
        std::vector<int> newcell(n), fate(n);
        std::vector<unsigned char> moved(n);
        std::vector<R> v2(n), absB(n);
        int i0 = 0;
        for (int k = 0; k < nclouds; ++k) {
            const CloudPhys<R>& C = phys[k];
            R cut = R(0);
            if (C.flags & F_KNIFE) {
                double eta = knife_eta(C.knife_nknots, C.knife_step, C.knife_eta, (double)step_no);
                cut = (R)knife_cut_v2(eta, C.kB, acc[k].T_knife, C.mass);
            }
            const bool box = C.trap == TRAP_BOX;
#pragma omp parallel for schedule(static) if (fast)
            for (int i = i0; i < i0 + natoms[k]; ++i) {
                const int oc = cell_of(C, pos[i].x, pos[i].y, pos[i].z, box);
                Atom<R> a;
                a.x = pos[i].x; a.y = pos[i].y; a.z = pos[i].z;
                a.vx = vel[i].x; a.vy = vel[i].y; a.vz = vel[i].z;
                a.ur = psi[i].x; a.ui = psi[i].y; a.dr = psi[i].z; a.di = psi[i].w;
                a.flags = lane_to_u32(vel[i].w);
                AtomOut<R> o;
                StepCtx sc;
                sc.id = lane_to_u32(pos[i].w);
                sc.step = (uint32_t)step_no;
                sc.cloud = (uint32_t)C.cloud_id;
                sc.mcwf = ((step_no % run.collide_every) == 0 ? 1u : 0u) |
                          (((step_no + 1) % run.collide_every) == 0 ? 2u : 0u);
                sc.seed = run.seed;
                advance_atom(C, cut, a, o, sc);
                pos[i].x = a.x; pos[i].y = a.y; pos[i].z = a.z;
                vel[i].x = a.vx; vel[i].y = a.vy; vel[i].z = a.vz; vel[i].w = lane_from_u32(a.flags, R(0));
                psi[i].x = a.ur; psi[i].y = a.ui; psi[i].z = a.dr; psi[i].w = a.di;
                newcell[i] = o.cell;
                fate[i] = o.fate;
                moved[i] = (o.cell != oc) ? 1 : 0;
                v2[i] = o.v2;
                absB[i] = o.absB;
            }
            i0 += natoms[k];
        }
        // 3. survivors sorted stably by (new cell, moved); the lost are tallied
        std::vector<int> order;
        if (!fast) {
            order.reserve(n);
            for (int i = 0; i < n; ++i)
                if (fate[i] == FATE_ALIVE) order.push_back(i);
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
                if (newcell[a] != newcell[b]) return newcell[a] < newcell[b];
                return moved[a] < moved[b];
            });
        } else {
            order = fast_order(newcell, fate, moved);
        }
        std::vector<V> P2(order.size()), V2(order.size()), S2(order.size());
#pragma omp parallel for schedule(static) if (fast)
        for (int j = 0; j < (int)order.size(); ++j) {
            P2[j] = pos[order[j]]; V2[j] = vel[order[j]]; S2[j] = psi[order[j]];
        }
        // diagnostics
        i0 = 0;
        for (int k = 0; k < nclouds; ++k) {
            CloudAcc& a = acc[k];
            i128 sv = 0, sb = 0, ev = 0, eb = 0;
            long long alive = 0, maj = 0, kn = 0;
            for (int i = i0; i < i0 + natoms[k]; ++i) {
                if (fate[i] == FATE_ALIVE) {
                    ++alive;
                    sv += fx_from((double)v2[i]);
                    sb += fx_from((double)absB[i]);
                } else {
                    ev += fx_from((double)v2[i]);
                    eb += fx_from((double)absB[i]);
                    if (fate[i] == FATE_MAJORANA) ++maj; else ++kn;
                    const uint32_t id = lane_to_u32(pos[i].w);
                    if ((rec_flags & DSMC_REC_EVAPORATED) && id < (uint32_t)phys[k].id_cap) {
                        const int64_t slot = phys[k].id_base + (int64_t)id;
                        rec_pos[slot] = pos[i];
                        rec_vel[slot] = vel[i];
                        rec_step[slot] = step_no;
                        rec_fate[slot] = fate[i];
                    }
                }
            }
            a.step = step_no + 1;
            a.n_alive = alive;
            a.sum_v2 = sv;
            a.sum_B = sb;
            a.cum_evap += maj + kn;
            a.cum_maj += maj;
            a.cum_knife += kn;
            a.cum_evap_v2 += ev;
            a.cum_evap_B += eb;
            a.cum_coll += coll[k];
            a.cum_cand += cand[k];
            a.cum_atom_steps += natoms[k];
            const CloudPhys<R>& C = phys[k];
            a.T_knife = knife_temperature(C.mass, C.kB, C.T0, (C.flags & F_KNIFE_FIXED_T) != 0, sv, alive);
            i0 += natoms[k];
            natoms[k] = (int)alive;
        }
        std::fill(start.begin(), start.end(), 0);
        for (int j = 0; j < (int)order.size(); ++j) start[newcell[order[j]] + 1]++;
        for (int c = 0; c < total_cells; ++c) start[c + 1] += start[c];
        pos.swap(P2); vel.swap(V2); psi.swap(S2);
        ++step_no;
    }

    void set_recording(int flags) override {
        rec_flags = flags;
        if (flags & DSMC_REC_EVAPORATED) {
            rec_pos.assign(id_slots, V{0, 0, 0, 0});
            rec_vel.assign(id_slots, V{0, 0, 0, 0});
            rec_step.assign(id_slots, -1);
            rec_fate.assign(id_slots, 0);
        }
        if (flags & DSMC_REC_CELL_COLLISIONS) {
            rec_coll_step.assign(total_cells, -1);
            rec_coll_count.assign(total_cells, 0);
        }
    }
    void get_evaporated(int k, double* p3, double* v3, int32_t* st, int32_t* fa, int64_t cap) override {
        if (!(rec_flags & DSMC_REC_EVAPORATED) || k < 0 || k >= nclouds || cap < phys[k].id_cap) throw OFail{"get_evaporated"};
        for (int i = 0; i < phys[k].id_cap; ++i) {
            const int64_t s = phys[k].id_base + i;
            for (int a = 0; a < 3; ++a) {
                if (p3) p3[3 * i + a] = (double)(&rec_pos[s].x)[a];
                if (v3) v3[3 * i + a] = (double)(&rec_vel[s].x)[a];
            }
            if (st) st[i] = rec_step[s];
            if (fa) fa[i] = rec_fate[s];
        }
    }
    void get_cell_collisions(int32_t* counts, int64_t cap) override {
        if (!(rec_flags & DSMC_REC_CELL_COLLISIONS) || cap < total_cells) throw OFail{"get_cell_collisions"};
        const int last = step_no > 0 ? ((step_no - 1) / run.collide_every) * run.collide_every : -1;
        for (int c = 0; c < total_cells; ++c) counts[c] = (last >= 0 && rec_coll_step[c] == last) ? rec_coll_count[c] : 0;
    }

    // The same order as the stable sort, built in parallel: for every new cell its stayers
    // (old order), then the atoms that entered it (old order).
    std::vector<int> fast_order(const std::vector<int>& newcell, const std::vector<int>& fate,
                                const std::vector<unsigned char>& moved) {
        const int n = (int)newcell.size();
        std::vector<int> stay(total_cells, 0), inc(total_cells, 0), dest(n, -1);
        // stayers are contiguous per old cell: rank them cell by cell
#pragma omp parallel for schedule(dynamic, 1024) if (fast)
        for (int c = 0; c < total_cells; ++c) {
            int r = 0;
            for (int i = start[c]; i < start[c + 1]; ++i)
                if (fate[i] == FATE_ALIVE && !moved[i]) dest[i] = r++;
            stay[c] = r;
        }
        for (int i = 0; i < n; ++i)
            if (fate[i] == FATE_ALIVE && moved[i]) inc[newcell[i]]++;
        std::vector<int> ns(total_cells + 1, 0), cur(total_cells);
        for (int c = 0; c < total_cells; ++c) ns[c + 1] = ns[c] + stay[c] + inc[c];
        for (int c = 0; c < total_cells; ++c) cur[c] = ns[c] + stay[c];
        std::vector<int> order(ns[total_cells]);
#pragma omp parallel for schedule(static) if (fast)
        for (int i = 0; i < n; ++i)
            if (fate[i] == FATE_ALIVE && !moved[i]) order[ns[newcell[i]] + dest[i]] = i;
        for (int i = 0; i < n; ++i)
            if (fate[i] == FATE_ALIVE && moved[i]) order[cur[newcell[i]]++] = i;
        return order;
    }

    // --------------------------------------------------------------- outputs
    void diag(int cloud, dsmc_diag* out) override {
        if (!ready) throw OFail{"diag before init"};
        int k0 = cloud < 0 ? 0 : cloud, k1 = cloud < 0 ? nclouds : cloud + 1;
        memset(out, 0, sizeof(*out));
        i128 sv = 0, sb = 0;
        double e_kin = 0, e_pot = 0, e_evap = 0, msum = 0;
        for (int k = k0; k < k1; ++k) {
            const CloudAcc& a = acc[k];
            const CloudPhys<R>& C = phys[k];
            out->step = step_no;
            out->n_alive += a.n_alive;
            sv += a.sum_v2;
            sb += a.sum_B;
            out->n_evaporated += a.cum_evap;
            out->n_majorana += a.cum_maj;
            out->n_knife += a.cum_knife;
            out->collisions += a.cum_coll;
            out->candidates += a.cum_cand;
            out->atom_steps += a.cum_atom_steps;
            e_kin += 0.5 * C.mass * fx_to_double(a.sum_v2);
            e_pot += C.moment * fx_to_double(a.sum_B);
            e_evap += 0.5 * C.mass * fx_to_double(a.cum_evap_v2) + C.moment * fx_to_double(a.cum_evap_B);
            msum += C.mass * fx_to_double(a.sum_v2);
        }
        out->time = (double)step_no * run.dt;
        out->e_kin = e_kin;
        out->e_pot = e_pot;
        out->sum_v2 = fx_to_double(sv);
        out->sum_absB = fx_to_double(sb);
        out->temperature = out->n_alive > 0 ? msum / (3.0 * phys[k0].kB * (double)out->n_alive) : 0.0;
        out->e_evaporated = e_evap;
    }

    void get_state(dsmc_state_buffers* o) override {
        const int n = (int)pos.size();
        if (o->n < n) throw OFail{"state buffers too small"};
        if (o->pos) memcpy(o->pos, pos.data(), n * sizeof(V));
        if (o->vel) memcpy(o->vel, vel.data(), n * sizeof(V));
        if (o->psi) memcpy(o->psi, psi.data(), n * sizeof(V));
        o->n = n;
        if (o->cloud_counts)
            for (int k = 0; k < nclouds; ++k) o->cloud_counts[k] = natoms[k];
    }
    void cell_starts(int32_t* st, int64_t cap, int64_t* total) override {
        if (total) *total = total_cells;
        if (!st) return;
        if (cap < total_cells + 1) throw OFail{"cell start buffer too small"};
        memcpy(st, start.data(), (total_cells + 1) * sizeof(int));
    }
    void get_sigvrmax(void* out, int64_t cap) override {
        if (cap < total_cells) throw OFail{"sigvrmax buffer too small"};
        memcpy(out, sigvrmax.data(), total_cells * sizeof(R));
    }
    void set_sigvrmax(const void* in, int64_t n) override {
        if (n != total_cells) throw OFail{"sigvrmax length must equal the number of cells"};
        memcpy(sigvrmax.data(), in, total_cells * sizeof(R));
    }
};

template <class F> int oguard(OracleBase* o, F&& f) {
    try {
        f();
        if (o) o->err.clear();
        return 0;
    } catch (const OFail& e) {
        if (o) o->err = e.msg;
        return 1;
    }
}

thread_local std::string g_err;

}  // namespace

#define OAPI extern "C" __attribute__((visibility("default")))

OAPI int oracle_create(const dsmc_params* run, const dsmc_cloud_params* clouds, int n, int fast, void** out) {
    try {
        if (run->precision == DSMC_FP32) *out = new Oracle<float>(*run, clouds, n, fast != 0);
        else *out = new Oracle<double>(*run, clouds, n, fast != 0);
        return 0;
    } catch (const OFail& e) {
        g_err = e.msg;
        *out = nullptr;
        return 1;
    }
}
OAPI const char* oracle_last_error(void* h) { return h ? ((OracleBase*)h)->err.c_str() : g_err.c_str(); }
OAPI void oracle_destroy(void* h) { delete (OracleBase*)h; }
OAPI int oracle_init(void* h, uint64_t seed) { return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->init(seed); }); }
OAPI int oracle_step(void* h, int n) { return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->step(n); }); }
OAPI int oracle_diag(void* h, int cloud, dsmc_diag* out) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->diag(cloud, out); });
}
OAPI int oracle_get_state(void* h, dsmc_state_buffers* o) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->get_state(o); });
}
OAPI int oracle_set_state(void* h, const dsmc_state_buffers* in) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->set_state(in); });
}
OAPI int oracle_get_cell_starts(void* h, int32_t* st, int64_t cap, int64_t* total) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->cell_starts(st, cap, total); });
}
OAPI int oracle_get_sigvrmax(void* h, void* out, int64_t cap) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->get_sigvrmax(out, cap); });
}
OAPI int oracle_set_sigvrmax(void* h, const void* in, int64_t n) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->set_sigvrmax(in, n); });
}
OAPI int oracle_set_recording(void* h, int flags) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->set_recording(flags); });
}
OAPI int oracle_get_evaporated(void* h, int cloud, double* pos, double* vel, int32_t* step, int32_t* fate, int64_t cap) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->get_evaporated(cloud, pos, vel, step, fate, cap); });
}
OAPI int oracle_get_cell_collisions(void* h, int32_t* counts, int64_t cap) {
    return oguard((OracleBase*)h, [&] { ((OracleBase*)h)->get_cell_collisions(counts, cap); });
}
OAPI int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
OAPI void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
OAPI int oracle_preset(int which, dsmc_params* run, dsmc_cloud_params* c) { return (int)fill_preset(which, run, c); }

// ---- primitives for unit tests ------------------------------------------------------------
OAPI void oracle_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    u32x4 c{ctr[0], ctr[1], ctr[2], ctr[3]};
    u32x4 r = philox4x32_10(c, key[0], key[1]);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}
// which: 0 sin, 1 cos, 2 log, 3 exp, 4 rsqrt
OAPI void oracle_math_f(int which, const float* x, float* y, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        float s, c;
        switch (which) {
        case 0: xsincos(x[i], &s, &c); y[i] = s; break;
        case 1: xsincos(x[i], &s, &c); y[i] = c; break;
        case 2: y[i] = xlog(x[i]); break;
        case 3: y[i] = xexp(x[i]); break;
        default: y[i] = xrsqrt(x[i]); break;
        }
    }
}
// the diagnostics' fixed-point conversion of each value (prec DSMC_FP32: the float form, else
// the double form), as (low 64 bits, high 64 bits) pairs
OAPI void oracle_fx(int prec, const void* x, uint64_t* out, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        const i128 q = prec == DSMC_FP32 ? fx_from(((const float*)x)[i]) : fx_from(((const double*)x)[i]);
        out[2 * i] = (uint64_t)q;
        out[2 * i + 1] = (uint64_t)((unsigned __int128)q >> 64);
    }
}
OAPI void oracle_math_d(int which, const double* x, double* y, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        double s, c;
        switch (which) {
        case 0: xsincos(x[i], &s, &c); y[i] = s; break;
        case 1: xsincos(x[i], &s, &c); y[i] = c; break;
        case 2: y[i] = xlog(x[i]); break;
        case 3: y[i] = xexp(x[i]); break;
        default: y[i] = xrsqrt(x[i]); break;
        }
    }
}
// trap field at n points for one cloud: out[7i..] = B^x, B^y, B^z, |B|, dB/dx, dB/dy, dB/dz
OAPI int oracle_field_d(const dsmc_params* run, const dsmc_cloud_params* c, const double* xyz, double* out, int64_t n) {
    CloudPhys<double> P;
    make_cloud_phys<double>(*run, *c, 0, 0, P);
    for (int64_t i = 0; i < n; ++i) {
        Field<double> f;
        trap_field(P, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], f);
        double* o = out + 7 * i;
        o[0] = f.bx; o[1] = f.by; o[2] = f.bz; o[3] = f.absB; o[4] = f.gx; o[5] = f.gy; o[6] = f.gz;
    }
    return 0;
}
// advance n atoms by nsteps (Larmor + Verlet + evaporation tests, no collisions, no sort) in
// FP64: the per-atom part of the step, for comparison with the reference's own kernels.
// fate[i] receives the fate after the last step (0 alive, 1 Majorana, 2 knife).
OAPI int oracle_advance_atoms_d(const dsmc_params* run, const dsmc_cloud_params* c, double* pos, double* vel,
                                double* psi, int32_t* fate, int64_t n, int nsteps) {
    CloudPhys<double> P;
    make_cloud_phys<double>(*run, *c, 0, 0, P);
    for (int64_t i = 0; i < n; ++i) {
        Atom<double> a;
        a.x = pos[4 * i]; a.y = pos[4 * i + 1]; a.z = pos[4 * i + 2];
        a.vx = vel[4 * i]; a.vy = vel[4 * i + 1]; a.vz = vel[4 * i + 2];
        a.ur = psi[4 * i]; a.ui = psi[4 * i + 1]; a.dr = psi[4 * i + 2]; a.di = psi[4 * i + 3];
        a.flags = lane_to_u32(vel[4 * i + 3]);
        AtomOut<double> o;
        o.fate = FATE_ALIVE;
        StepCtx sc = {};
        for (int s = 0; s < nsteps; ++s) advance_atom(P, 0.0, a, o, sc);
        pos[4 * i] = a.x; pos[4 * i + 1] = a.y; pos[4 * i + 2] = a.z;
        vel[4 * i] = a.vx; vel[4 * i + 1] = a.vy; vel[4 * i + 2] = a.vz;
        psi[4 * i] = a.ur; psi[4 * i + 1] = a.ui; psi[4 * i + 2] = a.dr; psi[4 * i + 3] = a.di;
        if (fate) fate[i] = o.fate;
    }
    return 0;
}

// one timestep of n atoms (Larmor, Verlet, Majorana and knife tests, new cell; no collisions, no
// sort) in FP64 with the knife cut cut_v2 in units of v^2 (2 eta kB T / m): for the restatement of
// the step in the tests.  fate[i] 0 alive, 1 Majorana, 2 knife; cell[i] the atom's new cell.
OAPI int oracle_step_atoms_d(const dsmc_params* run, const dsmc_cloud_params* c, double* pos, double* vel,
                             double* psi, double cut_v2, int32_t* fate, int32_t* cell, int64_t n) {
    CloudPhys<double> P;
    make_cloud_phys<double>(*run, *c, 0, 0, P);
    for (int64_t i = 0; i < n; ++i) {
        Atom<double> a;
        a.x = pos[4 * i]; a.y = pos[4 * i + 1]; a.z = pos[4 * i + 2];
        a.vx = vel[4 * i]; a.vy = vel[4 * i + 1]; a.vz = vel[4 * i + 2];
        a.ur = psi[4 * i]; a.ui = psi[4 * i + 1]; a.dr = psi[4 * i + 2]; a.di = psi[4 * i + 3];
        a.flags = lane_to_u32(vel[4 * i + 3]);
        AtomOut<double> o;
        StepCtx sc = {};
        advance_atom(P, cut_v2, a, o, sc);
        pos[4 * i] = a.x; pos[4 * i + 1] = a.y; pos[4 * i + 2] = a.z;
        vel[4 * i] = a.vx; vel[4 * i + 1] = a.vy; vel[4 * i + 2] = a.vz;
        psi[4 * i] = a.ur; psi[4 * i + 1] = a.ui; psi[4 * i + 2] = a.dr; psi[4 * i + 3] = a.di;
        fate[i] = o.fate;
        cell[i] = o.cell;
    }
    return 0;
}

namespace {
// records the accepted collisions of one cell: pair (i, j) and direction n^
struct ArrayCollisionLog {
    int32_t* ij;
    double* nv;
    int cap;
    int count;
    template <class R> void accept(uint32_t i, uint32_t j, R nx, R ny, R nz) {
        if (count < cap) {
            ij[2 * count] = (int32_t)i; ij[2 * count + 1] = (int32_t)j;
            nv[3 * count] = (double)nx; nv[3 * count + 1] = (double)ny; nv[3 * count + 2] = (double)nz;
        }
        ++count;
    }
};
}  // namespace

// the NTC collisions of one grid cell of n atoms in FP64 (vel: n x 4, updated in place; sigvrmax
// in/out), the cell's local index and the step keying its random numbers; the accepted pairs and
// their scattering directions go to ij / nv (up to log_cap).  Returns the accepted count.
OAPI int oracle_collide_cell_d(const dsmc_params* run, const dsmc_cloud_params* c, double* vel, int32_t n,
                               double* sigvrmax, uint32_t local_cell, uint32_t step, int32_t* candidates,
                               int32_t* ij, double* nv, int32_t log_cap) {
    CloudPhys<double> P;
    make_cloud_phys<double>(*run, *c, 0, 0, P);
    ArrayCollisionLog lg{ij, nv, log_cap, 0};
    Q4<double>* v = reinterpret_cast<Q4<double>*>(vel);
    const CollideResult<double> r =
        collide_cell<double, Q4<double>*, ArrayCollisionLog>(v, n, *sigvrmax, P, local_cell, step, run->seed, &lg);
    *candidates = r.candidates;
    return r.accepted;
}

// MCWF period end (flip + decoherence + renormalisation) of each atom at its position, in FP64:
// x0 = the trapped population recorded at the period start; flags bit 0 = anti-trapped on input
// and output; ids and step key the flip's random number.
OAPI int oracle_mcwf_end_d(const dsmc_params* run, const dsmc_cloud_params* c, const double* pos, double* vel,
                           double* psi, const double* x0, uint32_t* flags, const uint32_t* ids, int32_t step,
                           int64_t n) {
    CloudPhys<double> P;
    make_cloud_phys<double>(*run, *c, 0, 0, P);
    for (int64_t i = 0; i < n; ++i) {
        Atom<double> a;
        a.x = pos[3 * i]; a.y = pos[3 * i + 1]; a.z = pos[3 * i + 2];
        a.vx = vel[3 * i]; a.vy = vel[3 * i + 1]; a.vz = vel[3 * i + 2];
        a.ur = psi[4 * i]; a.ui = psi[4 * i + 1]; a.dr = psi[4 * i + 2]; a.di = psi[4 * i + 3];
        a.flags = mcwf_store(flags[i] & 1u, x0[i]);
        Field<double> f;
        trap_field(P, a.x, a.y, a.z, f);
        StepCtx sc;
        sc.id = ids[i]; sc.step = (uint32_t)step; sc.cloud = (uint32_t)P.cloud_id; sc.mcwf = 2u; sc.seed = run->seed;
        mcwf_end(P, f, a, sc);
        vel[3 * i] = a.vx; vel[3 * i + 1] = a.vy; vel[3 * i + 2] = a.vz;
        psi[4 * i] = a.ur; psi[4 * i + 1] = a.ui; psi[4 * i + 2] = a.dr; psi[4 * i + 3] = a.di;
        flags[i] = a.flags & 1u;
    }
    return 0;
}

// ---- smoothed model (gradient path) ---------------------------------------------------------
// theta = (B', B0, eta_0 .. eta_8); x, v: n x 3 and psi: n x 4 in atom-id order; log_off: steps +
// 1 offsets into the recorded collisions (pairs log_ij, directions log_n).  Returns the smoothed
// loss L_E + L_N (parts[0] = L_E, parts[1] = L_N) and, if grad_e / grad_n are not null, the
// gradients of each part by the hand-written adjoint (all states stored, serial).
#include "dsmc_adjoint.h"

namespace {
template <class R>
SmoothConsts<R> smooth_consts(const dsmc_params& run, const dsmc_cloud_params& c, const double* theta, double width_kT,
                              double maj_width) {
    const double kB = run_kB(run);
    SmoothConsts<R> C;
    C.Bp = (R)theta[0];
    C.B0 = (R)theta[1];
    C.B_floor = (R)0;
    C.dt = (R)run.dt;
    C.half_dt = (R)(0.5 * run.dt);
    C.accel_scale = (R)(c.moment / c.mass);
    C.kappa = (R)(2.0 * c.moment / c.mass);
    C.inv_width = (R)(1.0 / (2.0 * width_kT * kB * c.temperature / c.mass));
    C.theta_per_B = (c.flags & DSMC_F_LARMOR) ? (R)(c.moment * run.dt / run_hbar(run)) : (R)0;
    C.inv_width_maj = ((c.flags & DSMC_F_MAJORANA) && maj_width > 0) ? (R)(1.0 / maj_width) : (R)0;
    C.cut_scale = 2.0 * kB * c.temperature / c.mass;
    return C;
}

template <class R>
void smooth_run(const dsmc_params& run, const dsmc_cloud_params& c, const double* theta, double width_kT,
                double maj_width, const double* x0, const double* v0, const double* p0, int64_t n, int steps,
                const int* off, const int* ij, const double* ln, double* parts, double* grad_e, double* grad_n) {
    const SmoothConsts<R> C = smooth_consts<R>(run, c, theta, width_kT, maj_width);
    const int nk = c.knife_nknots;
    const double kB = run_kB(run);
    std::vector<R> x(3 * n), v(3 * n), ps(4 * n), w(n, R(1)), e(n);
    for (int64_t i = 0; i < 3 * n; ++i) { x[i] = (R)x0[i]; v[i] = (R)v0[i]; }
    for (int64_t i = 0; i < 4 * n; ++i) ps[i] = (R)p0[i];
    const bool keep = grad_e != nullptr || grad_n != nullptr;
    // per step: start x, post-collision v, start psi and w; pre-collision pairs
    std::vector<R> xs, vs, pss, ws, vpre;
    if (keep) { xs.resize((size_t)steps * 3 * n); vs.resize((size_t)steps * 3 * n); pss.resize((size_t)steps * 4 * n);
                ws.resize((size_t)steps * n); vpre.resize((size_t)off[steps] * 6); }
    std::vector<double> cuts(steps);
    for (int t = 0; t < steps; ++t) {
        for (int k = off[t]; k < off[t + 1]; ++k) {
            R* vi = &v[3 * ij[2 * k]];
            R* vj = &v[3 * ij[2 * k + 1]];
            if (keep) for (int a = 0; a < 3; ++a) { vpre[6 * k + a] = vi[a]; vpre[6 * k + 3 + a] = vj[a]; }
            const R nn[3] = {(R)ln[3 * k], (R)ln[3 * k + 1], (R)ln[3 * k + 2]};
            collide_fixed(vi, vj, nn);
        }
        const double eta = knife_eta(nk, c.knife_step, theta + 2, (double)t);
        const R cut = (R)(C.cut_scale * eta);
        cuts[t] = (double)cut;
        if (keep) {
            memcpy(&xs[(size_t)t * 3 * n], x.data(), 3 * n * sizeof(R));
            memcpy(&vs[(size_t)t * 3 * n], v.data(), 3 * n * sizeof(R));
            memcpy(&pss[(size_t)t * 4 * n], ps.data(), 4 * n * sizeof(R));
            memcpy(&ws[(size_t)t * n], w.data(), n * sizeof(R));
        }
        for (int64_t i = 0; i < n; ++i) e[i] = smooth_step(C, cut, &x[3 * i], &v[3 * i], &ps[4 * i], w[i]);
    }
    i128 W = 0, S = 0;
    for (int64_t i = 0; i < n; ++i) {
        W += fx_from((double)w[i]);
        S += fx_from((double)w[i] * (double)e[i]);
    }
    const double Wd = fx_to_double(W), Sd = fx_to_double(S), kT = kB * c.temperature;
    parts[0] = 0.5 * c.mass * Sd / Wd / kT;
    parts[1] = Wd / (double)n;
    if (!keep) return;
    // adjoint seeds at the final state: 0 = L_E, 1 = L_N
    std::vector<R> xb(ADJ_SEEDS * 3 * n, R(0)), vb(ADJ_SEEDS * 3 * n, R(0)), pb(ADJ_SEEDS * 4 * n, R(0)),
        wb(ADJ_SEEDS * n, R(0));
    double th[ADJ_SEEDS][ADJ_NPARAM] = {{0}};
    for (int64_t i = 0; i < n; ++i) {
        const double dEdw = 0.5 * c.mass * ((double)e[i] / Wd - Sd / (Wd * Wd)) / kT;
        const double dEde = 0.5 * c.mass * (double)w[i] / (Wd * kT);
        QuadField<R> f;
        quad_field(C.Bp, C.B0, x[3 * i], x[3 * i + 1], x[3 * i + 2], true, f);
        for (int a = 0; a < 3; ++a) {
            xb[3 * i + a] = (R)(dEde * (double)C.kappa * (double)f.g[a]);
            vb[3 * i + a] = (R)(dEde * 2.0 * (double)v[3 * i + a]);
        }
        wb[i] = (R)dEdw;
        wb[n + i] = (R)(1.0 / (double)n);
        th[0][0] += dEde * (double)C.kappa * (double)f.dabs_dBp;
        th[0][1] += dEde * (double)C.kappa * (double)f.dabs_dB0;
    }
    for (int t = steps - 1; t >= 0; --t) {
        const R cut = (R)cuts[t];
        double cutb_sum[ADJ_SEEDS] = {0, 0};
        for (int64_t i = 0; i < n; ++i) {
            R axb[ADJ_SEEDS][3], avb[ADJ_SEEDS][3], apb[ADJ_SEEDS][4], awb[ADJ_SEEDS], tb[ADJ_SEEDS][2], cb[ADJ_SEEDS];
            for (int q = 0; q < ADJ_SEEDS; ++q) {
                for (int a = 0; a < 3; ++a) { axb[q][a] = xb[(q * n + i) * 3 + a]; avb[q][a] = vb[(q * n + i) * 3 + a]; }
                for (int a = 0; a < 4; ++a) apb[q][a] = pb[(q * n + i) * 4 + a];
                awb[q] = wb[q * n + i];
                tb[q][0] = tb[q][1] = R(0);
                cb[q] = R(0);
            }
            smooth_step_adjoint(C, cut, &xs[(size_t)t * 3 * n + 3 * i], &vs[(size_t)t * 3 * n + 3 * i],
                                &pss[(size_t)t * 4 * n + 4 * i], ws[(size_t)t * n + i], axb, avb, apb, awb, tb, cb);
            for (int q = 0; q < ADJ_SEEDS; ++q) {
                for (int a = 0; a < 3; ++a) { xb[(q * n + i) * 3 + a] = axb[q][a]; vb[(q * n + i) * 3 + a] = avb[q][a]; }
                for (int a = 0; a < 4; ++a) pb[(q * n + i) * 4 + a] = apb[q][a];
                wb[q * n + i] = awb[q];
                th[q][0] += (double)tb[q][0];
                th[q][1] += (double)tb[q][1];
                cutb_sum[q] += (double)cb[q];
            }
        }
        int k0;
        double f;
        knot_weights(nk, c.knife_step, (double)t, &k0, &f);
        for (int q = 0; q < ADJ_SEEDS; ++q) {
            th[q][2 + k0] += cutb_sum[q] * C.cut_scale * (1.0 - f);
            if (f != 0.0) th[q][2 + k0 + 1] += cutb_sum[q] * C.cut_scale * f;
        }
        for (int k = off[t + 1] - 1; k >= off[t]; --k) {
            const R nn[3] = {(R)ln[3 * k], (R)ln[3 * k + 1], (R)ln[3 * k + 2]};
            for (int q = 0; q < ADJ_SEEDS; ++q)
                collide_fixed_adjoint(&vpre[6 * k], &vpre[6 * k + 3], nn, &vb[(q * n + ij[2 * k]) * 3],
                                      &vb[(q * n + ij[2 * k + 1]) * 3]);
        }
    }
    for (int p = 0; p < ADJ_NPARAM; ++p) {
        if (grad_e) grad_e[p] = th[0][p];
        if (grad_n) grad_n[p] = th[1][p];
    }
}
}  // namespace

// The smoothed loss of a recorded run (L_E + L_N; parts[0..1] = L_E, L_N) and the gradient of each
// part (grad_e, grad_n: 11 doubles each, or null).  psi holds the initial spinors by atom id;
// maj_width is the width of the Majorana survival sigmoid in <s.B^> (used when the cloud has
// Majorana loss).
OAPI double oracle_smooth_loss(const dsmc_params* run, const dsmc_cloud_params* c, const double* theta,
                               double width_kT, double maj_width, const double* x, const double* v, const double* psi,
                               int64_t n, int steps, const int* off, const int* ij, const double* ln, double* parts,
                               double* grad_e, double* grad_n, int fp64) {
    if (fp64) smooth_run<double>(*run, *c, theta, width_kT, maj_width, x, v, psi, n, steps, off, ij, ln, parts, grad_e, grad_n);
    else smooth_run<float>(*run, *c, theta, width_kT, maj_width, x, v, psi, n, steps, off, ij, ln, parts, grad_e, grad_n);
    return parts[0] + parts[1];
}
