// driver.cpp -- command-line driver with the call structure of CUDADSMC's main()
// (CUDADSMC/src/main.cu:36-619), running the B200 engine through the C ABI (include/dsmc.h).
//
//   dsmc_driver [Nc N] [--preset K] [--steps-per-print S] [--prints P] [--loops-per-collision L]
//               [--mcwf] [--fp64] [--out DIR] [--seed X]
//
// As in the reference: argv "Nc N" picks Nc^3 cells and N test atoms (main.cu:45-69), alpha is
// 3e6 / N real atoms per test atom (main.cu:53, initialSystemParameters.cuh:27), the cloud is
// initialised (main.cu:176-198), then numberOfPrints times the loop body runs
// collisionsPerPrint x loopsPerCollision motion steps (main.cu:410-524) and a snapshot is
// written (main.cu:526-577).  Snapshots replace the HDF5 file /atomData/* with one .npy file
// per dataset and frame in DIR (positions, velocities, psiUp, psiDn, atomID, atomIsSpinUp,
// cellID, atomCount, atomNumber, simuatedTime, evapPos, evapVel, collisionCount) -- the names
// of the reference datasets; cudadsmc_b200.snapshots.read_snapshots stacks the frames into the
// reference's (N, k, t) arrays.
// --loops-per-collision is the reference's loopsPerCollision (main.cu:168: motion steps per
// collision step, the engine's collide_every); --mcwf turns on the spin-flip and decoherence
// path that the reference runs once per collision step (main.cu:501-520).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <sys/stat.h>

#include "dsmc.h"

namespace {

bool check(dsmc_status st, dsmc_handle* h, const char* what) {
    if (st == DSMC_OK) return true;
    std::fprintf(stderr, "%s failed: %s (%s)\n", what, dsmc_status_string(st), dsmc_last_error(h));
    return false;
}

// minimal .npy writer (format version 1.0, little-endian, C order)
void write_npy(const std::string& path, const char* descr, const std::vector<long>& shape, const void* data,
               size_t bytes) {
    std::string sh = "(";
    for (size_t i = 0; i < shape.size(); ++i) sh += std::to_string(shape[i]) + (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
    sh += ")";
    std::string hdr = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': " + sh + ", }";
    size_t total = 10 + hdr.size() + 1;
    size_t pad = (64 - total % 64) % 64;
    hdr += std::string(pad, ' ') + "\n";
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); return; }
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    std::fwrite(magic, 1, 8, f);
    uint16_t hl = (uint16_t)hdr.size();
    std::fwrite(&hl, 2, 1, f);
    std::fwrite(hdr.data(), 1, hdr.size(), f);
    std::fwrite(data, 1, bytes, f);
    std::fclose(f);
}

template <class R>
void snapshot(dsmc_handle* h, const std::string& dir, int frame, int64_t cap, const dsmc_diag& d) {
    std::vector<R> pos(4 * cap), vel(4 * cap), psi(4 * cap);
    std::vector<int64_t> counts(1);
    dsmc_state_buffers b{pos.data(), vel.data(), psi.data(), cap, counts.data()};
    if (!check(dsmc_get_state(h, &b), h, "dsmc_get_state")) return;
    const long n = (long)b.n;
    int64_t ncells = 0;
    dsmc_get_cell_starts(h, nullptr, 0, &ncells);
    std::vector<int32_t> start(ncells + 1);
    dsmc_get_cell_starts(h, start.data(), ncells + 1, &ncells);
    std::vector<double> p3(3 * n), v3(3 * n), up(2 * n), dn(2 * n);
    std::vector<int32_t> id(n), cell(n), count(ncells);
    std::vector<uint8_t> spin_up(n);
    for (long i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            p3[3 * i + a] = pos[4 * i + a];
            v3[3 * i + a] = vel[4 * i + a];
        }
        up[2 * i] = psi[4 * i]; up[2 * i + 1] = psi[4 * i + 1];
        dn[2 * i] = psi[4 * i + 2]; dn[2 * i + 1] = psi[4 * i + 3];
        uint64_t bits = 0;
        std::memcpy(&bits, &pos[4 * i + 3], sizeof(R));
        id[i] = (int32_t)(uint32_t)bits;
        bits = 0;
        std::memcpy(&bits, &vel[4 * i + 3], sizeof(R));
        spin_up[i] = (bits & 1u) ? 0 : 1;  // flag bit 0: anti-trapped
    }
    for (int64_t c = 0; c < ncells; ++c) {
        count[c] = start[c + 1] - start[c];
        for (int32_t i = start[c]; i < start[c + 1]; ++i) cell[i] = (int32_t)c;
    }
    const std::string f = "_" + std::to_string(frame) + ".npy";
    write_npy(dir + "/positions" + f, "<f8", {n, 3}, p3.data(), p3.size() * 8);
    write_npy(dir + "/velocities" + f, "<f8", {n, 3}, v3.data(), v3.size() * 8);
    write_npy(dir + "/psiUp" + f, "<f8", {n, 2}, up.data(), up.size() * 8);
    write_npy(dir + "/psiDn" + f, "<f8", {n, 2}, dn.data(), dn.size() * 8);
    write_npy(dir + "/atomID" + f, "<i4", {n}, id.data(), id.size() * 4);
    write_npy(dir + "/atomIsSpinUp" + f, "|u1", {n}, spin_up.data(), spin_up.size());
    write_npy(dir + "/cellID" + f, "<i4", {n}, cell.data(), cell.size() * 4);
    write_npy(dir + "/atomCount" + f, "<i4", {(long)ncells}, count.data(), count.size() * 4);
    int32_t number = (int32_t)n;
    write_npy(dir + "/atomNumber" + f, "<i4", {1}, &number, 4);
    write_npy(dir + "/simuatedTime" + f, "<f8", {1}, &d.time, 8);
    // evaporated atoms by atom id (zeros for atoms not lost) and the last collision step's counts
    std::vector<double> ep(3 * cap), evl(3 * cap);
    if (check(dsmc_get_evaporated(h, 0, ep.data(), evl.data(), nullptr, nullptr, cap), h, "dsmc_get_evaporated")) {
        write_npy(dir + "/evapPos" + f, "<f8", {(long)cap, 3}, ep.data(), ep.size() * 8);
        write_npy(dir + "/evapVel" + f, "<f8", {(long)cap, 3}, evl.data(), evl.size() * 8);
    }
    std::vector<int32_t> coll(ncells);
    if (check(dsmc_get_cell_collisions(h, coll.data(), ncells, &ncells), h, "dsmc_get_cell_collisions"))
        write_npy(dir + "/collisionCount" + f, "<i4", {(long)ncells}, coll.data(), coll.size() * 4);
}

}  // namespace

int main(int argc, char** argv) {
    int Nc = -1;
    long N = -1;
    int preset = 0, prints = 10, steps_per_print = 100, loops_per_collision = 0;
    bool fp64 = false, mcwf = false;
    std::string out;
    uint64_t seed = 1234;
    std::vector<std::string> pos_args;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--preset" && i + 1 < argc) preset = std::atoi(argv[++i]);
        else if (a == "--prints" && i + 1 < argc) prints = std::atoi(argv[++i]);
        else if (a == "--steps-per-print" && i + 1 < argc) steps_per_print = std::atoi(argv[++i]);
        else if (a == "--fp64") fp64 = true;
        else if (a == "--mcwf") mcwf = true;
        else if (a == "--loops-per-collision" && i + 1 < argc) loops_per_collision = std::atoi(argv[++i]);
        else if (a == "--out" && i + 1 < argc) out = argv[++i];
        else if (a == "--seed" && i + 1 < argc) seed = std::strtoull(argv[++i], nullptr, 10);
        else pos_args.push_back(a);
    }
    if (pos_args.size() == 2) {  // main.cu:55-64
        Nc = std::atoi(pos_args[0].c_str());
        N = std::atol(pos_args[1].c_str());
    } else if (!pos_args.empty()) {
        std::printf("Too many arguments supplied.\n");  // main.cu:65-69
        return 0;
    }
    dsmc_params run;
    dsmc_cloud_params cloud;
    if (dsmc_preset(preset, &run, &cloud) != DSMC_OK) {
        std::fprintf(stderr, "unknown preset %d\n", preset);
        return 1;
    }
    if (Nc > 0) cloud.cells[0] = cloud.cells[1] = cloud.cells[2] = Nc;
    if (N >= 0) {
        cloud.n_atoms = cloud.capacity = N;
        cloud.alpha = N > 0 ? 3e6 / (double)N : 1.0;  // alpha = h_N / N (main.cu:53)
    }
    if (fp64) run.precision = DSMC_FP64;
    if (loops_per_collision > 0) run.collide_every = loops_per_collision;
    if (mcwf) cloud.flags |= DSMC_F_MCWF;
    dsmc_handle* h = nullptr;
    if (!check(dsmc_create(&run, &cloud, 1, &h), nullptr, "dsmc_create")) return 1;
    if (!check(dsmc_init_cloud(h, seed), h, "dsmc_init_cloud")) return 1;
    if (!out.empty()) {
        mkdir(out.c_str(), 0755);
        // the evapPos / evapVel / collisionCount datasets need the step's records
        if (!check(dsmc_set_recording(h, DSMC_REC_EVAPORATED | DSMC_REC_CELL_COLLISIONS), h, "dsmc_set_recording"))
            return 1;
    }
    dsmc_diag d;
    dsmc_diagnostics(h, -1, &d);
    const double e0 = d.e_kin + d.e_pot;
    auto report = [&](int i) {
        std::printf("{\"print\": %d, \"step\": %lld, \"t\": %.9g, \"N\": %lld, \"T_uK\": %.6f, \"E_drift\": %.3e, "
                    "\"collisions\": %lld, \"evaporated\": %lld, \"majorana\": %lld, \"error\": %d}\n",
                    i, (long long)d.step, d.time, (long long)d.n_alive, d.temperature * 1e6,
                    (d.e_kin + d.e_pot + d.e_evaporated - e0) / e0, (long long)d.collisions,
                    (long long)d.n_evaporated, (long long)d.n_majorana, d.error);
        std::fflush(stdout);
    };
    report(0);
    if (!out.empty()) {
        if (run.precision == DSMC_FP32) snapshot<float>(h, out, 0, cloud.capacity, d);
        else snapshot<double>(h, out, 0, cloud.capacity, d);
    }
    for (int i = 1; i <= prints; ++i) {
        if (!check(dsmc_step(h, steps_per_print), h, "dsmc_step")) return 1;
        if (!check(dsmc_diagnostics(h, -1, &d), h, "dsmc_diagnostics")) return 1;
        report(i);
        if (!out.empty()) {
            if (run.precision == DSMC_FP32) snapshot<float>(h, out, i, cloud.capacity, d);
            else snapshot<double>(h, out, i, cloud.capacity, d);
        }
    }
    dsmc_destroy(h);
    return d.error ? 2 : 0;
}
