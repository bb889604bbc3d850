// Host build of CUDADSMC/src/moveAtoms.cu (velocity Verlet in the Ioffe-Pritchard field),
// compiled from the reference tree in place; extern "C" entry points for the tests.
#include "cuda.h"
ref_dim3 blockIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1}, threadIdx = {0, 0, 0};
#include "moveAtoms.cu"

extern "C" {
void ref_set_dt(double dt) { copyConstantsToDevice(dt); }
void ref_update_acc(const double* pos, double* acc, int n) {
    for (int i = 0; i < n; ++i) {
        double3 a = updateAcc(make_double3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), true);
        acc[3 * i] = a.x; acc[3 * i + 1] = a.y; acc[3 * i + 2] = a.z;
    }
}
void ref_move_atoms(double* pos, double* vel, double* acc, hbool_t* spin_up, int* atom_id, int n) {
    moveAtoms((double3*)pos, (double3*)vel, (double3*)acc, spin_up, atom_id, n);
}
}
