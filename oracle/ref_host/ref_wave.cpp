// Host build of CUDADSMC/src/wavefunction.cu (Larmor precession, local populations,
// normalisation), compiled from the reference tree in place.
#include "cuda.h"
ref_dim3 blockIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1}, threadIdx = {0, 0, 0};
#include "wavefunction.cu"

extern "C" {
void ref_evolve_wavefunction(double* pos, double* psi_up, double* psi_dn, int* atom_id, int n) {
    evolveWavefunction((double3*)pos, (cuDoubleComplex*)psi_up, (cuDoubleComplex*)psi_dn, atom_id, n);
}
void ref_local_populations(double* pos, double* psi_up, double* psi_dn, double* pops, int* atom_id, int n) {
    getLocalPopulations((double3*)pos, (cuDoubleComplex*)psi_up, (cuDoubleComplex*)psi_dn, (double2*)pops, atom_id, n);
}
void ref_normalise(double* psi_up, double* psi_dn, int* atom_id, int n) {
    normalise((cuDoubleComplex*)psi_up, (cuDoubleComplex*)psi_dn, atom_id, n);
}
}
