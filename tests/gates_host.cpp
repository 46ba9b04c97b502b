// Test harness only: the kernels' residual gate
// (egspice_b200/csrc/lane_gates.cuh, __host__ __device__) compiled for the
// host, so the CPU tests check it against the reference's known answers and
// the oracle.
#define __host__
#define __device__

#include "../egspice_b200/csrc/lane_gates.cuh"

extern "C" double dev_residual_gate(double residual_tol, double reltol, double vntol, double diag, double xi) {
    return espl::residual_gate(residual_tol, reltol, vntol, diag, xi);
}
