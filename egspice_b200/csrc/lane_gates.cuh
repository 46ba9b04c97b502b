// Newton's per-row residual gate (src/solver/converger.zig residualGate
// :340-350, run per lane by src/solver/kernels/lane.zig residual :189-198):
// row i passes when |F_i| <= max(residual_tol, 10 s (reltol |x_i| + vntol)),
// s = |A_ii|, or 1 where the diagonal is zero (a voltage-defined branch
// row). fmax returns the other operand when one is NaN, as the reference's
// @max does.
#pragma once

#include <cmath>

namespace espl {

__host__ __device__ inline double residual_gate(double residual_tol, double reltol, double vntol, double diag,
                                                double xi) {
    const double scale = fabs(diag);
    const double s = scale == 0.0 ? 1.0 : scale;
    return fmax(residual_tol, 10.0 * s * (reltol * fabs(xi) + vntol));
}

}  // namespace espl
