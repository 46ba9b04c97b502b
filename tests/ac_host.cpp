// Test harness only: the AC lanes' complex replay and solves
// (egspice_b200/csrc/lane_ac_core.cuh, __host__ __device__) with the host
// tape builder (egspice_b200/csrc/tape.cpp) compiled for the host, laid out
// as the kernel lays them: lanes interleaved with stride P, the tape from
// lane 0's |G| + w_c |C| at the geometric centre frequency (as espl_ac_solve
// builds it). Returns 0, or 1 when the tape cannot be built.
#define __host__
#define __device__

#include <algorithm>
#include <cmath>
#include <vector>

#include "../egspice_b200/csrc/lane_ac_core.cuh"
#include "../egspice_b200/csrc/tape.h"

extern "C" int dev_ac(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, uint32_t P, const double* g,
                      const double* c, const double* omega, uint32_t n_freq, const double* b_re, const double* b_im,
                      uint32_t n_rhs, uint32_t adjoint, const uint32_t* rows, uint32_t n_rows, double* out_re,
                      double* out_im) {
    using namespace espl;
    const uint32_t nnz = col_ptr[n];
    std::vector<uint32_t> q;
    if (!order_columns(n, col_ptr, row_idx, q)) return 1;
    double lo = INFINITY, hi = 0.0;
    for (uint32_t f = 0; f < n_freq; f++) {
        if (omega[f] > 0.0) lo = std::min(lo, omega[f]);
        hi = std::max(hi, omega[f]);
    }
    const double wc = hi > 0.0 ? std::sqrt(lo * hi) : 0.0;
    std::vector<double> proxy(nnz);
    for (uint32_t p = 0; p < nnz; p++) proxy[p] = std::fabs(g[(size_t)p * P]) + wc * std::fabs(c[(size_t)p * P]);
    Tape t;
    if (!factor_tape(n, col_ptr, row_idx, proxy.data(), q, t) || !t.void_slots.empty()) return 1;
    std::vector<uint32_t> qinv(n);
    for (uint32_t j = 0; j < n; j++) qinv[t.q[j]] = j;
    const size_t nl = std::max<size_t>(t.li.size(), 1), nu = std::max<size_t>(t.ui.size(), 1);
    std::vector<double> ar(nnz * P), ai(nnz * P), wr(n * P, 0.0), wi(n * P, 0.0), lr(nl * P), li(nl * P),
        ur(nu * P), ui(nu * P), dr(n * P), di(n * P);
    const AcTape T{t.q.data(), qinv.data(), t.pinv.data(), t.prow.data(), t.lp.data(), t.li.data(),
                   t.up.data(),  t.ui.data(),  col_ptr,       n,           nnz};
    for (uint32_t l = 0; l < P; l++) {
        const AcWork W{ar.data(), ai.data(), wr.data(), wi.data(), lr.data(), li.data(),
                       ur.data(), ui.data(), dr.data(), di.data(), P,         l};
        for (uint32_t f = 0; f < n_freq; f++) {
            const bool ok = ac_factor(T, W, g, c, omega[f]);
            for (uint32_t e = 0; e < n_rhs; e++) {
                ac_solve(T, W, b_re + (size_t)e * n, b_im + (size_t)e * n, adjoint != 0);
                const size_t o = (((size_t)l * n_freq + f) * n_rhs + e) * n_rows;
                for (uint32_t k = 0; k < n_rows; k++) {
                    double re, im;
                    ac_value(T, W, adjoint != 0, rows[k], re, im);
                    out_re[o + k] = ok ? re : NAN;
                    out_im[o + k] = ok ? im : NAN;
                }
                ac_clear(T, W);
            }
        }
    }
    return 0;
}
