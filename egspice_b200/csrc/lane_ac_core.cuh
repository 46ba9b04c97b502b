// One AC lane's complex work, host and device alike (the kernel k_ac runs it
// per lane; the tests build it for the host): the replay of a real pivot
// tape on Y = G + jwC with the infinity-norm pivot check and reciprocal
// pivots (the reference's ComplexLaneLu, src/solver/lane/clu.zig), then
// solves of Y x = b or of the transpose Y^T z = b (the adjoint solve the
// reference's frequency lanes run for noise, src/analysis/gpu/freq.zig
// `adjoint`). Arrays are lane-interleaved: element i of lane l at i * P + l.
//
// With the tape's row order pinv, column order q, unit-lower L and upper U
// (diagonal d): P Y Q = L U. So Y x = b is L U w = P b, x = Q w, and
// Y^T z = b is U^T L^T (P z) = Q^T b: forward over U^T (U's columns as
// dot products, then times 1/d), back over L^T (L's columns as dot
// products), z[r] = t[pinv[r]].
#pragma once

#include <cmath>
#include <cstdint>

namespace espl {

// The tape of an AC replay (tape.h Tape) and the template's pattern.
struct AcTape {
    const uint32_t *q, *qinv, *pinv, *prow, *lp, *li, *up, *ui, *col_ptr;
    uint32_t n, nnz;
};

// One lane's complex scratch: A's values, the work vector, L, U, 1/d.
struct AcWork {
    double *ar, *ai, *wr, *wi, *lr, *li, *ur, *ui, *dr, *di;
    uint32_t P, l;
};

#define ACW(arr, i) (arr)[(size_t)(i) * W.P + W.l]

// Factors Y = g + j om c (g, c: the lane's G and C in pattern order, stride
// P); false when a pivot fails the check (zero, non-finite, or below 1e-12
// of its column under max(|re|, |im|)). The work vector is zero on return.
__host__ __device__ inline bool ac_factor(const AcTape& T, const AcWork& W, const double* g, const double* c,
                                          double om) {
    const double growth = 1e-12;
    for (uint32_t p = 0; p < T.nnz; p++) {
        ACW(W.ar, p) = ACW(g, p);
        ACW(W.ai, p) = om * ACW(c, p);
    }
    bool bad = false;
    for (uint32_t k = 0; k < T.n; k++) {
        const uint32_t col = T.q[k];
        for (uint32_t p = T.col_ptr[col]; p < T.col_ptr[col + 1]; p++) {
            ACW(W.wr, T.prow[p]) = ACW(W.ar, p);
            ACW(W.wi, T.prow[p]) = ACW(W.ai, p);
        }
        for (uint32_t p = T.up[k]; p < T.up[k + 1]; p++) {
            const uint32_t i = T.ui[p];
            const double ur = ACW(W.wr, i), ui = ACW(W.wi, i);
            ACW(W.wr, i) = 0.0;
            ACW(W.wi, i) = 0.0;
            ACW(W.ur, p) = ur;
            ACW(W.ui, p) = ui;
            for (uint32_t pl = T.lp[i]; pl < T.lp[i + 1]; pl++) {
                const uint32_t r = T.li[pl];
                const double lr = ACW(W.lr, pl), li = ACW(W.li, pl);
                ACW(W.wr, r) -= lr * ur - li * ui;
                ACW(W.wi, r) -= lr * ui + li * ur;
            }
        }
        const double pr = ACW(W.wr, k), pi = ACW(W.wi, k);
        ACW(W.wr, k) = 0.0;
        ACW(W.wi, k) = 0.0;
        const double pn = fmax(fabs(pr), fabs(pi));
        double cmax = pn;
        for (uint32_t p = T.lp[k]; p < T.lp[k + 1]; p++) {
            const uint32_t r = T.li[p];
            cmax = fmax(cmax, fmax(fabs(ACW(W.wr, r)), fabs(ACW(W.wi, r))));
        }
        bad |= !(pn > 0.0) || !(pn < INFINITY) || !(pn >= growth * cmax);
        const double den = pr * pr + pi * pi;
        const double rr = bad ? 1.0 : pr / den, ri = bad ? 0.0 : -pi / den;  // 1 / pivot
        ACW(W.dr, k) = rr;
        ACW(W.di, k) = ri;
        for (uint32_t p = T.lp[k]; p < T.lp[k + 1]; p++) {
            const uint32_t r = T.li[p];
            const double vr = ACW(W.wr, r), vi = ACW(W.wi, r);
            ACW(W.wr, r) = 0.0;
            ACW(W.wi, r) = 0.0;
            ACW(W.lr, p) = vr * rr - vi * ri;
            ACW(W.li, p) = vr * ri + vi * rr;
        }
    }
    return !bad;
}

// Solves with the factor of ac_factor for the right-hand side b (dense,
// length n, the same on every lane): Y x = b, or Y^T z = b when `adjoint`.
// The solution stays in the work vector in pivot positions; ac_value reads
// unknown r of it. ac_clear zeroes the work vector afterwards.
__host__ __device__ inline void ac_solve(const AcTape& T, const AcWork& W, const double* br, const double* bi,
                                         bool adjoint) {
    const uint32_t n = T.n;
    if (!adjoint) {
        for (uint32_t r = 0; r < n; r++) {
            ACW(W.wr, T.pinv[r]) = br[r];
            ACW(W.wi, T.pinv[r]) = bi[r];
        }
        for (uint32_t k = 0; k < n; k++) {
            const double ykr = ACW(W.wr, k), yki = ACW(W.wi, k);
            for (uint32_t p = T.lp[k]; p < T.lp[k + 1]; p++) {
                const uint32_t r = T.li[p];
                const double lr = ACW(W.lr, p), li = ACW(W.li, p);
                ACW(W.wr, r) -= lr * ykr - li * yki;
                ACW(W.wi, r) -= lr * yki + li * ykr;
            }
        }
        for (uint32_t k = n; k-- > 0;) {
            const double b_r = ACW(W.wr, k), b_i = ACW(W.wi, k);
            const double dr = ACW(W.dr, k), di = ACW(W.di, k);
            const double zr = b_r * dr - b_i * di, zi = b_r * di + b_i * dr;
            ACW(W.wr, k) = zr;
            ACW(W.wi, k) = zi;
            for (uint32_t p = T.up[k]; p < T.up[k + 1]; p++) {
                const uint32_t r = T.ui[p];
                const double ur = ACW(W.ur, p), ui = ACW(W.ui, p);
                ACW(W.wr, r) -= ur * zr - ui * zi;
                ACW(W.wi, r) -= ur * zi + ui * zr;
            }
        }
        return;
    }
    // U^T s = Q^T b, s[k] = (b[q[k]] - sum_{i<k} U[i,k] s[i]) / d[k]
    for (uint32_t k = 0; k < n; k++) {
        double ar = br[T.q[k]], ai = bi[T.q[k]];
        for (uint32_t p = T.up[k]; p < T.up[k + 1]; p++) {
            const uint32_t i = T.ui[p];
            const double ur = ACW(W.ur, p), ui = ACW(W.ui, p), sr = ACW(W.wr, i), si = ACW(W.wi, i);
            ar -= ur * sr - ui * si;
            ai -= ur * si + ui * sr;
        }
        const double dr = ACW(W.dr, k), di = ACW(W.di, k);
        ACW(W.wr, k) = ar * dr - ai * di;
        ACW(W.wi, k) = ar * di + ai * dr;
    }
    // L^T t = s, t[k] = s[k] - sum_{r>k} L[r,k] t[r]
    for (uint32_t k = n; k-- > 0;) {
        double ar = ACW(W.wr, k), ai = ACW(W.wi, k);
        for (uint32_t p = T.lp[k]; p < T.lp[k + 1]; p++) {
            const uint32_t r = T.li[p];
            const double lr = ACW(W.lr, p), li = ACW(W.li, p), tr = ACW(W.wr, r), ti = ACW(W.wi, r);
            ar -= lr * tr - li * ti;
            ai -= lr * ti + li * tr;
        }
        ACW(W.wr, k) = ar;
        ACW(W.wi, k) = ai;
    }
}

// Unknown r of the last ac_solve: x[r] = w[qinv[r]] (forward) or
// z[r] = t[pinv[r]] (adjoint).
__host__ __device__ inline void ac_value(const AcTape& T, const AcWork& W, bool adjoint, uint32_t r, double& re,
                                         double& im) {
    const uint32_t j = adjoint ? T.pinv[r] : T.qinv[r];
    re = ACW(W.wr, j);
    im = ACW(W.wi, j);
}

__host__ __device__ inline void ac_clear(const AcTape& T, const AcWork& W) {
    for (uint32_t r = 0; r < T.n; r++) {
        ACW(W.wr, r) = 0.0;
        ACW(W.wi, r) = 0.0;
    }
}

#undef ACW

}  // namespace espl
