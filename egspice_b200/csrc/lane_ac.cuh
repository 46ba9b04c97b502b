// Small-signal AC lanes: every lane linearized at its operating point, its
// response to a unit AC voltage at one source solved at each frequency of a
// list, Y(w) x = e with Y = G + jwC (the reference's frequency-domain lanes,
// src/solver/lane/clu.zig ComplexLaneLu over src/analysis/gpu/freq.zig).
// As there, the complex values replay a real pivot tape laid on the pattern
// (chosen on the host from a real proxy of the moduli, |G| + w_c |C| of the
// lead lane at the centre frequency), each pivot is checked against its
// column under the infinity norm max(|re|, |im|), and pivots are kept as
// reciprocals. A lane and frequency whose pivot check fails reports NaN.
// One thread per lane (warp 0 of the tile); the frequencies loop inside.
#pragma once

#include "lane_tile.cuh"

namespace espl {

#define ACM(arr, i) (arr)[(size_t)(i) * P + l]

// The AC replay's tape (tape.h Tape, uploaded by espl_ac) and the lanes'
// complex scratch, lane-interleaved like every lane array.
struct AcArgs {
    const uint32_t *q, *qinv, *pinv, *prow, *lp, *li, *up, *ui;
    uint32_t n, nnz_l, nnz_u, n_freq, n_rows, exc_row;
    const double* omega;      // n_freq angular frequencies
    const uint32_t* rows;     // n_rows unknowns reported
    const double *g, *c;      // the lanes' G and C at the operating point (nnz x P)
    double *ar, *ai, *wr, *wi, *lr, *li_, *ur, *ui_, *dr, *di;  // complex scratch
    double *out_re, *out_im;  // [lane][freq][row], the template's lanes
};

// G and C of every lane at its x (the limiter state seeded there, so each
// device is linearized at the operating point itself).
__global__ void __launch_bounds__(kTileThreads) k_ac_planes(TileMap m, double* __restrict__ g_out,
                                                            double* __restrict__ c_out) {
    TileCtx c = tile_ctx(m);
    const GroupDev& d = *c.d;
    const uint32_t P = d.P, l = c.l, nw = c.nw;
    const uint32_t ninst = n_instances(d);
    if (c.valid)
        for (uint32_t t = c.warp; t < ninst; t += nw) {
            inst_seed(d, l, t, 0, d.x);
            inst_eval(d, l, t, 0, 0.0, cell_buf(d, 0));
        }
    __syncthreads();
    if (!c.valid) return;
    const double* cells = cell_buf(d, 0);
    for (uint32_t p = c.warp; p < d.nnz; p += nw) {
        ACM(g_out, p) = gather_sum(cells, P, l, d.g_ptr, d.g_cell, p);
        ACM(c_out, p) = gather_sum(cells, P, l, d.c_ptr, d.c_cell, p);
    }
}

// (a + ib) (c + id)
#define CMUL_RE(a, b, c_, d_) ((a) * (c_) - (b) * (d_))
#define CMUL_IM(a, b, c_, d_) ((a) * (d_) + (b) * (c_))

__global__ void __launch_bounds__(kTileThreads) k_ac(TileMap m, AcArgs A) {
    TileCtx c = tile_ctx(m);
    if (!c.valid || c.warp != 0) return;
    const GroupDev& d = *c.d;
    const uint32_t P = d.P, l = c.l, n = A.n;
    const double growth = 1e-12;
    for (uint32_t f = 0; f < A.n_freq; f++) {
        const double om = A.omega[f];
        // Y = G + jwC in the tape's scatter order
        for (uint32_t p = 0; p < d.nnz; p++) {
            ACM(A.ar, p) = ACM(A.g, p);
            ACM(A.ai, p) = om * ACM(A.c, p);
        }
        bool bad = false;
        for (uint32_t k = 0; k < n; k++) {
            const uint32_t col = A.q[k];
            for (uint32_t p = d.col_ptr[col]; p < d.col_ptr[col + 1]; p++) {
                ACM(A.wr, A.prow[p]) = ACM(A.ar, p);
                ACM(A.wi, A.prow[p]) = ACM(A.ai, p);
            }
            for (uint32_t p = A.up[k]; p < A.up[k + 1]; p++) {
                const uint32_t i = A.ui[p];
                const double ur = ACM(A.wr, i), ui = ACM(A.wi, i);
                ACM(A.wr, i) = 0.0;
                ACM(A.wi, i) = 0.0;
                ACM(A.ur, p) = ur;
                ACM(A.ui_, p) = ui;
                for (uint32_t pl = A.lp[i]; pl < A.lp[i + 1]; pl++) {
                    const uint32_t r = A.li[pl];
                    const double lr = ACM(A.lr, pl), li = ACM(A.li_, pl);
                    ACM(A.wr, r) -= CMUL_RE(lr, li, ur, ui);
                    ACM(A.wi, r) -= CMUL_IM(lr, li, ur, ui);
                }
            }
            const double pr = ACM(A.wr, k), pi = ACM(A.wi, k);
            ACM(A.wr, k) = 0.0;
            ACM(A.wi, k) = 0.0;
            const double pn = fmax(fabs(pr), fabs(pi));
            double cmax = pn;
            for (uint32_t p = A.lp[k]; p < A.lp[k + 1]; p++) {
                const uint32_t r = A.li[p];
                cmax = fmax(cmax, fmax(fabs(ACM(A.wr, r)), fabs(ACM(A.wi, r))));
            }
            bad |= !(pn > 0.0) || !(pn < INFINITY) || !(pn >= growth * cmax);
            const double den = pr * pr + pi * pi;
            const double rr = bad ? 1.0 : pr / den, ri = bad ? 0.0 : -pi / den;  // 1 / pivot
            ACM(A.dr, k) = rr;
            ACM(A.di, k) = ri;
            for (uint32_t p = A.lp[k]; p < A.lp[k + 1]; p++) {
                const uint32_t r = A.li[p];
                const double vr = ACM(A.wr, r), vi = ACM(A.wi, r);
                ACM(A.wr, r) = 0.0;
                ACM(A.wi, r) = 0.0;
                ACM(A.lr, p) = CMUL_RE(vr, vi, rr, ri);
                ACM(A.li_, p) = CMUL_IM(vr, vi, rr, ri);
            }
        }
        // y[pinv[exc]] = 1, then the two sweeps (y in the work vector)
        double* yr = A.wr;
        double* yi = A.wi;
        for (uint32_t r = 0; r < n; r++) {
            ACM(yr, r) = 0.0;
            ACM(yi, r) = 0.0;
        }
        ACM(yr, A.pinv[A.exc_row]) = 1.0;
        for (uint32_t k = 0; k < n; k++) {
            const double ykr = ACM(yr, k), yki = ACM(yi, k);
            for (uint32_t p = A.lp[k]; p < A.lp[k + 1]; p++) {
                const uint32_t r = A.li[p];
                ACM(yr, r) -= CMUL_RE(ACM(A.lr, p), ACM(A.li_, p), ykr, yki);
                ACM(yi, r) -= CMUL_IM(ACM(A.lr, p), ACM(A.li_, p), ykr, yki);
            }
        }
        for (uint32_t k = n; k-- > 0;) {
            const double br = ACM(yr, k), bi = ACM(yi, k);
            const double zr = CMUL_RE(br, bi, ACM(A.dr, k), ACM(A.di, k)), zi = CMUL_IM(br, bi, ACM(A.dr, k), ACM(A.di, k));
            ACM(yr, k) = zr;
            ACM(yi, k) = zi;
            for (uint32_t p = A.up[k]; p < A.up[k + 1]; p++) {
                const uint32_t r = A.ui[p];
                ACM(yr, r) -= CMUL_RE(ACM(A.ur, p), ACM(A.ui_, p), zr, zi);
                ACM(yi, r) -= CMUL_IM(ACM(A.ur, p), ACM(A.ui_, p), zr, zi);
            }
        }
        // x[q[j]] = y[j]: unknown u sits at pivot position qinv[u]
        const size_t o = ((size_t)l * A.n_freq + f) * A.n_rows;
        for (uint32_t k = 0; k < A.n_rows; k++) {
            const uint32_t j = A.qinv[A.rows[k]];
            A.out_re[o + k] = bad ? NAN : ACM(yr, j);
            A.out_im[o + k] = bad ? NAN : ACM(yi, j);
        }
        for (uint32_t r = 0; r < n; r++) {
            ACM(yr, r) = 0.0;
            ACM(yi, r) = 0.0;
        }
    }
}

#undef CMUL_RE
#undef CMUL_IM
#undef ACM

}  // namespace espl
