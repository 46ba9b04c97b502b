// Small-signal AC lanes: every lane linearized at its operating point, and
// at each frequency of a list Y(w) = G + jwC solved for a list of
// right-hand sides, Y x = b or, for the adjoint (noise) solves, Y^T z = b
// (the reference's frequency-domain lanes, src/solver/lane/clu.zig
// ComplexLaneLu over src/analysis/gpu/freq.zig).
// As there, the complex values replay a real pivot tape laid on the pattern
// (chosen on the host from a real proxy of the moduli, |G| + w_c |C| of the
// lead lane at the centre frequency), each pivot is checked against its
// column under the infinity norm max(|re|, |im|), and pivots are kept as
// reciprocals. A lane and frequency whose pivot check fails reports NaN.
// One thread per lane (warp 0 of the tile) runs lane_ac_core.cuh; the
// frequencies and right-hand sides loop inside.
#pragma once

#include "lane_ac_core.cuh"
#include "lane_tile.cuh"

namespace espl {

#define ACM(arr, i) (arr)[(size_t)(i) * P + l]

// The AC replay's tape (tape.h Tape, uploaded by espl_ac) and the lanes'
// complex scratch, lane-interleaved like every lane array.
struct AcArgs {
    const uint32_t *q, *qinv, *pinv, *prow, *lp, *li, *up, *ui;
    uint32_t n, nnz_l, nnz_u, n_freq, n_rows, n_rhs, adjoint;
    const double* omega;      // n_freq angular frequencies
    const uint32_t* rows;     // n_rows unknowns reported
    const double *b_re, *b_im;  // n_rhs right-hand sides of length n, every lane's
    const double *g, *c;      // the lanes' G and C at the operating point (nnz x P)
    double *ar, *ai, *wr, *wi, *lr, *li_, *ur, *ui_, *dr, *di;  // complex scratch
    double *out_re, *out_im;  // [lane][freq][rhs][row], the template's lanes
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

// White noise current densities (A^2/Hz) of every lane's noise sources at
// its x, as the reference's models declare them at 27 C (tk = 300.15 K):
// resistors 4kT/R across their terminals (models/resistor.va, resnoise.c),
// diodes 2q|Id| of the junction current without the gmin shunt
// (models/diode.va:326, dionoise.c), level-1 MOS channel thermal noise
// 4kT (2/3)|gm| between drain and source (models/mos1.va:480-489, NLEV
// below 3; gm as mos1load.c computes it); flicker noise is zero (KF = 0)
// and RD/RS are absent. Source s (resistors, then diodes, then MOS in
// their batch order) of lane l goes to psd[s * P + l].
__global__ void __launch_bounds__(kTileThreads) k_noise(TileMap m, double* __restrict__ psd) {
    TileCtx c = tile_ctx(m);
    const GroupDev& d = *c.d;
    const uint32_t P = d.P, l = c.l, nw = c.nw;
    const uint32_t ninst = n_instances(d);
    double* cells = cell_buf(d, 0);
    if (c.valid)
        for (uint32_t t = c.warp; t < ninst; t += nw) {
            inst_seed(d, l, t, 0, d.x);
            inst_eval(d, l, t, 0, 0.0, cells);
        }
    __syncthreads();
    if (!c.valid) return;
    const double kt4 = 4.0 * 1.38064852e-23 * 300.15, q2 = 2.0 * 1.6021766208e-19;
    const uint32_t n_src = d.n_res + d.n_dio + d.n_mos;
    for (uint32_t s = c.warp; s < n_src; s += nw) {
        double v;
        if (s < d.n_res) {
            v = kt4 * fabs(ACM(cells, d.c_res + kResCells * s));
        } else if (s < d.n_res + d.n_dio) {
            const uint32_t i = s - d.n_res;
            const double vd = ACM(d.x, d.dio_t[2 * i]) - ACM(d.x, d.dio_t[2 * i + 1]);
            const double gmin = ACM(d.dio_d, DiodePrep::count * i + DiodePrep::gmin);
            v = q2 * fabs(ACM(cells, d.c_dio + kDioCells * i + 1) - gmin * vd);
        } else {
            const uint32_t i = s - d.n_res - d.n_dio;
            v = kt4 * (2.0 / 3.0) * fabs(ACM(cells, d.c_mos + kMosCells * i + 4));
        }
        ACM(psd, s) = v;
    }
}

__global__ void __launch_bounds__(kTileThreads) k_ac(TileMap m, AcArgs A) {
    TileCtx c = tile_ctx(m);
    if (!c.valid || c.warp != 0) return;
    const GroupDev& d = *c.d;
    const AcTape T{A.q, A.qinv, A.pinv, A.prow, A.lp, A.li, A.up, A.ui, d.col_ptr, A.n, d.nnz};
    const AcWork W{A.ar, A.ai, A.wr, A.wi, A.lr, A.li_, A.ur, A.ui_, A.dr, A.di, d.P, c.l};
    const bool adj = A.adjoint != 0;
    for (uint32_t f = 0; f < A.n_freq; f++) {
        const bool ok = ac_factor(T, W, A.g, A.c, A.omega[f]);
        for (uint32_t e = 0; e < A.n_rhs; e++) {
            ac_solve(T, W, A.b_re + (size_t)e * A.n, A.b_im + (size_t)e * A.n, adj);
            const size_t o = (((size_t)c.l * A.n_freq + f) * A.n_rhs + e) * A.n_rows;
            for (uint32_t k = 0; k < A.n_rows; k++) {
                double re, im;
                ac_value(T, W, adj, A.rows[k], re, im);
                A.out_re[o + k] = ok ? re : NAN;
                A.out_im[o + k] = ok ? im : NAN;
            }
            ac_clear(T, W);
        }
    }
}

#undef ACM

}  // namespace espl
