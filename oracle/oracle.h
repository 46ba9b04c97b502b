/* ORACLE: a CPU FP64 restatement of ESPice's lane-sweep path, used only
 * as test infrastructure (parity checks) and as the timed CPU baseline. It
 * is never linked into, loaded by or called from the product library.
 *
 * Parity status: the symbolic part (ordering, pivot sequence) is pinned by
 * the reference's own known-answer structures (src/solver/tests.zig) and
 * its property tests re-run here. The device-model math and the `$limit`
 * limiters come from VerA, which is not vendored: that boundary is
 * restated from the models' Verilog-A and ngspice's published limiters and
 * is pinned by finite differences and converged-answer parity only.
 */
#ifndef ESPICE_ORACLE_H
#define ESPICE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/espice_lanes.h"

#ifdef __cplusplus
extern "C" {
#endif

/* direct.zig:33, :36, :54; direct.zig:667 */
#define ORC_PIVOT_TOL 1e-3
#define ORC_REPIVOT_FILL_CAP 3.0
#define ORC_GROWTH_LIMIT 1e-12
#define ORC_REPLAY_RATIO_MAX 30.0

/* ---- ordering (order.c) ---- */
size_t orc_ws_size(size_t n, size_t nnz);
int orc_order(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q);
int orc_order_ws(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q, uint32_t *slab, size_t slab_len);
int orc_amd_ws(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q, uint32_t *slab, size_t slab_len);
uint64_t orc_chol_count(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, const uint32_t *perm, uint64_t cap);
uint64_t orc_diag_fill(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, const uint32_t *q);

/* ---- sparse LU (lu.c) ---- */
typedef struct orc_lu orc_lu;
typedef struct {
    uint32_t n, nnz, nnz_l, nnz_u;
    const uint32_t *q, *pinv, *lp, *li, *up, *ui, *prow;
    const uint8_t *void_col, *scaled_pivot;
    const uint32_t *void_slots;
    uint32_t n_void_slots;
    const double *lx, *ux, *udiag;
    uint32_t sn_dfs, n_panels;
} orc_tape;

orc_lu *orc_lu_new(uint32_t n, const uint32_t *col_ptr, const uint32_t *q);
void orc_lu_free(orc_lu *s);
void orc_lu_set_caps(orc_lu *s, uint64_t diag_fill, double fill_cap, double keep_min);
int orc_lu_factor(orc_lu *s, const uint32_t *col_ptr, const uint32_t *row_idx, const double *vals, double pivot_tol);
int orc_lu_refactor(orc_lu *s, const uint32_t *col_ptr, const double *vals, double growth_limit);
void orc_lu_solve(orc_lu *s, const double *b, double *x);
void orc_lu_solve_t(orc_lu *s, const double *b, double *x);
void orc_lu_tape(const orc_lu *s, orc_tape *t);

typedef struct orc_direct orc_direct;
orc_direct *orc_direct_new(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, const uint32_t *q_or_null);
void orc_direct_free(orc_direct *d);
orc_lu *orc_direct_lu(orc_direct *d);
const uint32_t *orc_direct_q(const orc_direct *d);
int orc_direct_factor(orc_direct *d, const double *vals, int *path);
void orc_direct_solve_neg(orc_direct *d, const double *b, double *x);

/* ---- circuit, Newton, transient (circuit.c) ---- */
typedef struct {
    uint32_t converged, singular, iterations, reserved;
} orc_newton_result;

/* Operating point of lanes [lane0, lane0 + count) of `net`, each from its
 * own cold start (init_fix = 1) or from x_in (warm). x_out is point-major
 * [count][n]. Runs on `threads` host threads, one lane per task. */
/* op.solve's ladder per lane (op.zig solveLadder / afterPlain rungs 1-3 and
 * the final solve): res[i].converged and .iterations (all rungs). */
int orc_op_ladder(const espl_netlist *net, uint32_t lane0, uint32_t count, const espl_newton_opts *opts,
                  double *x_out, orc_newton_result *res, uint32_t threads);
/* G and C of lane `lane` linearized at x (limiter state seeded there). */
int orc_planes(const espl_netlist *net, uint32_t lane, const double *x, double *g, double *c);
int orc_op_lanes(const espl_netlist *net, uint32_t lane0, uint32_t count, const espl_newton_opts *opts,
                 const double *x_in, double *x_out, orc_newton_result *res, uint32_t threads);

/* Transient of lanes [lane0, lane0 + count): operating point at t = 0 (the
 * sources at their t = 0 value), then steps to t_stop. probe rows of every
 * accepted step go to probe_out[lane][step][n_probes] when probe_out is not
 * NULL (max_rows steps kept). Reports as espl_step_report. A period measure
 * on `meas_row` (UINT32_MAX: none) is written to period[lane]. */
int orc_tran_lanes(const espl_netlist *net, uint32_t lane0, uint32_t count, const espl_tran_opts *opts,
                   const uint32_t *probes, uint32_t n_probes, uint32_t max_rows, double *probe_out,
                   double *x_final, espl_step_report *reports, uint32_t meas_row, double meas_level,
                   double meas_t_start, double *period, uint32_t threads);

/* The polish of every later Newton solve (the product's
 * espl_create_opts.polish): 0 the reference's test alone; k: after it passes,
 * iterate until the step passes it with the tolerances scaled by 10^-k (at
 * most 4 more iterations). Process-wide; set it before a run. */
void orc_set_polish(uint32_t digits);

/* Newton's residual gate of one row: |F_i| passes when <= this. */
double orc_residual_gate(double residual_tol, double reltol, double vntol, double diag, double xi);

/* Streaming .meas passes (measure.c, after src/output/scan.zig): one pass's
 * state, fed a sample at a time. */
typedef struct {
    int done, first, above, pending, found, inside, cut, np;
    int32_t rise, fall, cross, want_rise, want_fall, want_cross;
    double prev, prev2, prev_x, last, hit;
    uint64_t rows, count;
    double px, pv, py, value, xv, m, m_at, span;
    double p[4][2], first_x, cut_x, sum[3];
    /* FIND/DERIV WHEN and TARG: stage (0 waiting, 1 armed, 2 no event),
     * the event time they start at, rows kept (x, v, level) and read */
    int stage, ring_len;
    double t0, ring[3][3];
    uint64_t kept_rows;
} orc_meas_state;
void orc_meas_init(const espl_meas *c, orc_meas_state *s);
/* Feeds (x, v) to pass c; v2 is its level vector's value (WHEN/TARG with
 * level_row), prev_c/prev the pass before it (NULL for the first). */
void orc_meas_feed(const espl_meas *c, orc_meas_state *s, const espl_meas *prev_c, const orc_meas_state *prev,
                   double x, double v, double v2);
void orc_meas_result(const espl_meas *c, orc_meas_state *s, double *value, double *at);
/* One pass over a whole series (x[k], v[k]); the pass's row is ignored. */
int orc_meas_series(const espl_meas *c, const double *x, const double *v, uint32_t n, double *value, double *at);
/* n_passes passes over a series of n samples, column u of sample k at
 * cols[k * n_cols + u] (a pass reads column `row`, its level column
 * level_row - 1); value and at are [n_passes]. */
int orc_meas_table(const espl_meas *passes, uint32_t n_passes, const double *x, const double *cols, uint32_t n_cols,
                   uint32_t n, double *value, double *at);
/* orc_tran_lanes with .meas passes instead of probes and the period: each
 * pass reads its row at t = 0 and at every accepted step; value and at are
 * [count][n_passes]. */
int orc_tran_meas(const espl_netlist *net, uint32_t lane0, uint32_t count, const espl_tran_opts *opts,
                  const espl_meas *passes, uint32_t n_passes, double *value, double *at, double *x_final,
                  espl_step_report *reports, uint32_t threads);

/* Device-model probes for the finite-difference tests: evaluates instance
 * `inst` of batch `b` in lane `lane` at node voltages v (terminals order)
 * with no limiting; writes the residual rows f[terms] and the Jacobian
 * jac[terms][terms] (row-major, d f_r / d v_c). */
int orc_device_probe(const espl_netlist *net, uint32_t b, uint32_t inst, uint32_t lane, const double *v,
                     double *f, double *jac, double *q, double *cjac);

/* ngspice-style limiters as restated for the `$limit` boundary. */
double orc_pnjlim(double vnew, double vold, double vt, double vcrit, int *icheck);
double orc_fetlim(double vnew, double vold, double vto);
double orc_limvds(double vnew, double vold);

/* stepBound (src/solver/kernels/lane.zig:257-297) over one site. */
double orc_step_bound(uint32_t method, uint32_t cur_method, const double *q0, const double *q1, const double *q2,
                      const double *q3, const double *ip, uint32_t len, const double lte_in[10]);

/* The golden-vector hooks of the reference's own tests. */
double orc_normal_quantile(double u);
uint64_t orc_site_key(uint64_t owner, uint64_t salt);

#ifdef __cplusplus
}
#endif
#endif
