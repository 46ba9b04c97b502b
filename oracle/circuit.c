/* ORACLE (test infrastructure only; never linked into the product).
 *
 * One lane of the reference's CPU FP64 path:
 *   - plane stamping and the ground pin: src/analysis/Circuit.zig:861-928
 *     (groundStamp, clearPlanes, stamp), device eval with the limited image
 *     and its first-order correction: src/device/eval.zig:780-920
 *     (evalRange), the limiter pass with snapLimited: eval.zig:1115-1171;
 *   - Newton: src/solver/converger.zig:200-319 (newtonLanes at W = 1),
 *     loadExtras/loadGmin :286-298, :703-717, finalizeStep :400-470,
 *     updateAndNorm :798-826, plausibleLimit :361-368, residualGate
 *     :300-316; x_plausible = 1e9;
 *   - the operating point's plain rung: src/analysis/dc/op.zig:28-33
 *     (coldStart), :585-592 (gmin 0, init_fix = !warm_start);
 *   - transient: companion rows and A = G + ag0 C
 *     (src/solver/kernels/lane.zig:221-242), coefficients :473-482,
 *     stepBound :257-297, the step machine stepBegin/stepEndA/stepEndB
 *     :505-700, accepted-step history advance (src/solver/lane_device.zig
 *     accept, :428-462), the linear predictor (lane_device.zig predict,
 *     :388-398), and the first-step rule of src/analysis/tran/tran.zig:688-699.
 * A pool of host threads runs one lane per task for the CPU baseline.
 */
#include "devices.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define X_PLAUSIBLE 1e9

typedef struct {
    uint32_t kind, count, nt, np;
    const uint32_t *term;
    uint32_t *slot; /* [count][nt][nt], nnz = trash */
    double *raw;    /* [count][np] this lane's parameters */
    dev_diode *dio;
    dev_mos1 *mos;
    double *lim;    /* MOS1: 3 per instance (vgs, vds, vbs); diode: 1 (vd) */
    uint32_t site0; /* first LTE site */
} obat;

typedef struct {
    uint32_t n, nnz, nb, n_sites;
    const uint32_t *col_ptr, *row_idx;
    uint32_t *diag;
    uint8_t *cur_row;
    obat *b;
    double *g, *c, *rhs, *q, *a, *qs;
    int has_charge;
    orc_direct *slv;
    double *x_old, *dx;
    double src;           /* independent sources' scale (source stepping) */
    uint32_t *gst;        /* gmin stamps (slot, row, col) of the ladder's gmin steps */
    uint32_t n_gst;
    double gst_gmin;      /* the gmin they load (0: none) */
} ockt;

static uint32_t terms_of(uint32_t kind) {
    switch (kind) {
    case ESPL_RES: return ESPL_RES_TERMS;
    case ESPL_CAP: return ESPL_CAP_TERMS;
    case ESPL_VSRC: return ESPL_VSRC_TERMS;
    case ESPL_ISRC: return ESPL_ISRC_TERMS;
    case ESPL_DIODE: return ESPL_DIODE_TERMS;
    case ESPL_MOS1: return ESPL_MOS1_TERMS;
    }
    return 0;
}

static uint32_t params_of(uint32_t kind) {
    switch (kind) {
    case ESPL_RES: return ESPL_RES_PARAMS;
    case ESPL_CAP: return ESPL_CAP_PARAMS;
    case ESPL_VSRC: case ESPL_ISRC: return ESPL_SRC_PARAMS;
    case ESPL_DIODE: return ESPL_DIODE_PARAMS;
    case ESPL_MOS1: return ESPL_MOS1_PARAMS;
    }
    return 0;
}

static uint32_t find_slot(const ockt *k, uint32_t r, uint32_t c) {
    if (r == ESPL_GROUND || c == ESPL_GROUND) return k->nnz;
    for (uint32_t p = k->col_ptr[c]; p < k->col_ptr[c + 1]; p++)
        if (k->row_idx[p] == r) return p;
    return UINT32_MAX;
}

/* Whether a device of `kind` stamps Jacobian entry (terminal r, terminal c). */
static int stamps(uint32_t kind, uint32_t r, uint32_t c) {
    switch (kind) {
    case ESPL_RES: case ESPL_CAP: case ESPL_DIODE: return 1;
    case ESPL_VSRC: return (r < 2 && c == 2) || (r == 2 && c < 2);
    case ESPL_MOS1: return r != 1;
    }
    return 0;
}

static void ckt_free(ockt *k) {
    if (k) free(k->gst);
    if (!k) return;
    for (uint32_t i = 0; i < k->nb; i++) {
        free(k->b[i].slot);
        free(k->b[i].raw);
        free(k->b[i].dio);
        free(k->b[i].mos);
        free(k->b[i].lim);
    }
    free(k->b);
    free(k->diag);
    free(k->cur_row);
    free(k->g); free(k->c); free(k->rhs); free(k->q); free(k->a); free(k->qs);
    free(k->x_old); free(k->dx);
    orc_direct_free(k->slv);
    free(k);
}

static ockt *ckt_new(const espl_netlist *net, uint32_t lane, const uint32_t *q_order) {
    ockt *k = (ockt *)calloc(1, sizeof(ockt));
    k->n = net->n;
    k->nnz = net->nnz;
    k->col_ptr = net->col_ptr;
    k->row_idx = net->row_idx;
    k->nb = net->n_batches;
    k->diag = (uint32_t *)malloc(sizeof(uint32_t) * k->n);
    k->cur_row = (uint8_t *)calloc(k->n, 1);
    for (uint32_t i = 0; i < k->n; i++) {
        k->diag[i] = find_slot(k, i, i);
        if (k->diag[i] == UINT32_MAX) { ckt_free(k); return NULL; }
    }
    k->b = (obat *)calloc(k->nb ? k->nb : 1, sizeof(obat));
    uint32_t sites = 0;
    for (uint32_t bi = 0; bi < k->nb; bi++) {
        const espl_batch *sb = &net->batches[bi];
        obat *b = &k->b[bi];
        b->kind = sb->kind;
        b->count = sb->count;
        b->nt = terms_of(sb->kind);
        b->np = params_of(sb->kind);
        b->term = sb->term;
        b->slot = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)b->count * b->nt * b->nt + 1);
        b->raw = (double *)malloc(sizeof(double) * (size_t)b->count * b->np + 1);
        for (uint32_t i = 0; i < b->count; i++) {
            for (uint32_t r = 0; r < b->nt; r++)
                for (uint32_t c = 0; c < b->nt; c++) {
                    uint32_t tr = b->term[i * b->nt + r], tc = b->term[i * b->nt + c];
                    uint32_t s = find_slot(k, tr, tc);
                    if (s == UINT32_MAX && stamps(b->kind, r, c)) { k->nb = bi + 1; ckt_free(k); return NULL; }
                    b->slot[((size_t)i * b->nt + r) * b->nt + c] = s;
                }
            for (uint32_t p = 0; p < b->np; p++)
                b->raw[(size_t)i * b->np + p] = sb->param[((size_t)i * b->np + p) * net->lanes + lane];
        }
        if (b->kind == ESPL_VSRC)
            for (uint32_t i = 0; i < b->count; i++) k->cur_row[b->term[i * 3 + 2]] = 1;
        if (b->kind == ESPL_DIODE) {
            b->dio = (dev_diode *)malloc(sizeof(dev_diode) * (b->count ? b->count : 1));
            b->lim = (double *)calloc(b->count ? b->count : 1, sizeof(double));
            for (uint32_t i = 0; i < b->count; i++) dev_setup_diode(b->raw + (size_t)i * b->np, &b->dio[i]);
            b->site0 = sites;
            for (uint32_t i = 0; i < b->count; i++)
                if (b->dio[i].cjo > 0 || b->dio[i].tt > 0) k->has_charge = 1;
            sites += b->count;
        } else if (b->kind == ESPL_MOS1) {
            b->mos = (dev_mos1 *)malloc(sizeof(dev_mos1) * (b->count ? b->count : 1));
            b->lim = (double *)calloc(3 * (size_t)(b->count ? b->count : 1), sizeof(double));
            for (uint32_t i = 0; i < b->count; i++) dev_setup_mos1(b->raw + (size_t)i * b->np, &b->mos[i]);
        } else if (b->kind == ESPL_CAP) {
            b->site0 = sites;
            sites += b->count;
            if (b->count) k->has_charge = 1;
        }
    }
    k->n_sites = sites;
    size_t nnz1 = (size_t)k->nnz + 1, n1 = (size_t)k->n + 1;
    k->g = (double *)calloc(nnz1, sizeof(double));
    k->c = (double *)calloc(nnz1, sizeof(double));
    k->a = (double *)calloc(nnz1, sizeof(double));
    k->rhs = (double *)calloc(n1, sizeof(double));
    k->q = (double *)calloc(n1, sizeof(double));
    k->qs = (double *)calloc(sites ? sites : 1, sizeof(double));
    k->x_old = (double *)calloc(n1, sizeof(double));
    k->dx = (double *)calloc(n1, sizeof(double));
    k->slv = orc_direct_new(k->n, k->col_ptr, k->row_idx, q_order);
    if (!k->slv) { ckt_free(k); return NULL; }
    k->src = 1.0;
    return k;
}

static double xat(const double *x, uint32_t u) { return u == ESPL_GROUND ? 0.0 : x[u]; }

/* MOS1 normalized branch voltages of instance i at x. */
static void mos_branch(const obat *b, uint32_t i, const double *x, double v[3]) {
    const uint32_t *t = b->term + (size_t)i * 4;
    double ty = b->mos[i].type;
    double vd = xat(x, t[0]), vg = xat(x, t[1]), vs = xat(x, t[2]), vb = xat(x, t[3]);
    v[0] = ty * (vg - vs);
    v[1] = ty * (vd - vs);
    v[2] = ty * (vb - vs);
}

static double inst_scale(const obat *b, uint32_t i, const double *x) {
    double s = 0;
    for (uint32_t t = 0; t < b->nt; t++) {
        double a = fabs(xat(x, b->term[(size_t)i * b->nt + t]));
        if (a > s) s = a;
    }
    return s;
}

/* Cold start (op.zig coldStart): limiter states at the MODEINITJCT seeds,
 * MOS1 vgs = type*vbit + gamma*sqrt(phit), vds = 0, vbs = -1; the diode,
 * which has no seed, starts from x. Warm: every state is x's image. */
static void seed_limits(ockt *k, const double *x, int cold) {
    for (uint32_t bi = 0; bi < k->nb; bi++) {
        obat *b = &k->b[bi];
        if (b->kind == ESPL_MOS1) {
            for (uint32_t i = 0; i < b->count; i++) {
                double *s = b->lim + 3 * (size_t)i;
                if (cold) {
                    s[0] = b->mos[i].vgs_seed;
                    s[1] = 0.0;
                    s[2] = -1.0;
                } else {
                    mos_branch(b, i, x, s);
                }
            }
        } else if (b->kind == ESPL_DIODE) {
            for (uint32_t i = 0; i < b->count; i++) b->lim[i] = xat(x, b->term[2 * i]) - xat(x, b->term[2 * i + 1]);
        }
    }
}

/* The limiter pass (limitRange + snapLimited): returns 1 when any device
 * clamped its branch voltages. */
static int apply_limits(ockt *k, const double *x) {
    int flag = 0;
    for (uint32_t bi = 0; bi < k->nb; bi++) {
        obat *b = &k->b[bi];
        if (b->kind == ESPL_MOS1) {
            for (uint32_t i = 0; i < b->count; i++) {
                double cur[3], out[3];
                double *s = b->lim + 3 * (size_t)i;
                mos_branch(b, i, x, cur);
                dev_mos1_limit(&b->mos[i], s, cur, out);
                double tol = 16 * DBL_EPSILON * inst_scale(b, i, x);
                for (int j = 0; j < 3; j++) {
                    if (fabs(out[j] - cur[j]) <= tol) out[j] = cur[j];
                    if (out[j] != cur[j]) flag = 1;
                    s[j] = out[j];
                }
            }
        } else if (b->kind == ESPL_DIODE) {
            for (uint32_t i = 0; i < b->count; i++) {
                double vd = xat(x, b->term[2 * i]) - xat(x, b->term[2 * i + 1]);
                int chk;
                double l = orc_pnjlim(vd, b->lim[i], b->dio[i].vte, b->dio[i].vcrit, &chk);
                if (fabs(l - vd) <= 16 * DBL_EPSILON * inst_scale(b, i, x)) l = vd;
                if (l != vd) flag = 1;
                b->lim[i] = l;
            }
        }
    }
    return flag;
}

static void add_rhs(ockt *k, uint32_t u, double v) { k->rhs[u == ESPL_GROUND ? k->n : u] += v; }
static void add_q(ockt *k, uint32_t u, double v) { k->q[u == ESPL_GROUND ? k->n : u] += v; }

/* Stamps G, C, rhs (the residual F) and q at x, devices at their limited
 * images with the first-order correction, then the ground pin. `tran`
 * selects the transient source semantics at time t. */
static void eval_planes(ockt *k, const double *x, int tran, double t) {
    memset(k->g, 0, sizeof(double) * (k->nnz + 1));
    memset(k->c, 0, sizeof(double) * (k->nnz + 1));
    memset(k->rhs, 0, sizeof(double) * (k->n + 1));
    memset(k->q, 0, sizeof(double) * (k->n + 1));
    for (uint32_t bi = 0; bi < k->nb; bi++) {
        obat *b = &k->b[bi];
        for (uint32_t i = 0; i < b->count; i++) {
            const uint32_t *tm = b->term + (size_t)i * b->nt;
            const uint32_t *sl = b->slot + (size_t)i * b->nt * b->nt;
            const double *p = b->raw + (size_t)i * b->np;
            switch (b->kind) {
            case ESPL_RES: {
                double v = xat(x, tm[0]) - xat(x, tm[1]);
                double r = p[0];
                double cur = v / r, gg = 1.0 / r;
                add_rhs(k, tm[0], cur);
                k->g[sl[0]] += gg;
                k->g[sl[1]] += -gg;
                add_rhs(k, tm[1], -cur);
                k->g[sl[2]] += -gg;
                k->g[sl[3]] += gg;
                break;
            }
            case ESPL_CAP: {
                double v = xat(x, tm[0]) - xat(x, tm[1]);
                double cc = p[0];
                double qq = cc * v;
                add_q(k, tm[0], qq);
                k->c[sl[0]] += cc;
                k->c[sl[1]] += -cc;
                add_q(k, tm[1], -qq);
                k->c[sl[2]] += -cc;
                k->c[sl[3]] += cc;
                k->qs[b->site0 + i] = qq;
                break;
            }
            case ESPL_VSRC: {
                double ib = xat(x, tm[2]);
                double val = dev_source_value(p, tran, t);
                add_rhs(k, tm[0], ib);
                k->g[sl[0 * 3 + 2]] += 1.0;
                add_rhs(k, tm[1], -ib);
                k->g[sl[1 * 3 + 2]] += -1.0;
                add_rhs(k, tm[2], (xat(x, tm[0]) - xat(x, tm[1])) - val * k->src);
                k->g[sl[2 * 3 + 0]] += 1.0;
                k->g[sl[2 * 3 + 1]] += -1.0;
                break;
            }
            case ESPL_ISRC: {
                double val = dev_source_value(p, tran, t) * k->src;
                add_rhs(k, tm[0], val);
                add_rhs(k, tm[1], -val);
                break;
            }
            case ESPL_DIODE: {
                double vd = xat(x, tm[0]) - xat(x, tm[1]);
                double vl = b->lim[i];
                double id, gd, qd, cd;
                dev_diode_core(&b->dio[i], vl, &id, &gd, &qd, &cd);
                double f = id + gd * (vd - vl);
                add_rhs(k, tm[0], f);
                k->g[sl[0]] += gd;
                k->g[sl[1]] += -gd;
                add_rhs(k, tm[1], -f);
                k->g[sl[2]] += -gd;
                k->g[sl[3]] += gd;
                if (b->dio[i].cjo > 0 || b->dio[i].tt > 0) {
                    double qq = qd + cd * (vd - vl);
                    add_q(k, tm[0], qq);
                    k->c[sl[0]] += cd;
                    k->c[sl[1]] += -cd;
                    add_q(k, tm[1], -qq);
                    k->c[sl[2]] += -cd;
                    k->c[sl[3]] += cd;
                    k->qs[b->site0 + i] = qq;
                }
                break;
            }
            case ESPL_MOS1: {
                const dev_mos1 *m = &b->mos[i];
                const double *s = b->lim + 3 * (size_t)i;
                double va[3];
                mos_branch(b, i, x, va);
                dev_mos1_out o;
                dev_mos1_core(m, s[0], s[1], s[2], &o);
                double ty = m->type;
                double dgs = va[0] - s[0], dds = va[1] - s[1], dbs = va[2] - s[2];
                /* Channel, normalized drain-to-source current mode*id. */
                double gm = o.mode * o.gm, gds = o.mode * o.gds, gmbs = o.mode * o.gmbs;
                double ich = o.mode * o.id + gm * dgs + gds * dds + gmbs * dbs;
                /* Bulk junctions at vbd = vbs - vds and vbs. */
                double ibd = o.ibd + o.gbd * (dbs - dds);
                double ibs = o.ibs + o.gbs * dbs;
                /* Node currents (out of node): d: I_ds - I_bd, s: -I_ds - I_bs,
                 * b: I_bd + I_bs; node-frame currents carry `type`. */
                double fd = ty * ich - ty * ibd;
                double fs = -ty * ich - ty * ibs;
                double fb = ty * ibd + ty * ibs;
                /* d(node current)/d(node voltage): the two `type` factors cancel. */
                double jd[4], jg[4], js[4], jb[4]; /* rows d g s b over cols d g s b */
                double gsum = gm + gds + gmbs;
                /* Channel row (d): wrt vd = gds, vg = gm, vs = -gsum, vb = gmbs. */
                jd[0] = gds + o.gbd; jd[1] = gm; jd[2] = -gsum; jd[3] = gmbs - o.gbd;
                jg[0] = 0; jg[1] = 0; jg[2] = 0; jg[3] = 0;
                js[0] = -gds; js[1] = -gm; js[2] = gsum + o.gbs; js[3] = -gmbs - o.gbs;
                jb[0] = -o.gbd; jb[1] = 0; jb[2] = -o.gbs; jb[3] = o.gbd + o.gbs;
                double f[4] = {fd, 0.0, fs, fb};
                const double *rows[4] = {jd, jg, js, jb};
                for (int r = 0; r < 4; r++) {
                    if (r == 1) continue; /* the gate draws no current */
                    add_rhs(k, tm[r], f[r]);
                    for (int c = 0; c < 4; c++) k->g[sl[r * 4 + c]] += rows[r][c];
                }
                break;
            }
            }
        }
    }
    /* groundStamp (Circuit.zig:861-864). */
    k->g[k->diag[0]] += 1.0;
    k->rhs[0] += x[0];
}

static double bits2d(uint64_t b) { double d; memcpy(&d, &b, 8); return d; }
static uint64_t d2bits(double d) { uint64_t b; memcpy(&b, &d, 8); return b; }

static double norm_inf(const double *x, uint32_t n) {
    uint64_t m = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint64_t b = d2bits(fabs(x[i]));
        if (b > m) m = b;
    }
    return bits2d(m);
}

/* converger.zig plausibleLimit: a NaN anywhere keeps the floor. */
static double plausible_limit(const ockt *k, const double *x, const double *f, const double *vals) {
    double g = 1;
    for (uint32_t i = 0; i < k->n; i++) {
        double a = fabs(vals[k->diag[i]]);
        if (a > g) g = a;
    }
    double xm = norm_inf(x, k->n), fm = norm_inf(f, k->n) * g;
    double scale = xm > fm ? xm : fm;
    if (xm != xm || fm != fm) scale = NAN;
    if (scale > 1e18) scale = 1e18;
    return !(1e3 * scale > X_PLAUSIBLE) ? X_PLAUSIBLE : 1e3 * scale;
}

/* converger.zig updateAndNorm at W = 1 */
static double update_and_norm(const ockt *k, double *x, const double *dx, double *x_old, double reltol, double abstol, double vntol) {
    uint64_t worst = 0;
    for (uint32_t i = 0; i < k->n; i++) {
        double xo = x[i], d = dx[i];
        double xn = xo + d;
        x_old[i] = xo;
        x[i] = xn;
        double ax = fabs(xn), ao = fabs(xo);
        double tol = reltol * (ax > ao ? ax : ao) + (k->cur_row[i] ? abstol : vntol);
        int finite = fabs(xn) < INFINITY && fabs(d) < INFINITY;
        double q = fabs(d) / tol;
        double score = !finite ? INFINITY : (q == q ? q : 0);
        uint64_t b = d2bits(score);
        if (b > worst) worst = b;
    }
    return bits2d(worst);
}

/* converger.zig residualGate :340-350 (@max returns the other operand of a
 * NaN, as fmax does). */
double orc_residual_gate(double residual_tol, double reltol, double vntol, double diag, double xi) {
    double scale = fabs(diag);
    double s = scale == 0 ? 1.0 : scale;
    return fmax(residual_tol, 10.0 * s * (reltol * fabs(xi) + vntol));
}

static int residual_ok(const ockt *k, const espl_newton_opts *o, const double *res, const double *x, const double *vals) {
    for (uint32_t i = 0; i < k->n; i++) {
        double tol = orc_residual_gate(o->residual_tol, o->reltol, o->vntol, vals[k->diag[i]], x[i]);
        if (!(fabs(res[i]) <= tol)) return 0;
    }
    return 1;
}

/* Companion state of a transient attempt. */
typedef struct {
    int on;
    uint32_t method; /* 0 BE, 1 trap, 2 gear-2 */
    double ag0, ag1, ag2;
    const double *q1;     /* row charges at the last accepted step */
    const double *q2;     /* and at the one before (gear-2) */
    const double *i_prev; /* row companion currents there */
} companion;

/* The polish (espl_create_opts.polish of the product): 0 off, else the
 * tightened test's tolerances are scaled by 10^-digits. Set before a run;
 * read by every Newton solve. */
static double g_polish = 0.0;
#define ORC_POLISH_MAX 4u
void orc_set_polish(uint32_t digits) { g_polish = digits ? pow(10.0, -(double)digits) : 0.0; }

/* newtonLanes at W = 1 (converger.zig:200-319). With the polish on, a lane
 * whose step passes the reference's test keeps iterating from x + dx until
 * the step also passes the test with the tolerances scaled by g_polish (at
 * most ORC_POLISH_MAX more iterations), and publishes that iterate. */
static orc_newton_result newton(ockt *k, double *x, const espl_newton_opts *o, int tran, double t, const companion *cp, uint32_t *fail_factor) {
    orc_newton_result r = {0, 0, 0, 0};
    int init_fix = o->init_fix != 0;
    uint32_t polished = 0;
    double limit = X_PLAUSIBLE;
    for (uint32_t iter = 0; iter < o->max_iter; iter++) {
        eval_planes(k, x, tran, t);
        const double *v;
        if (cp && cp->on) {
            for (uint32_t i = 0; i < k->n; i++) {
                double d = cp->ag0 * (k->q[i] - cp->q1[i]);
                double base = k->rhs[i] + d;
                k->rhs[i] = cp->method == 1   ? base - cp->ag1 * cp->i_prev[i]
                            : cp->method == 2 ? base - cp->ag2 * (cp->q1[i] - cp->q2[i])
                                              : base;
            }
            for (uint32_t p = 0; p < k->nnz; p++) k->a[p] = k->g[p] + cp->ag0 * k->c[p];
            v = k->a;
        } else {
            memcpy(k->a, k->g, sizeof(double) * k->nnz);
            v = k->a;
        }
        if (o->gmin > 0) {
            for (uint32_t i = 0; i < k->n; i++) k->a[k->diag[i]] += o->gmin;
            for (uint32_t i = 0; i < k->n; i++) k->rhs[i] += o->gmin * x[i];
        }
        if (k->n_gst && k->gst_gmin > 0) { /* converger.zig loadGmin at the stamps */
            for (uint32_t s = 0; s < k->n_gst; s++) {
                k->a[k->gst[3 * s]] += k->gst_gmin;
                k->rhs[k->gst[3 * s + 1]] += k->gst_gmin * x[k->gst[3 * s + 2]];
            }
        }
        if (iter == 0) limit = plausible_limit(k, x, k->rhs, v);
        int path = -1;
        int frc = orc_direct_factor(k->slv, v, &path);
        if (getenv("ORC_DEBUG")) fprintf(stderr, "iter %u factor rc %d path %d\n", iter, frc, path);
        if (frc != 0) {
            r.singular = 1;
            r.iterations = iter;
            if (fail_factor) (*fail_factor)++;
            return r;
        }
        orc_direct_solve_neg(k->slv, k->rhs, k->dx);
        double scaled = update_and_norm(k, x, k->dx, k->x_old, o->reltol, o->abstol, o->vntol);
        int limited = apply_limits(k, x);
        int ok = !limited && iter != 0 && !(scaled >= 1.0);
        if (ok) {
            for (uint32_t i = 0; i < k->n; i++)
                if (!(fabs(x[i]) <= limit)) { ok = 0; break; }
        }
        if (ok) ok = residual_ok(k, o, k->rhs, x, v);
        if (ok && init_fix) {
            init_fix = 0;
        } else if (ok && g_polish > 0.0 && !(scaled < g_polish) && polished < ORC_POLISH_MAX) {
            polished++;
        } else if (ok) {
            memcpy(x, k->x_old, sizeof(double) * k->n);
            r.converged = 1;
            r.iterations = iter + 1;
            return r;
        }
    }
    r.iterations = o->max_iter;
    return r;
}

/* ---------------- lane runners ---------------- */

typedef struct {
    const espl_netlist *net;
    uint32_t lane0, count;
    const espl_newton_opts *opts;
    const double *x_in;
    double *x_out;
    orc_newton_result *res;
    const uint32_t *q;
    atomic_uint next;
    /* transient */
    const espl_tran_opts *topts;
    const uint32_t *probes;
    uint32_t n_probes, max_rows;
    double *probe_out;
    espl_step_report *reports;
    uint32_t meas_row;
    double meas_level, meas_t_start;
    const espl_meas *passes;
    uint32_t n_passes;
    double *meas_value, *meas_at;
    double *period;
} job_t;

static void op_one(job_t *j, uint32_t li) {
    uint32_t lane = j->lane0 + li;
    uint32_t n = j->net->n;
    ockt *k = ckt_new(j->net, lane, j->q);
    double *x = j->x_out + (size_t)li * n;
    if (!k) {
        memset(&j->res[li], 0, sizeof(orc_newton_result));
        j->res[li].singular = 1;
        return;
    }
    if (j->x_in) memcpy(x, j->x_in + (size_t)li * n, sizeof(double) * n);
    else memset(x, 0, sizeof(double) * n);
    seed_limits(k, x, j->opts->init_fix != 0);
    j->res[li] = newton(k, x, j->opts, 0, 0.0, NULL, NULL);
    ckt_free(k);
}

/* ---------------- the operating-point ladder ---------------- */

/* op.zig gminStamps :712-792: ngspice's diagonal-gmin places after Sparse's
 * spMNA_Preorder, read off the last assembly's G values (k->g). */
static void gmin_stamps(ockt *k) {
    uint32_t n = k->n, none = UINT32_MAX;
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * n), *dcol = (uint32_t *)malloc(sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t slot = k->diag[i];
        perm[i] = i;
        dcol[i] = (k->cur_row[i] && k->g[slot] == 0 && k->c[slot] == 0) ? none : i;
    }
    uint32_t start = 1;
    for (;;) {
        int swapped = 0, again = 0;
        for (int pass = 0; pass < 2; pass++) {
            for (uint32_t jj = start; jj < n; jj++) {
                if (pass == 1 && swapped) break;
                if (dcol[jj] != none) continue;
                /* CountTwins: +-1 entries of column position jj whose transposes are +-1 */
                uint32_t cnt = 0, trow = 0, col = perm[jj];
                for (uint32_t p = k->col_ptr[col]; p < k->col_ptr[col + 1]; p++) {
                    uint32_t r = k->row_idx[p];
                    if (fabs(k->g[p]) != 1.0) continue;
                    uint32_t q = find_slot(k, jj, perm[r]);
                    if (q >= k->nnz || fabs(k->g[q]) != 1.0) continue;
                    cnt++;
                    if (cnt == 1) trow = r;
                    else break;
                }
                int take = pass == 0 ? cnt == 1 : cnt > 0;
                if (take) {
                    dcol[jj] = perm[trow];
                    dcol[trow] = perm[jj];
                    uint32_t t = perm[jj]; perm[jj] = perm[trow]; perm[trow] = t;
                    swapped = 1;
                } else if (pass == 0 && cnt > 1 && !again) {
                    again = 1;
                    start = jj;
                }
            }
            if (pass == 0 && !again) break;
        }
        if (!again || !swapped) break;
    }
    free(k->gst);
    k->gst = (uint32_t *)malloc(sizeof(uint32_t) * 3 * (n ? n : 1));
    k->n_gst = 0;
    for (uint32_t i = 1; i < n; i++) {
        if (dcol[i] == none) continue;
        uint32_t slot = find_slot(k, i, dcol[i]);
        if (slot >= k->nnz) continue;
        k->gst[3 * k->n_gst] = slot;
        k->gst[3 * k->n_gst + 1] = i;
        k->gst[3 * k->n_gst + 2] = dcol[i];
        k->n_gst++;
    }
    free(perm);
    free(dcol);
}

static void cold_start(ockt *k, double *x) {
    memset(x, 0, sizeof(double) * k->n);
    seed_limits(k, x, 1);
}

static orc_newton_result run_rung(ockt *k, double *x, const espl_newton_opts *base, double gmin, double src,
                                  int init_fix, uint32_t max_iter, uint32_t *total) {
    espl_newton_opts o = *base;
    o.gmin = 0.0;
    o.init_fix = init_fix ? 1 : 0;
    o.max_iter = max_iter;
    k->gst_gmin = gmin;
    k->src = src;
    if (!init_fix) seed_limits(k, x, 0);
    orc_newton_result r = newton(k, x, &o, 0, 0.0, NULL, NULL);
    k->gst_gmin = 0.0;
    k->src = 1.0;
    uint32_t it = r.singular ? 0 : r.iterations;
    *total = *total + it > 65535u ? 65535u : *total + it;
    return r;
}

/* op.zig afterPlain rungs 2 and 3 and the final solve (:163-312), after the
 * plain rung failed; gminFactor :384-388, gminStalled :363-376,
 * sourcesOffGmin :397-421. */
static int ladder_one(ockt *k, double *x, const espl_newton_opts *o, uint32_t *total) {
    const double gtarget = 1e-12, gmin_start = 1e-2;
    const uint32_t budget = 100, max_solves = 1000, stall = 20;
    const double stall_factor = pow(10.0, 1.0 / stall);
    uint32_t n = k->n;
    double *x_good = (double *)malloc(sizeof(double) * n);
    double *st_g = (double *)malloc(sizeof(double) * max_solves);
    int *st_c = (int *)malloc(sizeof(int) * max_solves);
    int converged = 0;
    gmin_stamps(k);
    cold_start(k, x);
    {
        double factor = 10.0, good = gmin_start, g = good / factor;
        int have_good = 0;
        for (uint32_t solves = 0; solves < max_solves; solves++) {
            double tried = g;
            orc_newton_result r = run_rung(k, x, o, g, 1.0, !have_good, budget, total);
            int refused = r.singular;
            int conv = !refused && r.converged;
            if (conv) {
                if (g <= gtarget) {
                    orc_newton_result c = run_rung(k, x, o, 0.0, 1.0, 0, budget, total);
                    if (c.converged && !c.singular) { converged = 1; goto done; }
                    break;
                }
                memcpy(x_good, x, sizeof(double) * n);
                have_good = 1;
                good = g;
                uint32_t it = r.iterations;
                if (it <= budget / 4) factor = fmin(factor * sqrt(factor), 10.0);
                else if (it > 3 * (budget / 4)) factor = fmax(sqrt(factor), 1.00005);
                if (g < factor * gtarget) { factor = g / gtarget; g = gtarget; }
                else g /= factor;
            } else {
                if (factor < 1.00005) break;
                factor = refused ? sqrt(factor) : sqrt(sqrt(factor));
                g = good / factor;
                if (have_good) memcpy(x, x_good, sizeof(double) * n);
                else cold_start(k, x);
            }
            st_g[solves] = tried;
            st_c[solves] = conv;
            uint32_t m = solves + 1;
            if (m >= stall) {
                double gd = gmin_start;
                int stalled = 1;
                for (uint32_t i = 0; i < m; i++) {
                    if (st_c[i]) gd = st_g[i];
                    if (i < m - stall) continue;
                    double following = i + 1 < m ? st_g[i + 1] : g;
                    if (gd / following >= stall_factor) { stalled = 0; break; }
                }
                if (stalled) break;
            }
        }
    }
    cold_start(k, x);
    {
        double lambda = 0.0, lambda_good = -1.0, delta = 0.25;
        for (uint32_t solves = 0; solves < max_solves; solves++) {
            orc_newton_result r = run_rung(k, x, o, 0.0, lambda, lambda_good < 0.0, budget, total);
            int conv = !r.singular && r.converged;
            if (!conv && lambda_good < 0.0) {
                /* sourcesOffGmin: eleven solves from 1e10 x gmin down a decade each */
                cold_start(k, x);
                double g = gtarget * 1e10;
                conv = 1;
                for (int i = 0; i < 11; i++) {
                    orc_newton_result s = run_rung(k, x, o, g, lambda, i == 0, budget, total);
                    if (!(s.converged && !s.singular)) { conv = 0; break; }
                    g /= 10;
                }
            }
            if (conv) {
                if (lambda >= 1.0) break;
                lambda_good = lambda;
                memcpy(x_good, x, sizeof(double) * n);
                delta *= 1.5;
                lambda = fmin(lambda + delta, 1.0);
            } else {
                delta *= 0.5;
                if (delta < 1e-4) break;
                if (lambda_good < 0.0) break;
                memcpy(x, x_good, sizeof(double) * n);
                lambda = fmin(lambda_good + delta, 1.0);
            }
        }
    }
    {
        orc_newton_result f = run_rung(k, x, o, 0.0, 1.0, 0, budget, total);
        converged = f.converged && !f.singular;
    }
done:
    free(x_good);
    free(st_g);
    free(st_c);
    return converged;
}

static void op_ladder_one(job_t *j, uint32_t li) {
    uint32_t lane = j->lane0 + li;
    uint32_t n = j->net->n;
    ockt *k = ckt_new(j->net, lane, j->q);
    double *x = j->x_out + (size_t)li * n;
    orc_newton_result *res = &j->res[li];
    memset(res, 0, sizeof(*res));
    if (!k) { res->singular = 1; return; }
    cold_start(k, x);
    espl_newton_opts plain = *j->opts;
    plain.gmin = 0.0;
    plain.init_fix = 1;
    orc_newton_result r = newton(k, x, &plain, 0, 0.0, NULL, NULL);
    uint32_t total = r.singular ? 0 : r.iterations;
    int conv = r.converged && !r.singular;
    if (!conv) conv = ladder_one(k, x, j->opts, &total);
    res->converged = conv;
    res->iterations = total;
    ckt_free(k);
}

static void *op_ladder_worker(void *arg) {
    job_t *j = (job_t *)arg;
    for (;;) {
        uint32_t li = atomic_fetch_add(&j->next, 1);
        if (li >= j->count) break;
        op_ladder_one(j, li);
    }
    return NULL;
}

static void *op_worker(void *arg) {
    job_t *j = (job_t *)arg;
    for (;;) {
        uint32_t li = atomic_fetch_add(&j->next, 1);
        if (li >= j->count) break;
        op_one(j, li);
    }
    return NULL;
}

static int run_pool(job_t *j, uint32_t threads, void *(*fn)(void *)) {
    if (threads <= 1) {
        fn(j);
        return 0;
    }
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    for (uint32_t i = 0; i < threads; i++) pthread_create(&th[i], NULL, fn, j);
    for (uint32_t i = 0; i < threads; i++) pthread_join(th[i], NULL);
    free(th);
    return 0;
}

int orc_planes(const espl_netlist *net, uint32_t lane, const double *x, double *g, double *c) {
    uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * (net->n ? net->n : 1));
    if (orc_order(net->n, net->col_ptr, net->row_idx, q) != 0) { free(q); return -1; }
    ockt *k = ckt_new(net, lane, q);
    free(q);
    if (!k) return -1;
    double *xx = (double *)malloc(sizeof(double) * (net->n ? net->n : 1));
    memcpy(xx, x, sizeof(double) * net->n);
    seed_limits(k, xx, 0);
    eval_planes(k, xx, 0, 0.0);
    memcpy(g, k->g, sizeof(double) * k->nnz);
    memcpy(c, k->c, sizeof(double) * k->nnz);
    free(xx);
    ckt_free(k);
    return 0;
}

int orc_op_ladder(const espl_netlist *net, uint32_t lane0, uint32_t count, const espl_newton_opts *opts,
                  double *x_out, orc_newton_result *res, uint32_t threads) {
    uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * (net->n ? net->n : 1));
    if (orc_order(net->n, net->col_ptr, net->row_idx, q) != 0) { free(q); return -1; }
    job_t j;
    memset(&j, 0, sizeof(j));
    j.net = net;
    j.lane0 = lane0;
    j.count = count;
    j.opts = opts;
    j.x_out = x_out;
    j.res = res;
    j.q = q;
    atomic_init(&j.next, 0);
    run_pool(&j, threads, op_ladder_worker);
    free(q);
    return 0;
}

int orc_op_lanes(const espl_netlist *net, uint32_t lane0, uint32_t count, const espl_newton_opts *opts,
                 const double *x_in, double *x_out, orc_newton_result *res, uint32_t threads) {
    uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * (net->n ? net->n : 1));
    if (orc_order(net->n, net->col_ptr, net->row_idx, q) != 0) { free(q); return -1; }
    job_t j;
    memset(&j, 0, sizeof(j));
    j.net = net;
    j.lane0 = lane0;
    j.count = count;
    j.opts = opts;
    j.x_in = x_in;
    j.x_out = x_out;
    j.res = res;
    j.q = q;
    atomic_init(&j.next, 0);
    run_pool(&j, threads, op_worker);
    free(q);
    return 0;
}

/* ---------------- transient ---------------- */

/* kernels/lane.zig coeffs over method codes (BE, trap, gear-2), after
 * integrator.zig coeffs (src/analysis/tran/integrator.zig:39-52): gear-2 is
 * the variable-step BDF2 with r = dt / dt_prev, ag0 = (1 + 2r) / ((1 + r) dt),
 * ag2 = r^2 / ((1 + r) dt); ag1 defaults to 1. */
static void coeffs(uint32_t method, double dt, double dt_prev, double xmu, double *ag0, double *ag1, double *ag2) {
    *ag2 = 0;
    if (method == 0) { *ag0 = 1.0 / dt; *ag1 = 1; }
    else if (method == 1) { *ag0 = 1.0 / dt / (1.0 - xmu); *ag1 = xmu / (1.0 - xmu); }
    else {
        double r = dt / dt_prev;
        *ag0 = (1.0 + 2.0 * r) / ((1.0 + r) * dt);
        *ag2 = r * r / ((1.0 + r) * dt);
        *ag1 = 1;
    }
}

double orc_step_bound(uint32_t method, uint32_t cur_method, const double *q0, const double *q1, const double *q2,
                      const double *q3, const double *ip, uint32_t len, const double c[10]) {
    /* c: dt dt1 dt2 reltol abstol chgtol trtol ag0 ag1 ag2 (LteIn) */
    double dt = c[0], dt1 = c[1], dt2 = c[2], reltol = c[3], abstol = c[4], chgtol = c[5], trtol = c[6];
    double ag0 = c[7], ag1 = c[8], ag2 = c[9];
    double coeff = method == 0 ? 0.5 : method == 1 ? 0.08333333333 : 0.2222222222;
    double sum01 = dt + dt1, sum12 = dt1 + dt2, sum012 = dt + (dt1 + dt2);
    double vmin = INFINITY, poison = 0;
    for (uint32_t j = 0; j < len; j++) {
        double qc = q0[j], qp = q1[j], qp2 = q2[j], qp3 = q3[j], i_p = ip[j];
        double i_new = cur_method == 1 ? ag0 * (qc - qp) - ag1 * i_p
                     : cur_method == 2 ? ag0 * (qc - qp) - ag2 * (qp - qp2)
                                       : ag0 * (qc - qp);
        double ai = fabs(i_new), ap = fabs(i_p);
        double volttol = abstol + reltol * (ai > ap ? ai : ap);
        double aq = fabs(qc) > fabs(qp) ? fabs(qc) : fabs(qp);
        double chargetol = reltol * (aq > chgtol ? aq : chgtol) / dt;
        double tol = volttol > chargetol ? volttol : chargetol;
        poison += (qc - qc) + (qp - qp) + (qp2 - qp2) + (i_p - i_p);
        double f12 = (qp - qp2) / dt1;
        double dd = ((qc - qp) / dt - f12) / sum01;
        if (method != 0) {
            poison += qp3 - qp3;
            double f123 = (f12 - (qp2 - qp3) / dt2) / sum12;
            dd = (dd - f123) / sum012;
        }
        double den = coeff * fabs(dd);
        double del = trtol * tol / (abstol > den ? abstol : den);
        poison += del == del ? 0 : del;
        vmin = del < vmin ? del : vmin;
    }
    if (isnan(poison)) return NAN;
    return method == 0 ? vmin : sqrt(vmin);
}

static int at_stop(double t, double t_stop) {
    if (t == t_stop) return 1;
    if ((t < 0) != (t_stop < 0)) return 0;
    int64_t a, b;
    memcpy(&a, &t, 8);
    memcpy(&b, &t_stop, 8);
    int64_t d = a - b;
    return (d < 0 ? -d : d) <= 100;
}

/* tran.almostEqualUlps (src/solver/kernels/lane.zig:494-503) */
static int almost_equal_ulps(double a, double b, int64_t max_ulps) {
    if (a == b) return 1;
    int64_t ia, ib;
    memcpy(&ia, &a, 8);
    memcpy(&ib, &b, 8);
    __int128 la = ia < 0 ? (__int128)INT64_MIN - ia : ia;
    __int128 lb = ib < 0 ? (__int128)INT64_MIN - ib : ib;
    __int128 d = la - lb;
    if (d < 0) d = -d;
    return d <= max_ulps;
}

static double next_bp(const ockt *k, double t) {
    double best = INFINITY;
    for (uint32_t bi = 0; bi < k->nb; bi++) {
        const obat *b = &k->b[bi];
        if (b->kind != ESPL_VSRC && b->kind != ESPL_ISRC) continue;
        for (uint32_t i = 0; i < b->count; i++) {
            double v = dev_source_next_bp(b->raw + (size_t)i * b->np, t);
            if (v < best) best = v;
        }
    }
    return best;
}

/* Feeds the sample of every .meas pass at time t, in order (a pass that
 * reads the pass before it sees that pass after this sample). */
static void feed_passes(const espl_meas *passes, uint32_t n, orc_meas_state *mst, double t, const double *x) {
    for (uint32_t p = 0; p < n; p++) {
        const espl_meas *c = &passes[p];
        orc_meas_feed(c, &mst[p], p ? &passes[p - 1] : NULL, p ? &mst[p - 1] : NULL, t, x[c->row],
                      c->level_row ? x[c->level_row - 1] : 0.0);
    }
}

static void tran_one(job_t *j, uint32_t li) {
    const espl_tran_opts *o = j->topts;
    uint32_t lane = j->lane0 + li;
    uint32_t n = j->net->n;
    espl_step_report *rep = &j->reports[li];
    memset(rep, 0, sizeof(*rep));
    ockt *k = ckt_new(j->net, lane, j->q);
    double *x = j->x_out + (size_t)li * n;
    memset(x, 0, sizeof(double) * n);
    if (!k) { rep->status = 4; return; }
    /* Operating point at t = 0 (sources at their t = 0 value), cold. */
    espl_newton_opts op = {o->reltol, o->abstol, o->vntol, 0.0, o->residual_tol, 100, 1};
    seed_limits(k, x, 1);
    orc_newton_result r0 = newton(k, x, &op, 1, 0.0, NULL, NULL);
    if (!r0.converged) { rep->status = 4; ckt_free(k); return; }
    orc_meas_state mst[ESPL_MEAS_MAX_PASSES];
    for (uint32_t p = 0; p < j->n_passes; p++) orc_meas_init(&j->passes[p], &mst[p]);
    feed_passes(j->passes, j->n_passes, mst, 0.0, x);
    uint32_t n1 = n + 1;
    uint32_t ns = k->n_sites;
    /* Row charge ring: logical 1 and 2 start at q(x_op); site ring 1..3 too. */
    eval_planes(k, x, 1, 0.0);
    double *q1 = (double *)malloc(sizeof(double) * n1), *q2 = (double *)malloc(sizeof(double) * n1);
    double *ip = (double *)calloc(n1, sizeof(double));
    memcpy(q1, k->q, sizeof(double) * n1);
    memcpy(q2, k->q, sizeof(double) * n1);
    uint32_t nsa = ns ? ns : 1;
    double *s0 = (double *)calloc(nsa, sizeof(double)), *s1 = (double *)malloc(sizeof(double) * nsa);
    double *s2 = (double *)malloc(sizeof(double) * nsa), *s3 = (double *)malloc(sizeof(double) * nsa);
    double *sip = (double *)calloc(nsa, sizeof(double));
    memcpy(s1, k->qs, sizeof(double) * nsa);
    memcpy(s2, k->qs, sizeof(double) * nsa);
    memcpy(s3, k->qs, sizeof(double) * nsa);
    double *cur = (double *)malloc(sizeof(double) * n), *prev = (double *)malloc(sizeof(double) * n);
    memcpy(cur, x, sizeof(double) * n);
    memcpy(prev, x, sizeof(double) * n);
    double *lim_save = NULL;
    size_t lim_words = 0;
    for (uint32_t bi = 0; bi < k->nb; bi++)
        lim_words += k->b[bi].kind == ESPL_MOS1 ? 3 * (size_t)k->b[bi].count : k->b[bi].kind == ESPL_DIODE ? k->b[bi].count : 0;
    lim_save = (double *)malloc(sizeof(double) * (lim_words ? lim_words : 1));

    double t = 0, dt_max = o->dt_max > 0 ? o->dt_max : o->t_stop / 50.0;
    double dt;
    if (o->fixed_step) {
        dt = o->dt;
    } else {
        dt = fmin(fmin(o->dt, o->t_stop / 100.0) / 10.0, dt_max);
        double bp0 = next_bp(k, 0.0);
        if (bp0 < INFINITY) dt = fmin(dt, 0.1 * bp0);
        dt /= 10.0;
    }
    double dt_old[6];
    for (int i = 0; i < 6; i++) dt_old[i] = o->fixed_step ? o->dt : dt_max;
    uint32_t order = 1, top = o->method; /* top: 0 BE, 1 trap, 2 gear-2 */
    uint32_t steps = 0;
    double bp_next = o->fixed_step ? INFINITY : next_bp(k, 0.0);
    double bp_save_dt = 0;
    int bp_clamped = 0;
    double dt_min = o->dt_min > 0 ? o->dt_min : 1e-9 * dt_max;
    double delmin = 1e-11 * dt_max, min_break = 5e-5 * dt_max;
    uint32_t rows = 0;
    int has_meas = j->meas_row != UINT32_MAX;
    double m_prev_v = 0, m_prev_t = 0, m_first = NAN, m_last = NAN;
    uint32_t m_cross = 0;
    int m_have = 0;
    companion cp;
    while (1) {
        if (!(t < o->t_stop && !at_stop(t, o->t_stop) && steps < o->max_steps)) { rep->status = 1; break; }
        uint32_t method = (order == 1) ? 0 : top;
        double ag0, ag1, ag2;
        coeffs(method, dt, dt_old[0], 0.5, &ag0, &ag1, &ag2);
        double t_dev = t + dt;
        /* Predictor (lane_device.zig predict): trial = cur + xfact (cur - prev). */
        double xfact = dt / dt_old[0];
        if (o->predictor == 1) {
            for (uint32_t i = 0; i < n; i++) x[i] = cur[i] + xfact * (cur[i] - prev[i]);
        } else {
            memcpy(x, cur, sizeof(double) * n);
        }
        /* The limiter state restarts from the accepted point's image, then
         * limits the predicted iterate. */
        seed_limits(k, cur, 0);
        apply_limits(k, x);
        cp.on = 1;
        cp.method = method;
        cp.ag0 = ag0;
        cp.ag1 = ag1;
        cp.ag2 = ag2;
        cp.q1 = q1;
        cp.q2 = q2;
        cp.i_prev = ip;
        espl_newton_opts no = {o->reltol, o->abstol, o->vntol, 0.0, o->residual_tol, o->max_iter, 0};
        orc_newton_result nr = newton(k, x, &no, 1, t_dev, &cp, NULL);
        rep->attempts++;
        rep->nr_iters += nr.singular ? 0 : (nr.iterations < o->max_iter ? nr.iterations : o->max_iter);
        int accept = 0;
        double dt_next = dt;
        if (!nr.converged) {
            rep->rejects++;
            order = 1;
            if (o->fixed_step) { rep->status = 2; break; }
            double old = dt;
            dt = dt / 8.0;
            if (dt < dt_min && old > dt_min && t + dt_min > t) dt = dt_min;
            if (dt < dt_min) { rep->status = 2; break; }
        } else {
            /* The last eval ran at the published x_k: its row and site
             * charges are the converged point's. */
            memcpy(s0, k->qs, sizeof(double) * nsa);
            dt_next = steps == 0 ? dt : fmin(dt * 2.0, dt_max);
            int lte_reject = 0;
            if (!o->fixed_step && ns > 0 && steps > 0) {
                double lin[10] = {dt, dt_old[0], dt_old[1], o->reltol, o->abstol, o->chgtol, o->trtol, ag0, ag1, ag2};
                double del = orc_step_bound(method, method, s0, s1, s2, s3, sip, ns, lin);
                double del2 = method == 0 ? orc_step_bound(top, method, s0, s1, s2, s3, sip, ns, lin) : del;
                if (!(del >= 0.9 * dt)) {
                    rep->rejects++;
                    lte_reject = 1;
                    double old = dt;
                    if (isnan(del)) { order = 1; dt = dt / 8.0; }
                    else dt = del;
                    if (dt < dt_min && old > dt_min && t + dt_min > t) dt = dt_min;
                    if (dt < dt_min) rep->status = 2;
                } else {
                    dt_next = fmin(fmin(fmax(del, dt_min), 2 * dt), dt_max);
                    if (order == 1) {
                        double trial = (top == method) ? del : del2;
                        if (!isnan(trial)) {
                            double nd2 = fmin(2.0 * dt, trial);
                            if (nd2 > 1.05 * dt) order = 2;
                            dt_next = fmin(fmax(nd2, dt_min), dt_max);
                        }
                    }
                }
            } else if (o->fixed_step) {
                dt_next = dt;
                if (order == 1 && top != 0) order = 2;
            } else if (ns == 0) {
                /* No charge: no LTE; ngspice doubles up to dt_max. */
            }
            if (!lte_reject) accept = 1;
        }
        if (!accept) {
            if (rep->status) break;
            continue;
        }
        /* Accept: histories (lane_device.zig accept). */
        for (uint32_t i = 0; i < n1; i++) {
            double d = ag0 * (k->q[i] - q1[i]);
            double nip = method == 1 ? d - ag1 * ip[i] : method == 2 ? d - ag2 * (q1[i] - q2[i]) : d;
            ip[i] = nip;
            q2[i] = q1[i];
            q1[i] = k->q[i];
        }
        for (uint32_t s = 0; s < ns; s++) {
            double d = ag0 * (s0[s] - s1[s]);
            sip[s] = method == 1 ? d - ag1 * sip[s] : method == 2 ? d - ag2 * (s1[s] - s2[s]) : d;
        }
        {
            double *tmp = s3; s3 = s2; s2 = s1; s1 = s0; s0 = tmp;
        }
        memcpy(prev, cur, sizeof(double) * n);
        memcpy(cur, x, sizeof(double) * n);
        for (int i = 5; i > 0; i--) dt_old[i] = dt_old[i - 1];
        dt_old[0] = dt;
        double t_new = t + dt;
        steps++;
        if (j->probe_out && rows < j->max_rows) {
            double *row = j->probe_out + ((size_t)li * j->max_rows + rows) * j->n_probes;
            for (uint32_t pi = 0; pi < j->n_probes; pi++) row[pi] = x[j->probes[pi]];
        }
        rows++;
        feed_passes(j->passes, j->n_passes, mst, t_new, x);
        if (has_meas && t_new >= j->meas_t_start) {
            double v = x[j->meas_row];
            if (m_have && m_prev_v < j->meas_level && v >= j->meas_level) {
                double tc = m_prev_t + (j->meas_level - m_prev_v) * (t_new - m_prev_t) / (v - m_prev_v);
                if (m_cross == 0) m_first = tc;
                m_last = tc;
                m_cross++;
            }
            m_prev_v = v;
            m_prev_t = t_new;
            m_have = 1;
        }
        /* stepEndB: breakpoint landing and the next step's clamp. */
        t = t_new;
        if (!o->fixed_step) {
            double nb = next_bp(k, t_new + min_break);
            if (bp_next != INFINITY) {
                double bp = bp_next;
                int landed = bp_clamped ? fabs(t_new - bp) <= min_break : (bp - t_new <= delmin || almost_equal_ulps(t_new, bp, 100));
                if (landed) {
                    order = 1;
                    double shrink = bp_save_dt;
                    if (nb != INFINITY) shrink = fmin(shrink, nb - t_new);
                    dt_next = fmin(dt_next, 0.1 * shrink);
                }
            }
            bp_next = nb;
            bp_clamped = 0;
            if (nb != INFINITY) {
                double dt_to_bp = nb - t_new;
                if (dt_to_bp < dt_next) {
                    bp_save_dt = dt_next;
                    dt_next = dt_to_bp;
                    bp_clamped = 1;
                }
            }
        }
        dt = dt_next;
        if (t_new + dt > o->t_stop) dt = o->t_stop - t_new;
    }
    rep->t = t;
    rep->dt = dt;
    rep->steps = steps;
    if (has_meas && j->period) j->period[li] = m_cross >= 2 ? (m_last - m_first) / (double)(m_cross - 1) : NAN;
    for (uint32_t p = 0; p < j->n_passes; p++)
        orc_meas_result(&j->passes[p], &mst[p], &j->meas_value[(size_t)li * j->n_passes + p],
                        &j->meas_at[(size_t)li * j->n_passes + p]);
    free(q1); free(q2); free(ip); free(s0); free(s1); free(s2); free(s3); free(sip);
    free(cur); free(prev); free(lim_save);
    ckt_free(k);
}

static void *tran_worker(void *arg) {
    job_t *j = (job_t *)arg;
    for (;;) {
        uint32_t li = atomic_fetch_add(&j->next, 1);
        if (li >= j->count) break;
        tran_one(j, li);
    }
    return NULL;
}

int orc_tran_lanes(const espl_netlist *net, uint32_t lane0, uint32_t count, const espl_tran_opts *opts,
                   const uint32_t *probes, uint32_t n_probes, uint32_t max_rows, double *probe_out,
                   double *x_final, espl_step_report *reports, uint32_t meas_row, double meas_level,
                   double meas_t_start, double *period, uint32_t threads) {
    uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * (net->n ? net->n : 1));
    if (orc_order(net->n, net->col_ptr, net->row_idx, q) != 0) { free(q); return -1; }
    job_t j;
    memset(&j, 0, sizeof(j));
    j.net = net;
    j.lane0 = lane0;
    j.count = count;
    j.topts = opts;
    j.probes = probes;
    j.n_probes = n_probes;
    j.max_rows = max_rows;
    j.probe_out = probe_out;
    j.x_out = x_final;
    j.reports = reports;
    j.meas_row = meas_row;
    j.meas_level = meas_level;
    j.meas_t_start = meas_t_start;
    j.period = period;
    j.q = q;
    atomic_init(&j.next, 0);
    run_pool(&j, threads, tran_worker);
    free(q);
    return 0;
}

int orc_tran_meas(const espl_netlist *net, uint32_t lane0, uint32_t count, const espl_tran_opts *opts,
                  const espl_meas *passes, uint32_t n_passes, double *value, double *at, double *x_final,
                  espl_step_report *reports, uint32_t threads) {
    if (n_passes > ESPL_MEAS_MAX_PASSES) return -1;
    for (uint32_t li = 0; li < count * n_passes; li++) value[li] = at[li] = NAN;
    uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * (net->n ? net->n : 1));
    if (orc_order(net->n, net->col_ptr, net->row_idx, q) != 0) { free(q); return -1; }
    job_t j;
    memset(&j, 0, sizeof(j));
    j.net = net;
    j.lane0 = lane0;
    j.count = count;
    j.topts = opts;
    j.x_out = x_final;
    j.reports = reports;
    j.meas_row = UINT32_MAX;
    j.passes = passes;
    j.n_passes = n_passes;
    j.meas_value = value;
    j.meas_at = at;
    j.q = q;
    atomic_init(&j.next, 0);
    run_pool(&j, threads, tran_worker);
    free(q);
    return 0;
}

int orc_device_probe(const espl_netlist *net, uint32_t b, uint32_t inst, uint32_t lane, const double *v,
                     double *f, double *jac, double *q, double *cjac) {
    /* A one-instance view: evaluate with the limiter state at v (no
     * correction) through the same stamping code, reading rows and slots
     * back by terminal. */
    ockt *k = ckt_new(net, lane, NULL);
    if (!k) return -1;
    double *x = (double *)calloc(net->n + 1, sizeof(double));
    const obat *bb = &k->b[b];
    const uint32_t *tm = bb->term + (size_t)inst * bb->nt;
    for (uint32_t t = 0; t < bb->nt; t++)
        if (tm[t] != ESPL_GROUND) x[tm[t]] = v[t];
    seed_limits(k, x, 0);
    /* Disable every other instance by evaluating this batch alone. */
    obat *keep = k->b;
    uint32_t keep_nb = k->nb;
    obat one = k->b[b];
    one.term = bb->term + (size_t)inst * bb->nt;
    one.slot = bb->slot + (size_t)inst * bb->nt * bb->nt;
    one.raw = bb->raw + (size_t)inst * bb->np;
    one.dio = bb->dio ? bb->dio + inst : NULL;
    one.mos = bb->mos ? bb->mos + inst : NULL;
    one.lim = bb->lim ? bb->lim + (bb->kind == ESPL_MOS1 ? 3 * (size_t)inst : inst) : NULL;
    one.site0 = 0;
    one.count = 1;
    k->b = &one;
    k->nb = 1;
    eval_planes(k, x, 0, 0.0);
    for (uint32_t r = 0; r < one.nt; r++) {
        uint32_t row = tm[r];
        f[r] = row == ESPL_GROUND ? 0.0 : k->rhs[row] - (row == 0 ? x[0] : 0.0);
        if (q) q[r] = row == ESPL_GROUND ? 0.0 : k->q[row];
        for (uint32_t c = 0; c < one.nt; c++) {
            uint32_t s = one.slot[r * one.nt + c];
            double gv = (s == UINT32_MAX || s == k->nnz) ? 0.0 : k->g[s];
            if (s == k->diag[0]) gv -= 1.0;
            jac[r * one.nt + c] = gv;
            if (cjac) cjac[r * one.nt + c] = (s == UINT32_MAX || s == k->nnz) ? 0.0 : k->c[s];
        }
    }
    k->b = keep;
    k->nb = keep_nb;
    free(x);
    ckt_free(k);
    return 0;
}

/* Acklam's inverse normal, as src/core/numerics.zig:416-432 states it. */
double orc_normal_quantile(double u) {
    static const double a[] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                               1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                               6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                               -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                               3.754408661907416e+00};
    const double low = 0.02425;
    if (u < low || u > 1 - low) {
        double q = sqrt(-2 * log(u < low ? u : 1 - u));
        double x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
                   ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
        return u < low ? x : -x;
    }
    double q = u - 0.5, r = q * q;
    return (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
           (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1);
}

/* src/frontend/netlist.zig:683-688 */
uint64_t orc_site_key(uint64_t owner, uint64_t salt) {
    uint64_t z = owner ^ (salt + 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
