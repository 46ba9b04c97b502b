/* ORACLE (test infrastructure only; never linked into the product).
 *
 * Left-looking Gilbert-Peierls sparse LU restated from ESPice
 * src/solver/sparse_lu.zig:
 *   - factor / factorPass: sparse_lu.zig:274-311, 337-663 (DFS reach,
 *     triangular solve, threshold pivot with the row-scaled second chance,
 *     the want/want_of hand-off, void unknowns, the fill cap restart);
 *   - the supernodal walk: enter / panelEnd / linkStep / growPanel /
 *     panelRun, sparse_lu.zig:754-910;
 *   - refactor (column replay, growth monitor): sparse_lu.zig:973-1160;
 *   - solve / solveT: sparse_lu.zig:1277-1361.
 * and the LU engine of the direct solver src/solver/direct.zig:310-447
 * (bypass on unchanged values, replay + replayHolds probe, full factor;
 * pivot_tol direct.zig:33, repivot_fill_cap direct.zig:36,
 * refactor_growth_limit direct.zig:54, replay_ratio_max direct.zig:667).
 * The flat refactor tape (sparse_lu.zig:1166-1271) is bitwise the column
 * replay, so only the column replay is restated.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NONE 0xFFFFFFFFu
#define PANEL_MIN_ROWS 32u

typedef struct { uint32_t first, last, row_off, val_off; } panel_t;

#define VEC(T) struct { T *d; size_t len, cap; }
#define VPUSH(v, x)                                                            \
    do {                                                                       \
        if ((v).len == (v).cap) {                                              \
            (v).cap = (v).cap ? 2 * (v).cap : 64;                              \
            (v).d = realloc((v).d, sizeof(*(v).d) * (v).cap);                  \
        }                                                                      \
        (v).d[(v).len++] = (x);                                                \
    } while (0)
#define VRESERVE(v, m)                                                         \
    do {                                                                       \
        if ((v).len + (m) > (v).cap) {                                         \
            size_t nc_ = (v).cap ? (v).cap : 64;                               \
            while (nc_ < (v).len + (m)) nc_ *= 2;                              \
            (v).cap = nc_;                                                     \
            (v).d = realloc((v).d, sizeof(*(v).d) * (v).cap);                  \
        }                                                                      \
    } while (0)

struct orc_lu {
    uint32_t n, nnz;
    uint32_t *q; /* owned copy */
    uint32_t *pinv, *lp, *up, *prow;
    VEC(uint32_t) li;
    VEC(double) lx;
    VEC(uint32_t) ui;
    VEC(double) ux;
    double *udiag;
    uint8_t *void_col, *scaled_pivot;
    VEC(uint32_t) void_slots;
    double *w, *y, *rscale;
    uint32_t *want, *want_of, *prev, *flag, *topo, *stack, *pstack, *lend, *sn_of, *sn_slot, *sn_end;
    int sn_dfs;
    VEC(panel_t) panels;
    VEC(uint32_t) panel_rows;
    VEC(double) panel_vals;
    size_t base_lu;
    uint64_t diag_fill;
    double fill_cap, keep_min;
    int factored;
    int has_replay_mult;
    double replay_mult;
};

orc_lu *orc_lu_new(uint32_t n, const uint32_t *col_ptr, const uint32_t *q) {
    orc_lu *s = (orc_lu *)calloc(1, sizeof(orc_lu));
    s->n = n;
    s->nnz = col_ptr[n];
    size_t nn = n ? n : 1;
    s->q = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    memcpy(s->q, q, sizeof(uint32_t) * n);
    s->pinv = (uint32_t *)malloc(sizeof(uint32_t) * nn);
    s->lp = (uint32_t *)calloc(n + 1, sizeof(uint32_t));
    s->up = (uint32_t *)calloc(n + 1, sizeof(uint32_t));
    s->prow = (uint32_t *)malloc(sizeof(uint32_t) * (s->nnz ? s->nnz : 1));
    s->udiag = (double *)calloc(nn, sizeof(double));
    s->void_col = (uint8_t *)calloc(nn, 1);
    s->scaled_pivot = (uint8_t *)calloc(nn, 1);
    s->w = (double *)calloc(nn, sizeof(double));
    s->y = (double *)calloc(nn, sizeof(double));
    s->rscale = (double *)calloc(nn, sizeof(double));
    uint32_t **u32s[] = {&s->want, &s->want_of, &s->prev, &s->flag, &s->topo, &s->stack,
                         &s->pstack, &s->lend, &s->sn_of, &s->sn_slot, &s->sn_end};
    for (size_t i = 0; i < sizeof(u32s) / sizeof(u32s[0]); i++) *u32s[i] = (uint32_t *)calloc(nn, sizeof(uint32_t));
    return s;
}

void orc_lu_free(orc_lu *s) {
    if (!s) return;
    free(s->q); free(s->pinv); free(s->lp); free(s->up); free(s->prow);
    free(s->li.d); free(s->lx.d); free(s->ui.d); free(s->ux.d); free(s->udiag);
    free(s->void_col); free(s->scaled_pivot); free(s->void_slots.d);
    free(s->w); free(s->y); free(s->rscale);
    free(s->want); free(s->want_of); free(s->prev); free(s->flag); free(s->topo); free(s->stack);
    free(s->pstack); free(s->lend); free(s->sn_of); free(s->sn_slot); free(s->sn_end);
    free(s->panels.d); free(s->panel_rows.d); free(s->panel_vals.d);
    free(s);
}

void orc_lu_set_caps(orc_lu *s, uint64_t diag_fill, double fill_cap, double keep_min) {
    s->diag_fill = diag_fill;
    s->fill_cap = fill_cap;
    s->keep_min = keep_min;
}

static int is_finite(double x) { return fabs(x) <= DBL_MAX; }

static uint64_t bits_of(double x) {
    uint64_t b;
    memcpy(&b, &x, 8);
    return b;
}

static double float_of(uint64_t b) {
    double x;
    memcpy(&x, &b, 8);
    return x;
}

/* sparse_lu.zig:771-774 */
static uint32_t panel_end(const orc_lu *s, uint32_t kc) {
    panel_t pan = s->panels.d[s->sn_of[kc]];
    return pan.row_off + s->lp[pan.first + 1] - s->lp[pan.first];
}

/* sparse_lu.zig:754-768 */
static uint32_t enter(orc_lu *s, uint32_t r, uint32_t sp, uint32_t mark) {
    uint32_t kc = s->pinv[r];
    s->sn_end[sp] = NONE;
    if (kc == NONE) return 0;
    uint32_t id = s->sn_of[kc];
    if (id == NONE || !s->sn_dfs) return s->lp[kc];
    panel_t pan = s->panels.d[id];
    const uint32_t *rows = s->panel_rows.d + pan.row_off;
    uint32_t e = kc;
    while (e < pan.last && s->flag[rows[e - pan.first]] != mark) {
        s->flag[rows[e - pan.first]] = mark;
        e++;
    }
    s->sn_end[sp] = e;
    uint32_t m = pan.last - pan.first + 1;
    return e == pan.last ? pan.row_off + m - 1 : panel_end(s, kc);
}

/* sparse_lu.zig:803-850 */
static void grow_panel(orc_lu *s, uint32_t k, uint32_t piv) {
    uint32_t *lp = s->lp;
    if (s->sn_of[k - 1] == NONE) {
        uint32_t first = k - 1;
        s->sn_of[first] = (uint32_t)s->panels.len;
        panel_t np = {first, first, (uint32_t)s->panel_rows.len, (uint32_t)s->panel_vals.len};
        VPUSH(s->panels, np);
        for (uint32_t i = 0, p = lp[first]; p < lp[k]; p++, i++) {
            s->sn_slot[s->li.d[p]] = i;
            VPUSH(s->panel_rows, s->li.d[p]);
            VPUSH(s->panel_vals, s->lx.d[p]);
        }
    }
    uint32_t pid = s->sn_of[k - 1];
    panel_t *pan = &s->panels.d[pid];
    uint32_t nrows = lp[pan->first + 1] - lp[pan->first];
    VRESERVE(s->panel_vals, nrows);
    pan = &s->panels.d[pid];
    uint32_t *rows = s->panel_rows.d + pan->row_off;
    uint32_t b = k - pan->first - 1;
    uint32_t a = s->sn_slot[piv];
    if (a != b) {
        double *vals = s->panel_vals.d + pan->val_off;
        for (uint32_t col = 0; col < k - pan->first; col++) {
            double t = vals[col * nrows + a];
            vals[col * nrows + a] = vals[col * nrows + b];
            vals[col * nrows + b] = t;
        }
        s->sn_slot[rows[b]] = a;
        s->sn_slot[piv] = b;
        uint32_t t = rows[a];
        rows[a] = rows[b];
        rows[b] = t;
    }
    size_t dst0 = s->panel_vals.len;
    s->panel_vals.len += nrows;
    double *dst = s->panel_vals.d + dst0;
    memset(dst, 0, sizeof(double) * nrows);
    for (size_t p = lp[k]; p < s->li.len; p++) dst[s->sn_slot[s->li.d[p]]] = s->lx.d[p];
    pan->last = k;
    s->sn_of[k] = pid;
}

/* sparse_lu.zig:780-798 */
static void link_step(orc_lu *s, uint32_t k, uint32_t piv, uint32_t mark) {
    uint32_t sidx = k - 1;
    uint32_t at = NONE, last_out = NONE;
    uint32_t c0 = s->lp[sidx], c1 = s->lp[k];
    for (uint32_t p = c0, i = 0; p < c1; p++, i++) {
        uint32_t r = s->li.d[p];
        if (r == piv) at = i;
        else if (s->flag[r] != mark || s->pinv[r] != NONE) last_out = i;
    }
    if (at == NONE || (last_out != NONE && last_out > at)) return;
    s->lend[sidx] = s->lp[sidx] + at + 1;
    int joins = last_out == NONE && (c1 - c0) == s->li.len - s->lp[k] + 1;
    if (joins) grow_panel(s, k, piv);
}

/* sparse_lu.zig:857-892 */
static uint32_t panel_run(orc_lu *s, double *w, const uint32_t *topo, uint32_t idx0, uint32_t kc) {
    panel_t pan = s->panels.d[s->sn_of[kc]];
    uint32_t nrows = s->lp[pan.first + 1] - s->lp[pan.first];
    uint32_t m = pan.last - pan.first + 1;
    const uint32_t *rows = s->panel_rows.d + pan.row_off;
    const double *vals = s->panel_vals.d + pan.val_off;
    uint32_t len = 1;
    while (kc + len <= pan.last && len <= idx0 && s->pinv[topo[idx0 - len]] == kc + len) len++;
    uint32_t b0 = kc - pan.first;
    double *x = s->y;
    uint32_t xn = m - 1 - b0;
    for (uint32_t i = 0; i < xn; i++) x[i] = w[rows[b0 + i]];
    size_t run0 = s->ux.len;
    for (uint32_t j = 0; j < len; j++) {
        uint32_t t = kc + j;
        double ut = j == 0 ? w[topo[idx0]] : x[j - 1];
        VPUSH(s->ui, t);
        VPUSH(s->ux, ut);
        const double *col = vals + (size_t)(t - pan.first) * nrows;
        for (uint32_t i = j; i < xn; i++) x[i] -= col[b0 + i] * ut;
    }
    for (uint32_t i = 0; i < xn; i++) w[rows[b0 + i]] = x[i];
    const double *u = s->ux.d + run0;
    const double *cv = vals + (size_t)b0 * nrows;
    for (uint32_t i = m - 1; i < nrows; i++) {
        double acc = w[rows[i]];
        for (uint32_t j = 0; j < len; j++) acc -= cv[(size_t)j * nrows + i] * u[j];
        w[rows[i]] = acc;
    }
    return idx0 - (len - 1);
}

/* sparse_lu.zig:916-935 */
static int void_unknown(const orc_lu *s, const uint32_t *col_ptr, const uint32_t *row_idx, const double *vals, uint32_t c) {
    if (s->pinv[c] != NONE) return 0;
    for (uint32_t p = col_ptr[c]; p < col_ptr[c + 1]; p++)
        if (vals[p] != 0) return 0;
    for (uint32_t j = 0; j < s->n; j++) {
        if (j == c) continue;
        for (uint32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++)
            if (row_idx[p] == c && vals[p] != 0) return 0;
    }
    return 1;
}

/* One full factor (sparse_lu.zig:337-663). Returns 0 factored, 1 over the
 * fill cap (unfactored), -1 singular. */
static int factor_pass(orc_lu *s, const uint32_t *col_ptr, const uint32_t *row_idx, const double *vals,
                       double pivot_tol, size_t cap, int keep_prev) {
    uint32_t n = s->n;
    s->factored = 0;
    s->has_replay_mult = 0;
    for (uint32_t i = 0; i < n; i++) {
        s->pinv[i] = NONE;
        s->flag[i] = 0;
        s->void_col[i] = 0;
        s->scaled_pivot[i] = 0;
    }
    s->panels.len = s->panel_rows.len = s->panel_vals.len = 0;
    s->void_slots.len = 0;
    int has_void = 0;
    s->li.len = s->lx.len = s->ui.len = s->ux.len = 0;

    memset(s->rscale, 0, sizeof(double) * n);
    /* num.normInf over vals: NaN or inf fails the factor. */
    uint64_t mb = 0;
    for (uint32_t p = 0; p < s->nnz; p++) {
        uint64_t b = bits_of(fabs(vals[p]));
        if (b > mb) mb = b;
    }
    if (!(float_of(mb) <= DBL_MAX)) return -1;
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
            double a = fabs(vals[p]);
            if (a > s->rscale[row_idx[p]]) s->rscale[row_idx[p]] = a;
        }
    for (uint32_t i = 0; i < n; i++) {
        double v = s->rscale[i];
        s->rscale[i] = (v > 0 && is_finite(v)) ? 1 / v : 1;
    }
    uint32_t *pinv = s->pinv, *flag = s->flag, *stack = s->stack, *pstack = s->pstack, *topo = s->topo;
    uint32_t *lp = s->lp, *lend = s->lend, *want = s->want, *want_of = s->want_of;
    double *w = s->w, *rscale = s->rscale;
    uint64_t nonfinite = 0;
    for (uint32_t i = 0; i < n; i++) want[i] = keep_prev ? s->prev[i] : i;
    for (uint32_t c = 0; c < n; c++) want_of[want[c]] = c;

    uint32_t k = 0;
    for (int sn = 0; sn <= 1; sn++) {
        if (sn) {
            lp[k] = (uint32_t)s->li.len;
            for (uint32_t t = 0; t < k; t++) lend[t] = lp[t + 1];
            for (uint32_t t = 0; t < n; t++) s->sn_of[t] = NONE;
            s->sn_dfs = 0;
        }
        int broke = 0;
        while (k < n) {
            uint32_t c = s->q[k];
            lp[k] = (uint32_t)s->li.len;
            s->up[k] = (uint32_t)s->ui.len;
            uint32_t mark = k + 1;
            uint32_t nt = 0;
            for (uint32_t p = col_ptr[c]; p < col_ptr[c + 1]; p++) {
                uint32_t r = row_idx[p];
                if (flag[r] == mark) continue;
                uint32_t sp = 0;
                stack[sp] = r;
                flag[r] = mark;
                pstack[sp] = sn ? enter(s, r, sp, mark) : (pinv[r] == NONE ? 0 : lp[pinv[r]]);
                for (;;) {
                    r = stack[sp];
                    uint32_t kc = pinv[r];
                    int in_panel = sn && kc != NONE && s->sn_end[sp] != NONE;
                    const uint32_t *adj = in_panel ? s->panel_rows.d : s->li.d;
                    uint32_t end = kc == NONE ? 0 : in_panel ? panel_end(s, kc) : sn ? lend[kc] : lp[kc + 1];
                    uint32_t pos = pstack[sp];
                    int descended = 0;
                    while (pos < end) {
                        uint32_t child = adj[pos];
                        pos++;
                        if (flag[child] != mark) {
                            pstack[sp] = pos;
                            flag[child] = mark;
                            sp++;
                            stack[sp] = child;
                            pstack[sp] = sn ? enter(s, child, sp, mark) : (pinv[child] == NONE ? 0 : lp[pinv[child]]);
                            descended = 1;
                            break;
                        }
                    }
                    if (descended) continue;
                    if (in_panel) {
                        panel_t pan = s->panels.d[s->sn_of[kc]];
                        const uint32_t *rows = s->panel_rows.d + pan.row_off;
                        for (uint32_t t = s->sn_end[sp]; t > kc; t--) topo[nt++] = rows[t - pan.first - 1];
                    }
                    topo[nt++] = r;
                    if (sp == 0) break;
                    sp--;
                }
            }
            VRESERVE(s->ui, nt);
            VRESERVE(s->ux, nt);
            VRESERVE(s->li, nt);
            VRESERVE(s->lx, nt);
            for (uint32_t p = col_ptr[c]; p < col_ptr[c + 1]; p++) w[row_idx[p]] = vals[p];
            uint32_t idx = nt;
            while (idx > 0) {
                idx--;
                uint32_t r = topo[idx];
                uint32_t kc = pinv[r];
                if (kc == NONE) continue;
                if (sn && s->panels.len != 0 && s->sn_of[kc] != NONE) {
                    idx = panel_run(s, w, topo, idx, kc);
                    continue;
                }
                double ukr = w[r];
                s->ui.d[s->ui.len++] = kc;
                s->ux.d[s->ux.len++] = ukr;
                for (uint32_t q2 = lp[kc]; q2 < lp[kc + 1]; q2++) w[s->li.d[q2]] -= s->lx.d[q2] * ukr;
            }
            double amax = 0, smax = 0;
            uint32_t piv = NONE;
            for (uint32_t t = 0; t < nt; t++) {
                uint32_t r = topo[t];
                if (pinv[r] != NONE) continue;
                double a = fabs(w[r]);
                if (a > amax) { amax = a; piv = r; }
                double sa = a * rscale[r];
                /* @max: NaN-propagating. */
                smax = (sa != sa || smax != smax) ? NAN : (sa > smax ? sa : smax);
            }
            if (piv == NONE || amax == 0 || !is_finite(amax)) {
                if (!void_unknown(s, col_ptr, row_idx, vals, c)) {
                    for (uint32_t t = 0; t < nt; t++) w[topo[t]] = 0;
                    return -1;
                }
                s->void_col[k] = 1;
                has_void = 1;
                s->udiag[k] = 1;
                pinv[c] = k;
                if (sn) lend[k] = lp[k];
                for (uint32_t t = 0; t < nt; t++) w[topo[t]] = 0;
                k++;
                continue;
            }
            uint32_t pr = want[c];
            if (pinv[pr] == NONE) {
                double dmag = fabs(w[pr]);
                if (keep_prev) {
                    if (dmag > 0 && dmag >= s->keep_min * amax) piv = pr;
                } else if (dmag > 0 && dmag >= pivot_tol * amax) {
                    piv = pr;
                } else if (dmag > 0 && dmag * rscale[pr] >= pivot_tol * smax) {
                    piv = pr;
                    s->scaled_pivot[k] = 1;
                }
            }
            if (piv != pr) {
                uint32_t c2 = want_of[piv];
                want[c2] = pr;
                want_of[pr] = c2;
            }
            double d = w[piv];
            s->udiag[k] = d;
            pinv[piv] = k;
            for (uint32_t t = 0; t < nt; t++) {
                uint32_t r = topo[t];
                double v = w[r];
                nonfinite |= bits_of(v - v);
                if (pinv[r] == NONE) {
                    double l = v / d;
                    nonfinite |= bits_of(l - l);
                    s->li.d[s->li.len++] = r;
                    s->lx.d[s->lx.len++] = l;
                }
                w[r] = 0;
            }
            if (s->li.len + s->ui.len > cap) return 1;
            if (!sn) {
                if (s->li.len - lp[k] >= PANEL_MIN_ROWS) {
                    k++;
                    broke = 1;
                    break;
                }
                k++;
                continue;
            }
            lend[k] = (uint32_t)s->li.len;
            if (k > 0 && (lp[k] - lp[k - 1] >= PANEL_MIN_ROWS || s->sn_of[k - 1] != NONE)) link_step(s, k, piv, mark);
            if (s->panel_vals.len >= s->li.len / 5 * 4) s->sn_dfs = 1;
            k++;
        }
        (void)broke;
    }
    lp[n] = (uint32_t)s->li.len;
    s->up[n] = (uint32_t)s->ui.len;
    if (nonfinite != 0) return -1;
    for (size_t p = 0; p < s->li.len; p++) s->li.d[p] = pinv[s->li.d[p]];
    for (uint32_t p = 0; p < s->nnz; p++) s->prow[p] = pinv[row_idx[p]];
    if (has_void) {
        for (uint32_t j = 0; j < n; j++) {
            uint32_t c = s->q[j];
            for (uint32_t p = col_ptr[c]; p < col_ptr[c + 1]; p++)
                if (s->void_col[j] || s->void_col[s->prow[p]]) VPUSH(s->void_slots, p);
        }
    }
    s->factored = 1;
    return 0;
}

/* sparse_lu.zig:274-311. 0 ok, -1 singular. */
int orc_lu_factor(orc_lu *s, const uint32_t *col_ptr, const uint32_t *row_idx, const double *vals, double pivot_tol) {
    int repivot = s->factored && s->fill_cap > 0 && s->base_lu > 0;
    size_t cap = SIZE_MAX;
    if (repivot) {
        for (uint32_t r = 0; r < s->n; r++) s->prev[s->q[s->pinv[r]]] = r;
        double c = s->fill_cap * (double)s->base_lu;
        cap = (size_t)(c < 1e18 ? c : 1e18);
    } else if (s->fill_cap > 0 && s->diag_fill > 0) {
        for (uint32_t c = 0; c < s->n; c++) s->prev[c] = c;
        double c = s->fill_cap * (double)s->diag_fill;
        cap = (size_t)(c < 1e18 ? c : 1e18);
    }
    int r = factor_pass(s, col_ptr, row_idx, vals, pivot_tol, cap, 0);
    if (r < 0) return -1;
    if (r == 1) {
        int r2 = factor_pass(s, col_ptr, row_idx, vals, pivot_tol, repivot ? SIZE_MAX : cap, 1);
        if (r2 != 0) return -1;
    }
    if (!repivot) s->base_lu = s->li.len + s->ui.len;
    return 0;
}

/* sparse_lu.zig:973-1160 (column replay). 0 ok, -1 singular. */
int orc_lu_refactor(orc_lu *s, const uint32_t *col_ptr, const double *vals, double growth_limit) {
    for (size_t v = 0; v < s->void_slots.len; v++)
        if (vals[s->void_slots.d[v]] != 0) return -1;
    uint64_t nonfinite = 0;
    double mult = 0;
    double *w = s->w;
    const uint32_t *li = s->li.d, *ui = s->ui.d, *lp = s->lp, *up = s->up;
    double *lx = s->lx.d, *ux = s->ux.d;
    for (uint32_t k = 0; k < s->n; k++) {
        uint32_t c = s->q[k];
        for (uint32_t p = col_ptr[c]; p < col_ptr[c + 1]; p++) w[s->prow[p]] = vals[p];
        for (uint32_t p = up[k]; p < up[k + 1]; p++) {
            uint32_t i = ui[p];
            double uki = w[i];
            w[i] = 0;
            ux[p] = uki;
            nonfinite |= bits_of(uki - uki);
            for (uint32_t q2 = lp[i]; q2 < lp[i + 1]; q2++) w[li[q2]] -= lx[q2] * uki;
        }
        if (s->void_col[k]) {
            s->udiag[k] = 1;
            for (uint32_t p = lp[k]; p < lp[k + 1]; p++) { lx[p] = 0; w[li[p]] = 0; }
            w[k] = 0;
            for (uint32_t p = up[k]; p < up[k + 1]; p++) {
                uint32_t i = ui[p];
                for (uint32_t q2 = lp[i]; q2 < lp[i + 1]; q2++) w[li[q2]] = 0;
            }
            continue;
        }
        double d = w[k];
        w[k] = 0;
        if (d == 0 || !is_finite(d)) {
            for (uint32_t p = lp[k]; p < lp[k + 1]; p++) w[li[p]] = 0;
            s->has_replay_mult = 0;
            return -1;
        }
        s->udiag[k] = d;
        if (growth_limit > 0 && !s->scaled_pivot[k]) {
            int64_t cbits = (int64_t)bits_of(fabs(d));
            for (uint32_t p = lp[k]; p < lp[k + 1]; p++) {
                uint32_t row = li[p];
                double v = w[row];
                w[row] = 0;
                int64_t b = (int64_t)bits_of(fabs(v));
                if (b > cbits) cbits = b;
                lx[p] = v / d;
            }
            double cmax = float_of((uint64_t)cbits);
            if (!(fabs(d) >= growth_limit * cmax)) {
                /* The remaining columns still hold zero in w: only this
                 * column's rows were scattered, and they are cleared. */
                s->has_replay_mult = 0;
                return -1;
            }
            double r = cmax / fabs(d);
            if (r > mult) mult = r;
            continue;
        }
        for (uint32_t p = lp[k]; p < lp[k + 1]; p++) {
            uint32_t row = li[p];
            double l = w[row] / d;
            nonfinite |= bits_of(l - l);
            lx[p] = l;
            w[row] = 0;
        }
    }
    s->has_replay_mult = 0;
    if (nonfinite != 0) return -1;
    if (growth_limit > 0) { s->has_replay_mult = 1; s->replay_mult = mult; }
    return 0;
}

/* sparse_lu.zig:1277-1321. b and x may alias. */
void orc_lu_solve(orc_lu *s, const double *b, double *x) {
    uint32_t n = s->n;
    double *y = s->y;
    const uint32_t *li = s->li.d, *ui = s->ui.d;
    const double *lx = s->lx.d, *ux = s->ux.d;
    for (uint32_t r = 0; r < n; r++) y[s->pinv[r]] = b[r];
    for (uint32_t k = 0; k < n; k++) {
        double yk = y[k];
        if (yk == 0) continue;
        for (uint32_t p = s->lp[k]; p < s->lp[k + 1]; p++) y[li[p]] -= lx[p] * yk;
    }
    for (uint32_t k = n; k > 0;) {
        k--;
        double zk = y[k] / s->udiag[k];
        y[k] = zk;
        if (zk == 0) continue;
        for (uint32_t p = s->up[k]; p < s->up[k + 1]; p++) y[ui[p]] -= ux[p] * zk;
    }
    for (uint32_t j = 0; j < n; j++) x[s->q[j]] = y[j];
}

/* sparse_lu.zig:1326-1361 */
void orc_lu_solve_t(orc_lu *s, const double *b, double *x) {
    uint32_t n = s->n;
    double *y = s->y;
    for (uint32_t k = 0; k < n; k++) y[k] = b[s->q[k]];
    for (uint32_t k = 0; k < n; k++) {
        double yk = y[k];
        for (uint32_t p = s->up[k]; p < s->up[k + 1]; p++) yk -= s->ux.d[p] * y[s->ui.d[p]];
        y[k] = yk / s->udiag[k];
    }
    for (uint32_t k = n; k > 0;) {
        k--;
        double yk = y[k];
        for (uint32_t p = s->lp[k]; p < s->lp[k + 1]; p++) yk -= s->lx.d[p] * y[s->li.d[p]];
        y[k] = yk;
    }
    for (uint32_t r = 0; r < n; r++) x[r] = y[s->pinv[r]];
}

void orc_lu_tape(const orc_lu *s, orc_tape *t) {
    t->n = s->n;
    t->nnz = s->nnz;
    t->nnz_l = (uint32_t)s->li.len;
    t->nnz_u = (uint32_t)s->ui.len;
    t->q = s->q;
    t->pinv = s->pinv;
    t->lp = s->lp;
    t->li = s->li.d;
    t->up = s->up;
    t->ui = s->ui.d;
    t->prow = s->prow;
    t->void_col = s->void_col;
    t->scaled_pivot = s->scaled_pivot;
    t->void_slots = s->void_slots.d;
    t->n_void_slots = (uint32_t)s->void_slots.len;
    t->lx = s->lx.d;
    t->ux = s->ux.d;
    t->udiag = s->udiag;
    t->sn_dfs = (uint32_t)s->sn_dfs;
    t->n_panels = (uint32_t)s->panels.len;
}

/* ------------------------------------------------------------------ */
/* Direct solver, LU engine only: direct.zig:310-447.                  */

struct orc_direct {
    uint32_t n;
    const uint32_t *col_ptr, *row_idx;
    uint32_t *q;
    orc_lu *lu;
    double *vcopy;
    double *probe;
    int factored;
    double growth;
};

orc_direct *orc_direct_new(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, const uint32_t *q_or_null) {
    orc_direct *d = (orc_direct *)calloc(1, sizeof(orc_direct));
    d->n = n;
    d->col_ptr = col_ptr;
    d->row_idx = row_idx;
    d->q = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    if (q_or_null) memcpy(d->q, q_or_null, sizeof(uint32_t) * n);
    else if (orc_order(n, col_ptr, row_idx, d->q) != 0) { free(d->q); free(d); return NULL; }
    d->lu = orc_lu_new(n, col_ptr, d->q);
    /* direct.zig:240: at least nnz(A). */
    uint64_t df = orc_diag_fill(n, col_ptr, row_idx, d->q);
    if (df < col_ptr[n]) df = col_ptr[n];
    orc_lu_set_caps(d->lu, df, ORC_REPIVOT_FILL_CAP, ORC_GROWTH_LIMIT);
    d->vcopy = (double *)calloc(col_ptr[n] ? col_ptr[n] : 1, sizeof(double));
    d->probe = (double *)calloc(3 * (size_t)(n ? n : 1), sizeof(double));
    d->growth = ORC_GROWTH_LIMIT;
    return d;
}

void orc_direct_free(orc_direct *d) {
    if (!d) return;
    orc_lu_free(d->lu);
    free(d->q);
    free(d->vcopy);
    free(d->probe);
    free(d);
}

orc_lu *orc_direct_lu(orc_direct *d) { return d->lu; }
const uint32_t *orc_direct_q(const orc_direct *d) { return d->q; }

/* direct.zig:674-700 */
static double max_multiplier(const orc_lu *lu) {
    if (lu->has_replay_mult) return lu->replay_mult < 1 ? 1 : lu->replay_mult;
    uint64_t m = bits_of(1.0);
    for (uint32_t k = 0; k < lu->n; k++) {
        if (lu->scaled_pivot[k]) continue;
        for (uint32_t p = lu->lp[k]; p < lu->lp[k + 1]; p++) {
            uint64_t b = bits_of(fabs(lu->lx.d[p]));
            if (b > m) m = b;
        }
    }
    return float_of(m);
}

/* direct.zig:702-708 */
static void probe_rhs(double *b, uint32_t n) {
    double den = (double)((n > 2 ? n : 2) - 1);
    for (uint32_t i = 0; i < n; i++) {
        double mag = 1 + (double)i / den;
        b[i] = i % 2 == 0 ? mag : -mag;
    }
}

static double norm_inf(const double *x, uint32_t n) {
    uint64_t m = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint64_t b = bits_of(fabs(x[i]));
        if (b > m) m = b;
    }
    return float_of(m);
}

/* direct.zig:402-447 */
static int replay_holds(orc_direct *d, const double *vals) {
    orc_lu *lu = d->lu;
    if (max_multiplier(lu) <= 1 / ORC_PIVOT_TOL) return 1;
    uint32_t n = d->n;
    double *x = d->probe, *r = d->probe + n, *rows = d->probe + 2 * n;
    memset(rows, 0, sizeof(double) * n);
    double norm_1 = 0;
    for (uint32_t j = 0; j < n; j++) {
        double col = 0;
        for (uint32_t p = d->col_ptr[j]; p < d->col_ptr[j + 1]; p++) {
            double a = fabs(vals[p]);
            rows[d->row_idx[p]] += a;
            col += a;
        }
        norm_1 = col > norm_1 ? col : norm_1;
    }
    double norm_i = norm_inf(rows, n);
    double nf = (double)n;
    for (int transpose = 0; transpose <= 1; transpose++) {
        probe_rhs(r, n);
        if (transpose) orc_lu_solve_t(lu, r, x);
        else orc_lu_solve(lu, r, x);
        probe_rhs(r, n);
        for (uint32_t j = 0; j < n; j++)
            for (uint32_t p = d->col_ptr[j]; p < d->col_ptr[j + 1]; p++) {
                uint32_t i = d->row_idx[p];
                if (transpose) r[j] -= vals[p] * x[i];
                else r[i] -= vals[p] * x[j];
            }
        double a_norm = transpose ? norm_1 : norm_i;
        double ratio = norm_inf(r, n) / (a_norm * norm_inf(x, n) * nf * DBL_EPSILON);
        if (!(ratio <= ORC_REPLAY_RATIO_MAX / ORC_PIVOT_TOL)) return 0;
    }
    return 1;
}

/* direct.zig:310-388 (LU engine). 0 ok, -1 singular. Sets *path to 0
 * bypass, 1 replay, 2 full factor. */
int orc_direct_factor(orc_direct *d, const double *vals, int *path) {
    uint32_t nnz = d->col_ptr[d->n];
    if (nnz != 0 && d->factored && memcmp(d->vcopy, vals, sizeof(double) * nnz) == 0) {
        /* simdEql compares values: +0 == -0 and NaN != NaN; a bitwise match
         * is a value match except for NaN, which a factored matrix cannot
         * hold. Check the value comparison exactly. */
        if (path) *path = 0;
        return 0;
    }
    int equal = nnz != 0 && d->factored;
    for (uint32_t p = 0; equal && p < nnz; p++) equal = d->vcopy[p] == vals[p];
    if (equal) {
        if (path) *path = 0;
        return 0;
    }
    if (d->factored) {
        if (orc_lu_refactor(d->lu, d->col_ptr, vals, d->growth) == 0 && replay_holds(d, vals)) {
            memcpy(d->vcopy, vals, sizeof(double) * nnz);
            if (path) *path = 1;
            return 0;
        }
        d->factored = 0;
    }
    if (orc_lu_factor(d->lu, d->col_ptr, d->row_idx, vals, ORC_PIVOT_TOL) != 0) {
        d->factored = 0;
        return -1;
    }
    d->factored = 1;
    memcpy(d->vcopy, vals, sizeof(double) * nnz);
    if (path) *path = 2;
    return 0;
}

/* direct.Solver.solveNeg: x = -A^-1 b. */
void orc_direct_solve_neg(orc_direct *d, const double *b, double *x) {
    orc_lu_solve(d->lu, b, x);
    for (uint32_t i = 0; i < d->n; i++) x[i] = -x[i];
}
