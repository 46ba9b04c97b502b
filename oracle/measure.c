/* Test infrastructure only (the oracle): the streaming .meas passes the
 * GPU lanes run, restated in plain C from the reference's sample-at-a-time
 * measures (src/output/scan.zig: Cross :61-169, At :171-192, Extremum
 * :195-254, Integ :257-341), which follow ngspice's com_measure2.c. The
 * product never links this file. */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

/* scan.zig almostEqualUlps :49-59 (ngspice AlmostEqualUlps(a, b, 100)). */
static int ulps100(double a, double b) {
    if (a == b) return 1;
    int64_t ia, ib;
    memcpy(&ia, &a, 8);
    memcpy(&ib, &b, 8);
    if (ia < 0) ia = (int64_t)(0x8000000000000000ull - (uint64_t)ia);
    if (ib < 0) ib = (int64_t)(0x8000000000000000ull - (uint64_t)ib);
    uint64_t d = ia > ib ? (uint64_t)ia - (uint64_t)ib : (uint64_t)ib - (uint64_t)ia;
    return d <= 100;
}

/* scan.zig line :42-46. */
static double through(double x0, double y0, double x1, double y1, double x) {
    double slope = (y1 - y0) / (x1 - x0);
    double icept = y0 - slope * x0;
    return slope * x + icept;
}

void orc_meas_init(const espl_meas *c, orc_meas_state *s) {
    memset(s, 0, sizeof(*s));
    s->want_rise = c->rise;
    s->want_fall = c->fall;
    s->want_cross = c->cross;
    s->last = NAN;
    s->hit = NAN;
    s->value = NAN;
    s->first_x = NAN;
    s->cut_x = NAN;
}

/* Integ.panel :307-328: Simpson 3/8 over three equal spacings, Simpson over
 * two, else the trapezoid; points past `avail` read zero. */
static void panel(orc_meas_state *s, int avail) {
    double p[4][2];
    for (int k = 0; k < 4; k++) {
        p[k][0] = k < avail ? s->p[k][0] : 0.0;
        p[k][1] = k < avail ? s->p[k][1] : 0.0;
    }
    double w[3];
    for (int k = 0; k < 3; k++) w[k] = k + 1 < avail ? p[k + 1][0] - p[k][0] : 0.0;
    int used;
    if (ulps100(w[0], w[1]) && ulps100(w[0], w[2])) {
        s->sum[0] += 3 * w[0] * (p[0][1] + 3 * (p[1][1] + p[2][1]) + p[3][1]) / 8.0;
        used = 3;
    } else if (ulps100(w[0], w[1])) {
        s->sum[1] += w[0] * (p[0][1] + 4 * p[1][1] + p[2][1]) / 3.0;
        used = 2;
    } else {
        s->sum[2] += w[0] * (p[0][1] + p[1][1]) / 2;
        used = 1;
    }
    int keep = avail > used ? avail - used : 0;
    double q[4][2];
    memcpy(q, p, sizeof(q));
    for (int k = 0; k < keep; k++) {
        s->p[k][0] = q[avail - keep + k][0];
        s->p[k][1] = q[avail - keep + k][1];
    }
    s->np = keep;
}

void orc_meas_feed(const espl_meas *c, orc_meas_state *s, double x, double v) {
    if (s->done) return;
    switch (c->kind) {
    case ESPL_MEAS_WHEN: { /* Cross.feed, tran mode, one event */
        if (x < c->td) return;
        if (x < c->from) return;
        if (c->to != 0 && x > c->to) { s->done = 1; return; }
        double level = c->val;
        if (s->first == 1) {
            s->cross = 0;
            s->above = !(v < level);
            if (!s->above && s->prev >= level) { s->fall = 1; s->cross = 1; }
            else if (s->above && s->prev < level) { s->rise = 1; s->cross = 1; }
        }
        if (s->first > 1) {
            if (!s->above && v >= level) {
                s->above = 1; s->cross++; s->rise++;
                if (c->fall != ESPL_MEAS_LAST) s->pending = 1;
            } else if (s->above && v <= level) {
                s->above = 0; s->cross++; s->fall++;
                if (c->rise != ESPL_MEAS_LAST) s->pending = 1;
            }
            double hit = s->prev_x + (level - s->prev) * (x - s->prev_x) / (v - s->prev - level + level);
            if (s->cross == s->want_cross || s->rise == s->want_rise || s->fall == s->want_fall) {
                s->hit = hit; s->found = 1; s->done = 1; return;
            }
            if (s->pending) {
                if (c->cross == ESPL_MEAS_UNSET && c->rise == ESPL_MEAS_UNSET && c->fall == ESPL_MEAS_UNSET) {
                    s->hit = hit; s->found = 1; s->done = 1; return;
                }
                if (c->cross == ESPL_MEAS_LAST || c->rise == ESPL_MEAS_LAST || c->fall == ESPL_MEAS_LAST) s->last = hit;
                s->pending = 0;
            }
        }
        s->first++;
        s->prev = v;
        s->prev_x = x;
        return;
    }
    case ESPL_MEAS_FIND_AT: /* At.feed */
        if (s->rows > 0 && s->px <= c->at && x >= c->at) {
            s->value = s->pv + (c->at - s->px) * (v - s->pv) / (x - s->px);
            s->done = 1;
            return;
        }
        s->rows++;
        s->px = x;
        s->pv = v;
        return;
    case ESPL_MEAS_MIN:
    case ESPL_MEAS_MAX:
    case ESPL_MEAS_AVG: /* Extremum.feed */
        s->xv = x;
        if (x < c->from) return;
        if (c->to != 0 && x > c->to) { s->done = 1; return; }
        if (!s->first) {
            s->first = 1;
            s->m = c->kind == ESPL_MEAS_AVG ? 0.0 : v;
            s->m_at = x;
            s->pv = v;
            s->px = x;
            return;
        }
        if (c->kind == ESPL_MEAS_MIN) {
            if (v <= s->m) { s->m = v; s->m_at = x; }
        } else if (c->kind == ESPL_MEAS_MAX) {
            if (v >= s->m) { s->m = v; s->m_at = x; }
        } else {
            s->m += 0.5 * (v + s->pv) * (x - s->px);
            s->span += x - s->px;
            s->pv = v;
            s->px = x;
        }
        return;
    case ESPL_MEAS_INTEG:
    case ESPL_MEAS_RMS: { /* Integ.feed */
        double ox = s->px, oy = s->py;
        uint64_t orows = s->rows;
        s->rows++;
        s->px = x;
        s->py = v;
        if (!s->inside) {
            if (x < c->from) return;
            s->inside = 1;
        }
        s->cut = c->to != 0 && x > c->to;
        double ptx = x, pty = v;
        if (s->cut) {
            if (orows > 0 && !ulps100(x, c->to)) { ptx = c->to; pty = through(ox, oy, x, v, c->to); }
        } else if (s->count == 0 && c->from != 0 && orows > 0 && !ulps100(x, c->from)) {
            ptx = c->from;
            pty = through(ox, oy, x, v, c->from);
        }
        if (c->kind == ESPL_MEAS_RMS) pty = pty * pty;
        if (s->count == 0) s->first_x = ptx;
        if (s->cut) s->cut_x = ptx;
        s->count++;
        s->p[s->np][0] = ptx;
        s->p[s->np][1] = pty;
        s->np++;
        if (s->np == 4) panel(s, 4);
        if (s->cut) s->done = 1;
        return;
    }
    default:
        return;
    }
}

void orc_meas_result(const espl_meas *c, orc_meas_state *s, double *value, double *at) {
    *value = NAN;
    *at = NAN;
    switch (c->kind) {
    case ESPL_MEAS_WHEN: /* Cross.finish */
        *value = s->found ? s->hit : s->last;
        *at = *value;
        return;
    case ESPL_MEAS_FIND_AT:
        *value = s->value;
        *at = c->at;
        return;
    case ESPL_MEAS_MIN:
    case ESPL_MEAS_MAX: /* Extremum.stat */
        if (s->first) { *value = s->m; *at = s->m_at; }
        return;
    case ESPL_MEAS_AVG:
        *value = s->m / (s->first ? s->span : 1.0);
        *at = s->xv;
        return;
    case ESPL_MEAS_INTEG:
    case ESPL_MEAS_RMS: { /* Integ.result */
        if (s->rows == 0) return;
        while (s->np > 1) panel(s, s->np);
        double from = s->count > (uint64_t)(s->cut ? 1 : 0) ? s->first_x : NAN;
        double to = s->cut ? s->cut_x : s->px;
        double total = s->sum[0] + s->sum[1] + s->sum[2];
        *value = c->kind == ESPL_MEAS_RMS ? sqrt(total / (to - from)) : total;
        *at = to;
        return;
    }
    default:
        return;
    }
}

int orc_meas_series(const espl_meas *c, const double *x, const double *v, uint32_t n, double *value, double *at) {
    orc_meas_state s;
    orc_meas_init(c, &s);
    for (uint32_t k = 0; k < n; k++) orc_meas_feed(c, &s, x[k], v[k]);
    orc_meas_result(c, &s, value, at);
    return 0;
}
