/* Test infrastructure only (the oracle): the streaming .meas passes the
 * GPU lanes run, restated in plain C from the reference's sample-at-a-time
 * measures (src/output/scan.zig: Cross :61-169 with its level vector, At
 * :171-192 with its slope, Extremum :195-254, Integ :257-341, Find
 * :340-390), which follow ngspice's com_measure2.c, and the TARG stage of
 * src/output/measure.zig Stream.next :708-733 (a Cross with TD at the TRIG
 * event). The product never links this file. */
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
    s->t0 = NAN;
}

/* Cross.feed (scan.zig :88-160, tran mode, one event): returns 1 where the
 * pass stops. The level is c->val, or v2 with a level vector. */
static int cross_feed(const espl_meas *c, orc_meas_state *s, double td, double x, double v, double v2) {
    if (x < td) return 0;
    if (x < c->from) return 0;
    if (c->to != 0 && x > c->to) return 1;
    int two = c->level_row != 0;
    double level = two ? v2 : c->val;
    double prev_level = two ? s->prev2 : c->val;
    if (s->first == 1) {
        s->cross = 0;
        s->above = !(v < level);
        if (!s->above && s->prev >= prev_level) { s->fall = 1; s->cross = 1; }
        else if (s->above && s->prev < prev_level) { s->rise = 1; s->cross = 1; }
    }
    if (s->first > 1) {
        if (!s->above && v >= level) {
            s->above = 1; s->cross++; s->rise++;
            if (c->fall != ESPL_MEAS_LAST) s->pending = 1;
        } else if (s->above && v <= level) {
            s->above = 0; s->cross++; s->fall++;
            if (c->rise != ESPL_MEAS_LAST) s->pending = 1;
        }
        double hit = s->prev_x + (prev_level - s->prev) * (x - s->prev_x) / (v - s->prev - level + prev_level);
        if (s->cross == s->want_cross || s->rise == s->want_rise || s->fall == s->want_fall) {
            s->hit = hit; s->found = 1; return 1;
        }
        if (s->pending) {
            if (c->cross == ESPL_MEAS_UNSET && c->rise == ESPL_MEAS_UNSET && c->fall == ESPL_MEAS_UNSET) {
                s->hit = hit; s->found = 1; return 1;
            }
            if (c->cross == ESPL_MEAS_LAST || c->rise == ESPL_MEAS_LAST || c->fall == ESPL_MEAS_LAST) s->last = hit;
            s->pending = 0;
        }
    }
    s->first++;
    s->prev = v;
    if (two) s->prev2 = v2;
    s->prev_x = x;
    return 0;
}

/* Cross.finish (scan.zig :163-169) for one event: the count's, else LAST's. */
static double cross_event(const orc_meas_state *s) { return s->found ? s->hit : s->last; }

/* At.feed (scan.zig :182-192): 1 once the segment from the previous sample
 * holds `at`, with the value (or slope) there in s->value. */
static int at_feed(orc_meas_state *s, double at, int slope, double x, double v) {
    if (s->rows > 0 && s->px <= at && x >= at) {
        s->value = slope ? (v - s->pv) / (x - s->px) : s->pv + (at - s->px) * (v - s->pv) / (x - s->px);
        return 1;
    }
    s->rows++;
    s->px = x;
    s->pv = v;
    return 0;
}

/* Find.push (scan.zig :357-361) with the level value kept beside. */
static void ring_push(orc_meas_state *s, double x, double v, double v2) {
    if (s->ring_len == 3) memmove(s->ring[0], s->ring[1], sizeof(s->ring[0]) * 2);
    if (s->ring_len < 3) s->ring_len++;
    s->ring[s->ring_len - 1][0] = x;
    s->ring[s->ring_len - 1][1] = v;
    s->ring[s->ring_len - 1][2] = v2;
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

void orc_meas_feed(const espl_meas *c, orc_meas_state *s, const espl_meas *prev_c, const orc_meas_state *prev,
                   double x, double v, double v2) {
    (void)prev_c;
    if (s->done) return;
    switch (c->kind) {
    case ESPL_MEAS_WHEN:
        s->done = cross_feed(c, s, c->td, x, v, v2);
        return;
    case ESPL_MEAS_FIND_AT:
    case ESPL_MEAS_DERIV_AT: /* Dev.feed's .at: past `at` no later segment holds it */
        s->done = at_feed(s, c->at, c->kind == ESPL_MEAS_DERIV_AT, x, v) || x > c->at;
        return;
    case ESPL_MEAS_FIND_WHEN:
    case ESPL_MEAS_DERIV_WHEN: { /* Find.feed */
        int slope = c->kind == ESPL_MEAS_DERIV_WHEN;
        if (s->stage == 1) {
            s->done = at_feed(s, s->t0, slope, x, v) || x > s->t0;
            return;
        }
        ring_push(s, x, v, 0.0);
        s->kept_rows++;
        if (!prev || !prev->done) return;
        double t = cross_event(prev);
        if (isnan(t)) { s->stage = 2; s->done = 1; return; }
        s->stage = 1;
        s->t0 = t;
        if (s->kept_rows > (uint64_t)s->ring_len && t <= s->ring[0][0]) { s->done = 1; return; }
        for (int k = 0; k < s->ring_len; k++)
            if (at_feed(s, t, slope, s->ring[k][0], s->ring[k][1]) || s->ring[k][0] > t) { s->done = 1; return; }
        return;
    }
    case ESPL_MEAS_TARG: { /* Stream.next's TARG: a Cross from the TRIG event on */
        if (s->stage == 1) {
            s->done = cross_feed(c, s, s->t0, x, v, v2);
            return;
        }
        ring_push(s, x, v, v2);
        s->kept_rows++;
        if (!prev || !prev->done) return;
        double t = cross_event(prev);
        if (isnan(t)) { s->stage = 2; s->done = 1; return; }
        s->stage = 1;
        s->t0 = t;
        if (s->kept_rows > (uint64_t)s->ring_len && t < s->ring[0][0]) { s->done = 1; return; }
        for (int k = 0; k < s->ring_len; k++)
            if (cross_feed(c, s, t, s->ring[k][0], s->ring[k][1], s->ring[k][2])) { s->done = 1; return; }
        return;
    }
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
        *value = cross_event(s);
        *at = *value;
        return;
    case ESPL_MEAS_TARG:
        *at = cross_event(s);
        *value = *at - s->t0;
        return;
    case ESPL_MEAS_FIND_AT:
    case ESPL_MEAS_DERIV_AT:
        *value = s->value;
        *at = c->at;
        return;
    case ESPL_MEAS_FIND_WHEN:
    case ESPL_MEAS_DERIV_WHEN:
        *value = s->value;
        *at = s->t0;
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
    espl_meas one = *c;
    one.row = 0;
    one.level_row = 0;
    return orc_meas_table(&one, 1, x, v, 1, n, value, at);
}

int orc_meas_table(const espl_meas *passes, uint32_t n_passes, const double *x, const double *cols, uint32_t n_cols,
                   uint32_t n, double *value, double *at) {
    if (n_passes > ESPL_MEAS_MAX_PASSES) return 1;
    orc_meas_state s[ESPL_MEAS_MAX_PASSES];
    for (uint32_t p = 0; p < n_passes; p++) {
        if (passes[p].row >= n_cols || passes[p].level_row > n_cols) return 1;
        orc_meas_init(&passes[p], &s[p]);
    }
    for (uint32_t k = 0; k < n; k++)
        for (uint32_t p = 0; p < n_passes; p++) {
            const espl_meas *c = &passes[p];
            const double *row = cols + (size_t)k * n_cols;
            orc_meas_feed(c, &s[p], p ? &passes[p - 1] : NULL, p ? &s[p - 1] : NULL, x[k], row[c->row],
                          c->level_row ? row[c->level_row - 1] : 0.0);
        }
    for (uint32_t p = 0; p < n_passes; p++) orc_meas_result(&passes[p], &s[p], &value[p], &at[p]);
    return 0;
}
