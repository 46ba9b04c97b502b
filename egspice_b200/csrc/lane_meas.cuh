// Streaming .meas passes over a lane's transient, one sample (t, v) at a
// time: the event count of WHEN (against a constant or a second vector),
// the value or slope at a point (FIND/DERIV ... AT), the value or slope at
// the previous pass's WHEN event (FIND/DERIV ... WHEN), a TARG event counted
// from the previous pass's TRIG event, the extremum and average (MIN, MAX,
// AVG) and the integral (INTEG, RMS), with ngspice's com_measure2.c
// semantics as the reference streams them on its lanes (src/output/scan.zig
// Cross :60-169, At :171-192, Extremum, Integ, Find :340-390; run per lane in
// src/solver/lane_device.zig). A pass's state is kMeasWords doubles, word k
// of pass p of lane l at ((p * kMeasWords + k) * P + l); feeding stops once
// a pass reports the end of its window. Passes are fed in order, so a pass
// that reads the one before it sees that pass after the same sample.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/espice_lanes.h"

namespace espl {

constexpr uint32_t kMeasWords = 32;
constexpr uint32_t kMeasDone = 0;  // the pass read its last sample

#define MW(k) st[(size_t)(k) * stride]

// ngspice AlmostEqualUlps(a, b, 100): within 100 units in the last place.
__host__ __device__ inline bool meas_almost_equal(double a, double b) {
    if (a == b) return true;
    auto ord = [](double d) {
        int64_t i;
        memcpy(&i, &d, 8);
        return i < 0 ? (int64_t)(0x8000000000000000ull - (uint64_t)i) : i;
    };
    const int64_t da = ord(a), db = ord(b);
    const uint64_t diff = da > db ? (uint64_t)da - (uint64_t)db : (uint64_t)db - (uint64_t)da;
    return diff <= 100;
}

// The line through (x0, y0) and (x1, y1) at x, slope-intercept form.
__host__ __device__ inline double meas_line(double x0, double y0, double x1, double y1, double x) {
    const double slope = (y1 - y0) / (x1 - x0);
    const double icept = y0 - slope * x0;
    return slope * x + icept;
}

// WHEN state words (also the TARG pass's event count).
enum : uint32_t {
    kWFirst = 1, kWAbove, kWPending, kWRise, kWFall, kWCross, kWWantRise, kWWantFall, kWWantCross, kWPrev,
    kWPrevX, kWFound, kWLast, kWHit, kWPrev2
};
// FIND/DERIV ... AT, and the value pass of FIND/DERIV ... WHEN.
enum : uint32_t { kARows = 1, kAPx, kAPv, kAValue };
// FIND/DERIV ... WHEN: the event time once armed, the stage (kMeas*), rows
// read, and the last rows (scale, value, level) oldest first.
enum : uint32_t { kFAt = 5, kFStage, kFRows, kFRingLen, kFRing };
// TARG: the TRIG event time, the stage, rows read and the ring after the
// event count's words.
enum : uint32_t { kTTrig = 16, kTStage, kTRows, kTRingLen, kTRing };
enum : uint32_t { kMeasWaiting = 0, kMeasArmed = 1, kMeasNoEvent = 2 };
constexpr uint32_t kMeasRing = 3;
static_assert(kTRing + 3 * kMeasRing <= kMeasWords, "the TARG state fits a pass");

__host__ __device__ constexpr bool meas_reads_previous(uint32_t kind) {
    return kind == ESPL_MEAS_FIND_WHEN || kind == ESPL_MEAS_DERIV_WHEN || kind == ESPL_MEAS_TARG;
}
// MIN, MAX, AVG.
enum : uint32_t { kXFirst = 1, kXM, kXAt, kXLast, kXPv, kXPx, kXSpan };
// INTEG, RMS: up to four pending window points (scale, value) from word kIP.
enum : uint32_t { kIInside = 1, kIRows, kIPx, kIPy, kIP, kINp = kIP + 8, kICount, kIFirstX, kICut, kICutX, kISum };

// Fresh state of pass c.
__host__ __device__ inline void meas_init(const espl_meas& c, double* st, size_t stride) {
    for (uint32_t k = 0; k < kMeasWords; k++) MW(k) = 0.0;
    switch (c.kind) {
    case ESPL_MEAS_WHEN:
    case ESPL_MEAS_TARG:
        MW(kWWantRise) = c.rise;
        MW(kWWantFall) = c.fall;
        MW(kWWantCross) = c.cross;
        MW(kWLast) = NAN;
        MW(kWHit) = NAN;
        MW(kTTrig) = c.kind == ESPL_MEAS_TARG ? NAN : 0.0;
        break;
    case ESPL_MEAS_FIND_AT:
    case ESPL_MEAS_DERIV_AT: MW(kAValue) = NAN; break;
    case ESPL_MEAS_FIND_WHEN:
    case ESPL_MEAS_DERIV_WHEN:
        MW(kAValue) = NAN;
        MW(kFAt) = NAN;
        break;
    case ESPL_MEAS_INTEG:
    case ESPL_MEAS_RMS:
        MW(kIFirstX) = NAN;
        MW(kICutX) = NAN;
        break;
    default: break;
    }
}

// Folds the oldest `avail` pending window points into one panel: Simpson's
// 3/8 rule over three equal spacings, Simpson's rule over two, else the
// trapezoid; points past `avail` read zero.
__host__ __device__ inline void meas_panel(double* st, size_t stride, uint32_t avail) {
    double p[4][2];
    for (uint32_t j = 0; j < 4; j++) {
        p[j][0] = j < avail ? MW(kIP + 2 * j) : 0.0;
        p[j][1] = j < avail ? MW(kIP + 2 * j + 1) : 0.0;
    }
    double w[3];
    for (uint32_t j = 0; j < 3; j++) w[j] = j + 1 < avail ? p[j + 1][0] - p[j][0] : 0.0;
    uint32_t used;
    if (meas_almost_equal(w[0], w[1]) && meas_almost_equal(w[0], w[2])) {
        MW(kISum) += 3 * w[0] * (p[0][1] + 3 * (p[1][1] + p[2][1]) + p[3][1]) / 8.0;
        used = 3;
    } else if (meas_almost_equal(w[0], w[1])) {
        MW(kISum + 1) += w[0] * (p[0][1] + 4 * p[1][1] + p[2][1]) / 3.0;
        used = 2;
    } else {
        MW(kISum + 2) += w[0] * (p[0][1] + p[1][1]) / 2;
        used = 1;
    }
    const uint32_t keep = avail > used ? avail - used : 0u;
    for (uint32_t j = 0; j < keep; j++) {
        MW(kIP + 2 * j) = p[avail - keep + j][0];
        MW(kIP + 2 * j + 1) = p[avail - keep + j][1];
    }
    MW(kINp) = keep;
}

__host__ __device__ inline bool meas_nan(double v) { return v != v; }

// Cross.feed (scan.zig :88-160) on the event-count words 1..15 of `st`:
// samples before `td` or `from` are skipped, the first past a nonzero `to`
// ends the pass (true), as does the event the counts ask for. The level is
// `val`, or the second vector's value `v2` when the pass names one.
__host__ __device__ inline bool meas_cross(const espl_meas& c, double* st, size_t stride, double td, double x,
                                           double v, double v2) {
    if (x < td || x < c.from) return false;
    if (c.to != 0 && x > c.to) return true;
    const bool two = c.level_row != 0;
    const double level = two ? v2 : c.val;
    const double prev_level = two ? MW(kWPrev2) : c.val;
    const double first = MW(kWFirst);
    if (first == 1.0) {
        MW(kWCross) = 0;
        const bool above = !(v < level);
        MW(kWAbove) = above;
        if (!above && MW(kWPrev) >= prev_level) {
            MW(kWFall) = 1;
            MW(kWCross) = 1;
        } else if (above && MW(kWPrev) < prev_level) {
            MW(kWRise) = 1;
            MW(kWCross) = 1;
        }
    }
    if (first > 1.0) {
        if (MW(kWAbove) == 0.0 && v >= level) {
            MW(kWAbove) = 1;
            MW(kWCross) += 1;
            MW(kWRise) += 1;
            if (c.fall != ESPL_MEAS_LAST) MW(kWPending) = 1;
        } else if (MW(kWAbove) != 0.0 && v <= level) {
            MW(kWAbove) = 0;
            MW(kWCross) += 1;
            MW(kWFall) += 1;
            if (c.rise != ESPL_MEAS_LAST) MW(kWPending) = 1;
        }
        const double px = MW(kWPrevX), pv = MW(kWPrev);
        const double hit = px + (prev_level - pv) * (x - px) / (v - pv - level + prev_level);
        if (MW(kWCross) == MW(kWWantCross) || MW(kWRise) == MW(kWWantRise) || MW(kWFall) == MW(kWWantFall)) {
            MW(kWHit) = hit;
            MW(kWFound) = 1;
            return true;
        }
        if (MW(kWPending) != 0.0) {
            if (c.cross == ESPL_MEAS_UNSET && c.rise == ESPL_MEAS_UNSET && c.fall == ESPL_MEAS_UNSET) {
                MW(kWHit) = hit;
                MW(kWFound) = 1;
                return true;
            }
            if (c.cross == ESPL_MEAS_LAST || c.rise == ESPL_MEAS_LAST || c.fall == ESPL_MEAS_LAST) MW(kWLast) = hit;
            MW(kWPending) = 0;
        }
    }
    MW(kWFirst) = first + 1;
    MW(kWPrev) = v;
    if (two) MW(kWPrev2) = v2;
    MW(kWPrevX) = x;
    return false;
}

// The event time of a WHEN pass's state (Cross.finish :163-169): the one its
// count asked for, else the last one (LAST), else NaN.
__host__ __device__ inline double meas_event(const double* st, size_t stride) {
    return MW(kWFound) != 0.0 ? MW(kWHit) : MW(kWLast);
}

// At.feed (scan.zig :182-192) on words kARows..kAValue: true once the
// segment from the previous sample holds `at`, with the value there (linear)
// or the segment's slope.
__host__ __device__ inline bool meas_at(double* st, size_t stride, double at, bool slope, double x, double v) {
    const double px = MW(kAPx), pv = MW(kAPv);
    if (MW(kARows) > 0 && px <= at && x >= at) {
        MW(kAValue) = slope ? (v - pv) / (x - px) : pv + (at - px) * (v - pv) / (x - px);
        return true;
    }
    MW(kARows) += 1;
    MW(kAPx) = x;
    MW(kAPv) = v;
    return false;
}

// Find.push (scan.zig :357-361): appends (x, v, v2) to the ring of the last
// kMeasRing samples at word `ring`, length at word `len_word`.
__host__ __device__ inline void meas_push(double* st, size_t stride, uint32_t ring, uint32_t len_word, double x,
                                          double v, double v2) {
    uint32_t len = (uint32_t)MW(len_word);
    if (len == kMeasRing)
        for (uint32_t k = 0; k < 3 * (kMeasRing - 1); k++) MW(ring + k) = MW(ring + 3 + k);
    len = len < kMeasRing ? len + 1 : kMeasRing;
    MW(len_word) = len;
    MW(ring + 3 * (len - 1)) = x;
    MW(ring + 3 * (len - 1) + 1) = v;
    MW(ring + 3 * (len - 1) + 2) = v2;
}

// Feeds sample (x, v) to pass c unless it is done, v2 being the value of
// the pass's level vector (unused without one) and `prev` the state of the
// pass before it (FIND/DERIV WHEN and TARG read it; nullptr for pass 0);
// marks the pass done where the whole-waveform scan would stop.
__host__ __device__ inline void meas_feed(const espl_meas& c, double* st, size_t stride, const double* prev,
                                          double x, double v, double v2) {
    if (MW(kMeasDone) != 0.0) return;
    bool stop = false;
    switch (c.kind) {
    case ESPL_MEAS_WHEN: stop = meas_cross(c, st, stride, c.td, x, v, v2); break;
    case ESPL_MEAS_FIND_AT:
    case ESPL_MEAS_DERIV_AT:
        // a transient's times rise: past `at`, no later segment holds it
        stop = meas_at(st, stride, c.at, c.kind == ESPL_MEAS_DERIV_AT, x, v) || x > c.at;
        break;
    case ESPL_MEAS_FIND_WHEN:
    case ESPL_MEAS_DERIV_WHEN: {
        // Find.feed (scan.zig :365-388): the last rows are kept until the
        // WHEN pass ends; at its event this becomes the At there, fed those
        // rows first.
        const bool slope = c.kind == ESPL_MEAS_DERIV_WHEN;
        if (MW(kFStage) == kMeasArmed) {
            stop = meas_at(st, stride, MW(kFAt), slope, x, v) || x > MW(kFAt);
            break;
        }
        meas_push(st, stride, kFRing, kFRingLen, x, v, 0.0);
        MW(kFRows) += 1;
        if (!prev || prev[(size_t)kMeasDone * stride] == 0.0) break;
        const double t = meas_event(prev, stride);
        if (meas_nan(t)) {
            MW(kFStage) = kMeasNoEvent;
            stop = true;
            break;
        }
        MW(kFStage) = kMeasArmed;
        MW(kFAt) = t;
        const uint32_t len = (uint32_t)MW(kFRingLen);
        if (MW(kFRows) > len && t <= MW(kFRing)) {
            stop = true;
            break;
        }
        for (uint32_t j = 0; j < len && !stop; j++) {
            const double rx = MW(kFRing + 3 * j), rv = MW(kFRing + 3 * j + 1);
            stop = meas_at(st, stride, t, slope, rx, rv) || rx > t;
        }
        break;
    }
    case ESPL_MEAS_TARG: {
        // TARG's event count with TD = the TRIG pass's event (the reference
        // replays its recording from there, measure.zig Stream.next): the
        // last rows are kept until the TRIG pass ends, then fed first. A
        // TRIG event before the oldest kept row, with rows before it, leaves
        // TARG unresolved.
        if (MW(kTStage) == kMeasArmed) {
            stop = meas_cross(c, st, stride, MW(kTTrig), x, v, v2);
            break;
        }
        meas_push(st, stride, kTRing, kTRingLen, x, v, v2);
        MW(kTRows) += 1;
        if (!prev || prev[(size_t)kMeasDone * stride] == 0.0) break;
        const double t = meas_event(prev, stride);
        if (meas_nan(t)) {
            MW(kTStage) = kMeasNoEvent;
            stop = true;
            break;
        }
        MW(kTStage) = kMeasArmed;
        MW(kTTrig) = t;
        const uint32_t len = (uint32_t)MW(kTRingLen);
        if (MW(kTRows) > len && t < MW(kTRing)) {
            stop = true;
            break;
        }
        for (uint32_t j = 0; j < len && !stop; j++)
            stop = meas_cross(c, st, stride, t, MW(kTRing + 3 * j), MW(kTRing + 3 * j + 1), MW(kTRing + 3 * j + 2));
        break;
    }
    case ESPL_MEAS_MIN:
    case ESPL_MEAS_MAX:
    case ESPL_MEAS_AVG: {
        MW(kXLast) = x;
        if (x < c.from) break;
        if (c.to != 0 && x > c.to) {
            stop = true;
            break;
        }
        if (MW(kXFirst) == 0.0) {
            MW(kXFirst) = 1;
            MW(kXM) = c.kind == ESPL_MEAS_AVG ? 0.0 : v;
            MW(kXAt) = x;
            MW(kXPv) = v;
            MW(kXPx) = x;
            break;
        }
        if (c.kind == ESPL_MEAS_MIN) {
            if (v <= MW(kXM)) {
                MW(kXM) = v;
                MW(kXAt) = x;
            }
        } else if (c.kind == ESPL_MEAS_MAX) {
            if (v >= MW(kXM)) {
                MW(kXM) = v;
                MW(kXAt) = x;
            }
        } else {
            MW(kXM) += 0.5 * (v + MW(kXPv)) * (x - MW(kXPx));
            MW(kXSpan) += x - MW(kXPx);
            MW(kXPv) = v;
            MW(kXPx) = x;
        }
        break;
    }
    case ESPL_MEAS_INTEG:
    case ESPL_MEAS_RMS: {
        const double px = MW(kIPx), py = MW(kIPy), rows = MW(kIRows);
        MW(kIRows) = rows + 1;
        MW(kIPx) = x;
        MW(kIPy) = v;
        if (MW(kIInside) == 0.0) {
            if (x < c.from) break;
            MW(kIInside) = 1;
        }
        const bool cut = c.to != 0 && x > c.to;
        MW(kICut) = cut;
        double ptx = x, pty = v;
        if (cut) {
            if (rows > 0 && !meas_almost_equal(x, c.to)) {
                ptx = c.to;
                pty = meas_line(px, py, x, v, c.to);
            }
        } else if (MW(kICount) == 0 && c.from != 0 && rows > 0 && !meas_almost_equal(x, c.from)) {
            ptx = c.from;
            pty = meas_line(px, py, x, v, c.from);
        }
        if (c.kind == ESPL_MEAS_RMS) pty = pty * pty;
        if (MW(kICount) == 0) MW(kIFirstX) = ptx;
        if (cut) MW(kICutX) = ptx;
        MW(kICount) += 1;
        const uint32_t np = (uint32_t)MW(kINp);
        MW(kIP + 2 * np) = ptx;
        MW(kIP + 2 * np + 1) = pty;
        MW(kINp) = np + 1;
        if (np + 1 == 4) meas_panel(st, stride, 4);
        stop = cut;
        break;
    }
    default: break;
    }
    if (stop) MW(kMeasDone) = 1;
}

// The result of pass c from its state: `value`, and `at` (the event time of
// WHEN is its value; FIND/DERIV AT: `at`; FIND/DERIV WHEN: the event time;
// TARG: the TARG event, its value the time from the TRIG event; MIN/MAX:
// where; AVG: the last scale value read; INTEG/RMS: the window's end). Folds
// pending INTEG/RMS points on a copy.
__host__ inline void meas_result(const espl_meas& c, const double* st_in, size_t stride, double& value, double& at) {
    double st_copy[kMeasWords];
    for (uint32_t k = 0; k < kMeasWords; k++) st_copy[k] = st_in[(size_t)k * stride];
    double* st = st_copy;
    stride = 1;
    const double nan = NAN;
    value = nan;
    at = nan;
    switch (c.kind) {
    case ESPL_MEAS_WHEN:
        value = meas_event(st, 1);
        at = value;
        break;
    case ESPL_MEAS_TARG:
        at = meas_event(st, 1);
        value = at - MW(kTTrig);
        break;
    case ESPL_MEAS_FIND_AT:
    case ESPL_MEAS_DERIV_AT:
        value = MW(kAValue);
        at = c.at;
        break;
    case ESPL_MEAS_FIND_WHEN:
    case ESPL_MEAS_DERIV_WHEN:
        value = MW(kAValue);
        at = MW(kFAt);
        break;
    case ESPL_MEAS_MIN:
    case ESPL_MEAS_MAX:
        if (MW(kXFirst) != 0.0) {
            value = MW(kXM);
            at = MW(kXAt);
        }
        break;
    case ESPL_MEAS_AVG:
        value = MW(kXM) / (MW(kXFirst) != 0.0 ? MW(kXSpan) : 1.0);
        at = MW(kXLast);
        break;
    case ESPL_MEAS_INTEG:
    case ESPL_MEAS_RMS: {
        if (MW(kIRows) == 0) break;
        while (MW(kINp) > 1) meas_panel(st, 1, (uint32_t)MW(kINp));
        const bool cut = MW(kICut) != 0.0;
        const double from = MW(kICount) > (cut ? 1.0 : 0.0) ? MW(kIFirstX) : nan;
        const double to = cut ? MW(kICutX) : MW(kIPx);
        const double total = MW(kISum) + MW(kISum + 1) + MW(kISum + 2);
        value = c.kind == ESPL_MEAS_RMS ? sqrt(total / (to - from)) : total;
        at = to;
        break;
    }
    default: break;
    }
}

#undef MW

}  // namespace espl
