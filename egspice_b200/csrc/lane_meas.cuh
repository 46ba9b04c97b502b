// Streaming .meas passes over a lane's transient, one sample (t, v) at a
// time: the event count of WHEN, the value at a point (FIND ... AT), the
// extremum and average (MIN, MAX, AVG) and the integral (INTEG, RMS), with
// ngspice's com_measure2.c semantics as the reference streams them on its
// lanes (src/output/scan.zig Cross, At, Extremum, Integ; run per lane in
// src/solver/lane_device.zig). A pass's state is kMeasWords doubles, word k
// of pass p of lane l at ((p * kMeasWords + k) * P + l); feeding stops once
// a pass reports the end of its window.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/espice_lanes.h"

namespace espl {

constexpr uint32_t kMeasWords = 24;
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

// WHEN state words.
enum : uint32_t {
    kWFirst = 1, kWAbove, kWPending, kWRise, kWFall, kWCross, kWWantRise, kWWantFall, kWWantCross, kWPrev,
    kWPrevX, kWFound, kWLast, kWHit
};
// FIND ... AT.
enum : uint32_t { kARows = 1, kAPx, kAPv, kAValue };
// MIN, MAX, AVG.
enum : uint32_t { kXFirst = 1, kXM, kXAt, kXLast, kXPv, kXPx, kXSpan };
// INTEG, RMS: up to four pending window points (scale, value) from word kIP.
enum : uint32_t { kIInside = 1, kIRows, kIPx, kIPy, kIP, kINp = kIP + 8, kICount, kIFirstX, kICut, kICutX, kISum };

// Fresh state of pass c.
__host__ __device__ inline void meas_init(const espl_meas& c, double* st, size_t stride) {
    for (uint32_t k = 0; k < kMeasWords; k++) MW(k) = 0.0;
    switch (c.kind) {
    case ESPL_MEAS_WHEN:
        MW(kWWantRise) = c.rise;
        MW(kWWantFall) = c.fall;
        MW(kWWantCross) = c.cross;
        MW(kWLast) = NAN;
        MW(kWHit) = NAN;
        break;
    case ESPL_MEAS_FIND_AT: MW(kAValue) = NAN; break;
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

// Feeds sample (x, v) to pass c unless it is done; marks it done where the
// whole-waveform scan would stop.
__host__ __device__ inline void meas_feed(const espl_meas& c, double* st, size_t stride, double x, double v) {
    if (MW(kMeasDone) != 0.0) return;
    bool stop = false;
    switch (c.kind) {
    case ESPL_MEAS_WHEN: {
        if (x < c.td || x < c.from) break;
        if (c.to != 0 && x > c.to) {
            stop = true;
            break;
        }
        const double level = c.val;
        const double first = MW(kWFirst);
        if (first == 1.0) {
            MW(kWCross) = 0;
            const bool above = !(v < level);
            MW(kWAbove) = above;
            if (!above && MW(kWPrev) >= level) {
                MW(kWFall) = 1;
                MW(kWCross) = 1;
            } else if (above && MW(kWPrev) < level) {
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
            const double hit = px + (level - pv) * (x - px) / (v - pv - level + level);
            if (MW(kWCross) == MW(kWWantCross) || MW(kWRise) == MW(kWWantRise) || MW(kWFall) == MW(kWWantFall)) {
                MW(kWHit) = hit;
                MW(kWFound) = 1;
                stop = true;
                break;
            }
            if (MW(kWPending) != 0.0) {
                if (c.cross == ESPL_MEAS_UNSET && c.rise == ESPL_MEAS_UNSET && c.fall == ESPL_MEAS_UNSET) {
                    MW(kWHit) = hit;
                    MW(kWFound) = 1;
                    stop = true;
                    break;
                }
                if (c.cross == ESPL_MEAS_LAST || c.rise == ESPL_MEAS_LAST || c.fall == ESPL_MEAS_LAST) MW(kWLast) = hit;
                MW(kWPending) = 0;
            }
        }
        MW(kWFirst) = first + 1;
        MW(kWPrev) = v;
        MW(kWPrevX) = x;
        break;
    }
    case ESPL_MEAS_FIND_AT: {
        const double px = MW(kAPx), pv = MW(kAPv);
        if (MW(kARows) > 0 && px <= c.at && x >= c.at) {
            MW(kAValue) = pv + (c.at - px) * (v - pv) / (x - px);
            stop = true;
            break;
        }
        MW(kARows) += 1;
        MW(kAPx) = x;
        MW(kAPv) = v;
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
// WHEN is its value; MIN/MAX: where; AVG: the last scale value read;
// INTEG/RMS: the window's end). Folds pending INTEG/RMS points on a copy.
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
        value = MW(kWFound) != 0.0 ? MW(kWHit) : MW(kWLast);
        at = value;
        break;
    case ESPL_MEAS_FIND_AT:
        value = MW(kAValue);
        at = c.at;
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
