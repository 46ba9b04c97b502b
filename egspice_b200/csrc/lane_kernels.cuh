// Kernels of the lane sweep: one thread per lane, the whole Newton solve of
// an operating point, or up to `launch_steps` transient steps with device
// step control, in one launch. A warp holds 32 lanes of one template; the
// warp -> template table lets one launch carry templates of different sizes.
#pragma once

#include "lane_engine.cuh"

namespace espl {

// plausibleLimit (kernels/lane.zig:202-214): the runaway bound of a solve,
// read off its first assembly.
__device__ double plausible_limit(const GroupDev& d, uint32_t l) {
    const uint32_t P = d.P;
    double g = 1.0;
    for (uint32_t i = 0; i < d.n; i++) g = fmax(g, fabs(LM(d.a, d.diag[i])));
    uint64_t xm = 0, fm = 0;
    for (uint32_t i = 0; i < d.n; i++) {
        uint64_t xb = dbits(fabs(LM(d.x, i))), fb = dbits(fabs(LM(d.rhs, i)));
        xm = xm > xb ? xm : xb;
        fm = fm > fb ? fm : fb;
    }
    double scale = fmin(fmax(bitsd(xm), bitsd(fm) * g), 1e18);
    if (isnan(bitsd(xm)) || isnan(bitsd(fm))) scale = NAN;
    return !(1e3 * scale > kXPlausible) ? kXPlausible : 1e3 * scale;
}

// updateNorm (kernels/lane.zig:161-179): x_old = x, x += dx, the delta score.
__device__ double update_norm(const GroupDev& d, uint32_t l, double reltol, double abstol, double vntol) {
    const uint32_t P = d.P;
    uint64_t worst = 0;
    for (uint32_t i = 0; i < d.n; i++) {
        double xo = LM(d.x, i), dd = LM(d.dx, i);
        double xn = xo + dd;
        LM(d.x_old, i) = xo;
        LM(d.x, i) = xn;
        double tol = reltol * fmax(fabs(xn), fabs(xo)) + (d.cur_row[i] ? abstol : vntol);
        bool finite = fabs(xn) < INFINITY && fabs(dd) < INFINITY;
        double q = fabs(dd) / tol;
        double score = !finite ? INFINITY : (q == q ? q : 0.0);
        uint64_t b = dbits(score);
        worst = worst > b ? worst : b;
    }
    return bitsd(worst);
}

__device__ bool residual_ok(const GroupDev& d, uint32_t l, const NewtonParams& o) {
    const uint32_t P = d.P;
    for (uint32_t i = 0; i < d.n; i++) {
        double scale = fabs(LM(d.a, d.diag[i]));
        double s = scale == 0.0 ? 1.0 : scale;
        double tol = fmax(o.residual_tol, 10.0 * s * (o.reltol * fabs(LM(d.x, i)) + o.vntol));
        if (!(fabs(LM(d.rhs, i)) <= tol)) return false;
    }
    return true;
}

// A failed replay of a lane with n <= 64 solves densely in a pool slot
// (the place of arp_lane_peel_dense, lane_device.zig:120-147), re-pivoting
// as the host factor would. False when the pool is spent or the factor
// fails.
__device__ bool peel_dense(const GroupDev& d, uint32_t l, LaneState& s, const PeelPool& pool) {
    const uint32_t P = d.P;
    if (d.n > kDensePeelMax || pool.scratch == nullptr) return false;
    if (s.peel_slot == 0xFFFFFFFFu) {
        uint32_t slot = atomicAdd(pool.next, 1u);
        if (slot >= pool.n_slots) {
            atomicAdd(pool.over, 1u);
            return false;
        }
        s.peel_slot = slot;
    }
    double* m = pool.scratch + (size_t)s.peel_slot * pool.slot_words;
    double* xv = m + (size_t)d.n * d.n;
    uint32_t n = d.n;
    for (uint32_t i = 0; i < n * n; i++) m[i] = 0.0;
    for (uint32_t c = 0; c < n; c++)
        for (uint32_t p = d.col_ptr[c]; p < d.col_ptr[c + 1]; p++) m[d.row_idx[p] * n + c] += LM(d.a, p);
    for (uint32_t i = 0; i < n; i++) xv[i] = LM(d.rhs, i);
    if (!dense_repivot_neg(n, d.q, m, xv)) return false;
    for (uint32_t i = 0; i < n; i++) LM(d.dx, i) = xv[i];
    return true;
}

// One lane's Newton (converger.newtonLanes at W = 1 as the lane kernels
// split it: assemble, gmin, refactor, solve, update, limit, gates, finalize).
template <bool MIXED>
__device__ void newton_lane(const GroupDev& d, uint32_t l, LaneState& s, const NewtonParams& o, int tran, double t,
                            const Companion& cp, const PeelPool& pool) {
    const uint32_t P = d.P;
    uint32_t bits = kActive | (o.init_fix ? kInitFix : 0u);
    double limit = kXPlausible;
    s.iterations = o.max_iter;
    for (uint32_t it = 0; it < o.max_iter; it++) {
        eval_lane(d, l, tran, t);
        if (cp.on) {
            for (uint32_t i = 0; i < d.n; i++) {
                double dq = cp.ag0 * (LM(d.qrow, i) - LM(d.q1, i));
                double base = LM(d.rhs, i) + dq;
                LM(d.rhs, i) = cp.method == 1 ? base - cp.ag1 * LM(d.ip, i) : base;
            }
            for (uint32_t p = 0; p < d.nnz; p++) LM(d.a, p) = LM(d.g, p) + cp.ag0 * LM(d.c, p);
        } else {
            for (uint32_t p = 0; p < d.nnz; p++) LM(d.a, p) = LM(d.g, p);
        }
        if (o.gmin > 0.0) {
            for (uint32_t i = 0; i < d.n; i++) LM(d.a, d.diag[i]) += o.gmin;
            for (uint32_t i = 0; i < d.n; i++) LM(d.rhs, i) += o.gmin * LM(d.x, i);
        }
        if (it == 0) limit = plausible_limit(d, l);
        bool fail;
        bool use32 = MIXED && !s.fp64;
        if (use32 && refactor32(d, l)) {
            s.fp64 = 1;
            s.fallbacks++;
            use32 = false;
        }
        if (use32) {
            fail = false;
        } else {
            int rc = refactor64(d, l);
            fail = rc == 1 || (rc == 2 && !replay_holds64(d, l));
        }
        if (fail) {
            if (!peel_dense(d, l, s, pool)) {
                bits = (bits | kSingular) & ~kActive;
                s.iterations = it;
                break;
            }
        } else if (use32) {
            solve32(d, l, d.rhs, d.dx);
            for (uint32_t r = 0; r < o.refine; r++) refine_mixed(d, l);
        } else {
            solve64(d, l, d.rhs, d.dx);
        }
        double scaled = update_norm(d, l, o.reltol, o.abstol, o.vntol);
        bool limited = limit_lane(d, l);
        bool ok = !limited && it != 0 && !(scaled >= 1.0);
        if (ok)
            for (uint32_t i = 0; i < d.n; i++)
                if (!(fabs(LM(d.x, i)) <= limit)) { ok = false; break; }
        if (ok) ok = residual_ok(d, l, o);
        if (ok && (bits & kInitFix)) {
            bits &= ~kInitFix;
        } else if (ok) {
            for (uint32_t i = 0; i < d.n; i++) LM(d.x, i) = LM(d.x_old, i);
            bits = (bits | kConverged) & ~kActive;
            s.iterations = it + 1;
            break;
        }
        if (MIXED && !s.fp64 && it + 1 >= o.stall_ticks) {
            s.fp64 = 1;
            s.fallbacks++;
        }
    }
    s.bits = bits & ~kActive;
}

struct LaunchMap {
    const GroupDev* groups;
    const uint32_t* warp_group;
    uint32_t n_warps;
};

__device__ __forceinline__ bool lane_of(const LaunchMap& m, const GroupDev*& d, uint32_t& l) {
    uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw >= m.n_warps) return false;
    d = &m.groups[m.warp_group[gw]];
    l = ((gw - d->warp0) << 5) | (threadIdx.x & 31);
    return l < d->lanes;
}

template <bool MIXED>
__global__ void __launch_bounds__(128) k_static(LaunchMap m, NewtonParams o, LaneState* st, int tran, PeelPool pool) {
    const GroupDev* d;
    uint32_t l;
    if (!lane_of(m, d, l)) return;
    LaneState& s = st[d->lane0 + l];
    s.peel_slot = 0xFFFFFFFFu;  // the pool's counter restarts every solve
    Companion cp{0, 0, 0.0, 0.0};
    newton_lane<MIXED>(*d, l, s, o, tran, 0.0, cp, pool);
}

// Bias-independent prep per (instance, lane), from the raw lane-major rows.
__global__ void __launch_bounds__(128) k_prep(LaunchMap m, const double* const* mos_raw, const double* const* dio_raw) {
    const GroupDev* d;
    uint32_t l;
    if (!lane_of(m, d, l)) return;
    const uint32_t P = d->P;
    uint32_t g = m.warp_group[(blockIdx.x * blockDim.x + threadIdx.x) >> 5];
    const double* mr = mos_raw[g];
    const double* dr = dio_raw[g];
    double* md = const_cast<double*>(d->mos_d);
    double* dd = const_cast<double*>(d->dio_d);
    for (uint32_t i = 0; i < d->n_mos; i++) {
        double p[9], o[Mos1Prep::count];
        for (int k = 0; k < 9; k++) p[k] = LM(mr, 9 * i + k);
        mos1_setup(p, o);
        for (int k = 0; k < Mos1Prep::count; k++) LM(md, Mos1Prep::count * i + k) = o[k];
    }
    for (uint32_t i = 0; i < d->n_dio; i++) {
        double p[7], o[DiodePrep::count];
        for (int k = 0; k < 7; k++) p[k] = LM(dr, 7 * i + k);
        diode_setup(p, o);
        for (int k = 0; k < DiodePrep::count; k++) LM(dd, DiodePrep::count * i + k) = o[k];
    }
}

// Seeds the limiter states for a cold (MODEINITJCT) or warm start.
__global__ void __launch_bounds__(128) k_seed(LaunchMap m, int cold, LaneState* st) {
    const GroupDev* d;
    uint32_t l;
    if (!lane_of(m, d, l)) return;
    seed_limits(*d, l, cold, d->x);
    LaneState& s = st[d->lane0 + l];
    s.fp64 = 0;
    s.fallbacks = 0;
    s.peel_slot = 0xFFFFFFFFu;
}

// Stamps every lane at its x and writes A = G (+ C / dt) for the lead
// lane's tape (ownTape's matrix).
__global__ void __launch_bounds__(128) k_assemble(LaunchMap m, int tran, double t, double inv_dt) {
    const GroupDev* d;
    uint32_t l;
    if (!lane_of(m, d, l)) return;
    const uint32_t P = d->P;
    eval_lane(*d, l, tran, t);
    for (uint32_t p = 0; p < d->nnz; p++)
        LM(d->a, p) = inv_dt > 0.0 ? LM(d->g, p) + inv_dt * LM(d->c, p) : LM(d->g, p);
}

// ---------------------------------------------------------------------------
// Transient

__device__ __forceinline__ bool at_stop(double t, double t_stop) {
    if (t == t_stop) return true;
    if ((t < 0) != (t_stop < 0)) return false;
    long long a = __double_as_longlong(t), b = __double_as_longlong(t_stop);
    long long dd = a - b;
    return (dd < 0 ? -dd : dd) <= 100;
}

__device__ __forceinline__ bool almost_equal_ulps(double a, double b, long long max_ulps) {
    if (a == b) return true;
    long long ia = __double_as_longlong(a), ib = __double_as_longlong(b);
    // lex order of IEEE bits as tran.almostEqualUlps defines it, in 128 bits.
    __int128 la = ia < 0 ? (__int128)LLONG_MIN - ia : ia;
    __int128 lb = ib < 0 ? (__int128)LLONG_MIN - ib : ib;
    __int128 dd = la - lb;
    if (dd < 0) dd = -dd;
    return dd <= max_ulps;
}

__device__ double next_bp(const GroupDev& d, uint32_t l, double t) {
    const uint32_t P = d.P;
    double best = INFINITY;
    for (uint32_t i = 0; i < d.n_vsrc; i++) {
        const double* pp = d.vsrc_p;
        uint32_t b9 = 9 * i;
        best = fmin(best, source_next_bp(LM(pp, b9 + 1), LM(pp, b9 + 4), LM(pp, b9 + 5), LM(pp, b9 + 6),
                                         LM(pp, b9 + 7), LM(pp, b9 + 8), t));
    }
    for (uint32_t i = 0; i < d.n_isrc; i++) {
        const double* pp = d.isrc_p;
        uint32_t b9 = 9 * i;
        best = fmin(best, source_next_bp(LM(pp, b9 + 1), LM(pp, b9 + 4), LM(pp, b9 + 5), LM(pp, b9 + 6),
                                         LM(pp, b9 + 7), LM(pp, b9 + 8), t));
    }
    return best;
}

// stepBound (kernels/lane.zig:257-297) over the lane's sites; ring slots
// are the logical 0..3 of the site ring.
__device__ double step_bound(const GroupDev& d, uint32_t l, uint32_t rot, uint32_t method, uint32_t cur_method,
                             double dt, double dt1, double dt2, double reltol, double abstol, double chgtol,
                             double trtol, double ag0, double ag1) {
    const uint32_t P = d.P;
    const uint32_t ns = d.n_sites;
    double coeff = method == 0 ? 0.5 : method == 1 ? 0.08333333333 : 0.2222222222;
    double sum01 = dt + dt1, sum12 = dt1 + dt2, sum012 = dt + (dt1 + dt2);
    double vmin = INFINITY, poison = 0.0;
    const double* r0 = d.sring + (size_t)((rot + 0) & 3) * ns * P;
    const double* r1 = d.sring + (size_t)((rot + 1) & 3) * ns * P;
    const double* r2 = d.sring + (size_t)((rot + 2) & 3) * ns * P;
    const double* r3 = d.sring + (size_t)((rot + 3) & 3) * ns * P;
    for (uint32_t j = 0; j < ns; j++) {
        double qc = LM(r0, j), qp = LM(r1, j), qp2 = LM(r2, j), qp3 = LM(r3, j), i_p = LM(d.sip, j);
        double i_new = cur_method == 1 ? ag0 * (qc - qp) - ag1 * i_p : ag0 * (qc - qp);
        double volttol = abstol + reltol * fmax(fabs(i_new), fabs(i_p));
        double chargetol = reltol * fmax(fmax(fabs(qc), fabs(qp)), chgtol) / dt;
        double tol = fmax(volttol, chargetol);
        poison += (qc - qc) + (qp - qp) + (qp2 - qp2) + (i_p - i_p);
        double f12 = (qp - qp2) / dt1;
        double dd = ((qc - qp) / dt - f12) / sum01;
        if (method != 0) {
            poison += qp3 - qp3;
            double f123 = (f12 - (qp2 - qp3) / dt2) / sum12;
            dd = (dd - f123) / sum012;
        }
        double del = trtol * tol / fmax(abstol, coeff * fabs(dd));
        poison += del == del ? 0.0 : del;
        vmin = fmin(vmin, del);
    }
    if (isnan(poison)) return NAN;
    return method == 0 ? vmin : sqrt(vmin);
}

// Transient start from the operating point in x: histories, the site ring,
// the first step (tran.zig:688-699 for LTE control), breakpoints.
__global__ void __launch_bounds__(128) k_tran_init(LaunchMap m, TranParams o, LaneState* st) {
    const GroupDev* d;
    uint32_t l;
    if (!lane_of(m, d, l)) return;
    const uint32_t P = d->P;
    LaneState& s = st[d->lane0 + l];
    seed_limits(*d, l, 0, d->x);
    eval_lane(*d, l, 1, 0.0);
    for (uint32_t i = 0; i < d->n; i++) {
        LM(d->cur, i) = LM(d->x, i);
        LM(d->prev, i) = LM(d->x, i);
        LM(d->q1, i) = LM(d->qrow, i);
        LM(d->ip, i) = 0.0;
    }
    uint32_t ns = d->n_sites;
    for (uint32_t k = 0; k < 4; k++)
        for (uint32_t j = 0; j < ns; j++) LM(d->sring + (size_t)k * ns * P, j) = LM(d->qs, j);
    for (uint32_t j = 0; j < ns; j++) LM(d->sip, j) = 0.0;
    s.s_rot = 0;
    s.t = 0.0;
    double dt;
    if (o.fixed_step) {
        dt = o.dt;
        s.dt_old0 = s.dt_old1 = o.dt;
    } else {
        dt = fmin(fmin(o.dt, o.t_stop / 100.0) / 10.0, o.dt_max);
        double bp0 = next_bp(*d, l, 0.0);
        if (bp0 < INFINITY) dt = fmin(dt, 0.1 * bp0);
        dt /= 10.0;
        s.dt_old0 = s.dt_old1 = o.dt_max;
    }
    s.dt = dt;
    s.order = 1;
    s.steps = 0;
    s.status = 0;
    s.rejects = 0;
    s.attempts = 0;
    s.nr_iters = 0;
    s.bp_next = o.fixed_step ? INFINITY : next_bp(*d, l, 0.0);
    s.bp_save_dt = 0.0;
    s.bp_clamped = 0;
    s.m_cross = 0;
    s.m_have = 0;
    s.m_first = s.m_last = NAN;
    s.fp64 = 0;
    s.peel_slot = 0xFFFFFFFFu;
}

// Up to o.launch_steps accepted-or-rejected attempts per lane.
template <bool MIXED>
__global__ void __launch_bounds__(128) k_tran(LaunchMap m, TranParams o, NewtonParams no, LaneState* st, PeelPool pool) {
    const GroupDev* dp;
    uint32_t l;
    if (!lane_of(m, dp, l)) return;
    const GroupDev& d = *dp;
    const uint32_t P = d.P;
    LaneState& s = st[d.lane0 + l];
    s.peel_slot = 0xFFFFFFFFu;  // the pool's counter restarts every launch
    const uint32_t ns = d.n_sites;
    for (uint32_t attempt = 0; attempt < o.launch_steps; attempt++) {
        if (s.status != 0) break;
        if (!(s.t < o.t_stop && !at_stop(s.t, o.t_stop) && s.steps < o.max_steps)) {
            s.status = 1;
            break;
        }
        double dt = s.dt;
        uint32_t method = s.order == 1 ? 0 : o.method;
        Companion cp;
        cp.on = 1;
        cp.method = method;
        if (method == 0) { cp.ag0 = 1.0 / dt; cp.ag1 = 1.0; }
        else { cp.ag0 = 1.0 / dt / (1.0 - 0.5); cp.ag1 = 0.5 / (1.0 - 0.5); }
        double t_dev = s.t + dt;
        double xfact = dt / s.dt_old0;
        for (uint32_t i = 0; i < d.n; i++) {
            double c = LM(d.cur, i);
            LM(d.x, i) = o.predictor == 1 ? c + xfact * (c - LM(d.prev, i)) : c;
        }
        // The limiter state restarts from the accepted point, then limits
        // the predicted iterate.
        seed_limits(d, l, 0, d.cur);
        limit_lane(d, l);
        NewtonParams np = no;
        np.init_fix = 0;
        np.max_iter = o.max_iter;
        s.fp64 = 0;
        newton_lane<MIXED>(d, l, s, np, 1, t_dev, cp, pool);
        s.attempts++;
        bool conv = (s.bits & kConverged) != 0;
        if (!(s.bits & kSingular)) s.nr_iters += s.iterations < o.max_iter ? s.iterations : o.max_iter;
        if (!conv) {
            s.rejects++;
            s.order = 1;
            if (o.fixed_step) { s.status = 2; break; }
            double ndt = dt / 8.0;
            if (ndt < o.dt_min && dt > o.dt_min && s.t + o.dt_min > s.t) ndt = o.dt_min;
            s.dt = ndt;
            if (ndt < o.dt_min) { s.status = 2; break; }
            continue;
        }
        // The last eval ran at the published x: its charges are the point's.
        double* r0 = d.sring + (size_t)(s.s_rot & 3) * ns * P;
        for (uint32_t j = 0; j < ns; j++) LM(r0, j) = LM(d.qs, j);
        double dt_next = s.steps == 0 ? dt : fmin(dt * 2.0, o.dt_max);
        if (o.fixed_step) {
            dt_next = dt;
            if (s.order == 1 && o.method != 0) s.order = 2;
        } else if (ns > 0 && s.steps > 0) {
            double del = step_bound(d, l, s.s_rot, method, method, dt, s.dt_old0, s.dt_old1, o.reltol, o.abstol,
                                    o.chgtol, o.trtol, cp.ag0, cp.ag1);
            double del2 = method == 0 ? step_bound(d, l, s.s_rot, o.method, method, dt, s.dt_old0, s.dt_old1,
                                                   o.reltol, o.abstol, o.chgtol, o.trtol, cp.ag0, cp.ag1)
                                      : del;
            if (!(del >= 0.9 * dt)) {
                s.rejects++;
                double ndt;
                if (isnan(del)) { s.order = 1; ndt = dt / 8.0; }
                else ndt = del;
                if (ndt < o.dt_min && dt > o.dt_min && s.t + o.dt_min > s.t) ndt = o.dt_min;
                s.dt = ndt;
                if (ndt < o.dt_min) { s.status = 2; break; }
                continue;
            }
            dt_next = fmin(fmin(fmax(del, o.dt_min), 2 * dt), o.dt_max);
            if (s.order == 1) {
                double trial = o.method == method ? del : del2;
                if (!isnan(trial)) {
                    double nd2 = fmin(2.0 * dt, trial);
                    if (nd2 > 1.05 * dt) s.order = 2;
                    dt_next = fmin(fmax(nd2, o.dt_min), o.dt_max);
                }
            }
        }
        // Accept (lane_device.zig accept): row histories, companion currents.
        for (uint32_t i = 0; i < d.n; i++) {
            double dq = cp.ag0 * (LM(d.qrow, i) - LM(d.q1, i));
            LM(d.ip, i) = method == 1 ? dq - cp.ag1 * LM(d.ip, i) : dq;
            LM(d.q1, i) = LM(d.qrow, i);
            LM(d.prev, i) = LM(d.cur, i);
            LM(d.cur, i) = LM(d.x, i);
        }
        {
            const double* q0 = d.sring + (size_t)((s.s_rot + 0) & 3) * ns * P;
            const double* q1 = d.sring + (size_t)((s.s_rot + 1) & 3) * ns * P;
            for (uint32_t j = 0; j < ns; j++) {
                double dq = cp.ag0 * (LM(q0, j) - LM(q1, j));
                LM(d.sip, j) = method == 1 ? dq - cp.ag1 * LM(d.sip, j) : dq;
            }
        }
        s.s_rot = (s.s_rot + 3) & 3;  // rotate right: new logical k = old k - 1
        s.dt_old1 = s.dt_old0;
        s.dt_old0 = dt;
        double t_new = s.t + dt;
        s.steps++;
        if (d.meas_row != 0xFFFFFFFFu && t_new >= d.meas_t0) {
            double v = LM(d.x, d.meas_row);
            if (s.m_have && s.m_prev_v < d.meas_level && v >= d.meas_level) {
                double tc = s.m_prev_t + (d.meas_level - s.m_prev_v) * (t_new - s.m_prev_t) / (v - s.m_prev_v);
                if (s.m_cross == 0) s.m_first = tc;
                s.m_last = tc;
                s.m_cross++;
            }
            s.m_prev_v = v;
            s.m_prev_t = t_new;
            s.m_have = 1;
        }
        // stepEndB (kernels/lane.zig:667-700).
        s.t = t_new;
        if (!o.fixed_step) {
            double nb = next_bp(d, l, t_new + o.min_break);
            if (s.bp_next != INFINITY) {
                double bp = s.bp_next;
                bool landed = s.bp_clamped ? fabs(t_new - bp) <= o.min_break
                                           : (bp - t_new <= o.delmin || almost_equal_ulps(t_new, bp, 100));
                if (landed) {
                    s.order = 1;
                    double shrink = s.bp_save_dt;
                    if (nb != INFINITY) shrink = fmin(shrink, nb - t_new);
                    dt_next = fmin(dt_next, 0.1 * shrink);
                }
            }
            s.bp_next = nb;
            s.bp_clamped = 0;
            if (nb != INFINITY) {
                double to_bp = nb - t_new;
                if (to_bp < dt_next) {
                    s.bp_save_dt = dt_next;
                    dt_next = to_bp;
                    s.bp_clamped = 1;
                }
            }
        }
        s.dt = dt_next;
        if (t_new + s.dt > o.t_stop) s.dt = o.t_stop - t_new;
    }
}

#undef LM

}  // namespace espl
