// The per-lane sequential engine of the lane sweep: the tape refactor, the
// triangular solves, the replay probe and the re-pivoting peel, each run by
// the thread that owns the lane. Lanes of one template sit
// interleaved (element i of lane l at i * P + l, P = lanes padded to a warp
// multiple), so a warp's 32 lanes read every nonzero of the shared pattern as
// one coalesced 256-byte load, while the tape's index words are warp-uniform.
//
// Semantics restated from ESPice:
//   eval + ground pin        src/device/eval.zig:780-920, src/analysis/Circuit.zig:861-864
//   refactor replay          src/solver/kernels/lane.zig:56-125 (Bodies.refactor)
//   luSolve (negated)        src/solver/kernels/lane.zig:137-157
//   updateNorm / plausible   src/solver/kernels/lane.zig:161-185
//   residual gate            src/solver/kernels/lane.zig:189-198
//   plausibleLimit           src/solver/kernels/lane.zig:202-214
//   gates / finalize         src/solver/lane_device.zig:326-384
//   companion rows / combine src/solver/kernels/lane.zig:221-242
//   stepBound                src/solver/kernels/lane.zig:257-297
//   step machine             src/solver/kernels/lane.zig:505-700
//   dense peel               src/solver/kernels/lane.zig:310-350
#pragma once

#include <cstdint>

#include "lane_gates.cuh"
#include "lane_meas.cuh"
#include "lane_models.cuh"

namespace espl {

constexpr uint32_t kTrashNone = 0xFFFFFFFFu;
constexpr double kXPlausible = 1e9;    // converger.x_plausible
constexpr double kWide = 1.0 / 1e-3;   // LaneTab.wide = 1 / pivot_tol
// Lanes of templates up to this size whose replay fails re-pivot densely on
// the device. The reference stops at 64 unknowns (kernels/lane.zig:301) and
// hands larger failed lanes to the host factor; with no host path here the
// dense peel covers up to 256, within a scratch budget (alloc_group).
constexpr uint32_t kDensePeelMax = 256;
constexpr uint32_t kFactKeys = 6;  // GroupDev fact_key words per lane
constexpr uint32_t kRefGroups = 8;  // column groups of a large template's refactor

// Gate bits (kernels/lane.zig:708-711).
constexpr uint32_t kActive = 1, kInitFix = 2, kConverged = 4, kSingular = 8, kPassed = 16, kParked = 32;

struct GroupDev {
    uint32_t n, nnz, nnz_l, nnz_u, lanes, P, warp0, lane0;
    uint32_t n_void, n_res, n_cap, n_vsrc, n_isrc, n_dio, n_mos, n_sites;
    uint32_t has_charge, meas_row;
    double meas_level, meas_t0;
    // Streaming .meas passes (lane_meas.cuh): n_mpass descriptors and their
    // lane-major states (n_mpass * kMeasWords * P).
    const espl_meas* mpass;
    double* mstate;
    uint32_t n_mpass, mpass_pad;
    const uint32_t *col_ptr, *row_idx, *prow, *q, *pinv, *lp, *li, *up, *ui, *flags, *void_slots, *diag;
    const uint32_t *rt_ptr, *rt_col, *rt_pos;  // row view of the pattern: per row, (column, slot) by column
    const uint32_t* lu_prog;                   // the replay as a flat program (tape.h lu_program)
    uint32_t n_prog, prog_pad;
    const uint32_t* lu_rec;                    // the replay as 16-byte records (tape.h lu_records)
    uint32_t n_rec, rec_stage;                 // n_rec words (0: the shared chain replays from the tape);
                                               // rec_stage: the records are staged in shared memory
    const uint32_t* sol_rec;                   // the solves as 16-byte records (tape.h solve_records)
    uint32_t n_srec, srec_stage;               // likewise for the solves
    // The banded streaming replay (lane_band.cuh, tape.h BandPlan): ring
    // sizes, chunk capacities and count, the shared-memory offset of its
    // buffers, and the chunk tables and scatter slots in global memory.
    uint32_t band_ok, band_w, band_l, band_chunks, band_cw, band_ce, band_off, band_b;
    uint32_t band_nblk, band_pad;
    const uint32_t *band_cpc, *band_cent, *band_slot, *band_scol, *band_rowof;
    const uint8_t* cur_row;
    const uint32_t *res_t, *res_s, *cap_t, *cap_s, *vsrc_t, *vsrc_s, *isrc_t, *dio_t, *dio_s, *mos_t, *mos_s;
    const double *res_r, *cap_c, *vsrc_p, *isrc_p, *dio_d, *mos_d;
    // When every MOS has the same type, gamma, phi, lambda and IS on all
    // lanes (Monte Carlo varies VTO and KP), the prep values that depend only
    // on those are the same on every lane: mos_u holds them once per
    // instance (kMosUni values: type, vt, lambda, gamma, phit, isat, vcrit,
    // gmin), read as broadcast loads instead of one load per lane.
    const double* mos_u;
    uint32_t mos_uni, mos_uni_pad;
    double *x, *x_old, *dx, *rhs, *qrow, *g, *c, *a, *lx, *ux, *udiag, *w, *y, *lim_mos, *lim_dio;
    float *lx32, *ux32, *udiag32, *w32, *y32;
    double *q1, *q2, *ip, *cur, *prev, *sring, *sip;  // q2: row charges two accepted steps back (gear-2)
    double *rr, *corr;
    double* peel_m;      // n <= kDensePeelMax: the lanes' dense peel scratch (peel_doubles(n) per lane)
    uint32_t* peel_i;    // n <= kDensePeelMax: its index words (peel_words(n) per lane)
    // Stamp plan: per-instance output cells (lane-major) and, per Jacobian
    // slot and residual/charge row, the cells that sum into it in the
    // reference's stamping order (bit 31: the cell enters negated).
    uint32_t tile0, n_cells, c_res, c_cap, c_vsrc, c_isrc, c_dio, c_mos, c_pin, c_const;
    const uint32_t *g_ptr, *g_cell, *c_ptr, *c_cell, *r_ptr, *r_cell, *q_ptr, *q_cell, *site_cell;
    const uint8_t* slot_diag;
    double* cells;
    double* site_prev;  // an iteration's site charges, kept before its limiter pass overwrites the cells
    uint32_t n_gc, n_cc, n_rc, n_qc;  // lengths of g_cell, c_cell, r_cell, q_cell
    // The same sums as one flat list for the Newton gather (lane_tile.cuh
    // gather_items): items are the nnz slots, then the n rows; an item's
    // entries (gi_ptr[k] .. gi_ptr[k + 1]) are its G (R) cells, its C (Q)
    // cells, and for a row the q1, ip, q2 and x values its companion and gmin
    // terms read. Each warp of a tile takes a run of items with about the
    // same number of entries: gsplit4 for 4-warp tiles, gsplit16 for 16.
    const uint32_t *gi_ptr, *gi_ent;
    uint32_t n_gi, n_items;
    uint32_t gsplit4[5], gsplit16[17];
    uint32_t gsplit_pad[2];
    const uint32_t* gsplit_big;  // the same for the kBigWarps shares of a large template's part
    // Stale-tape words of the template: [0] set when, in some Newton
    // iteration, at least half of a tile's active lanes failed the replay;
    // [1] the smallest such failing lane (the host retapes from its A).
    uint32_t* stale;
    // ngspice's diagonal-gmin placement for the ladder's gmin steps (slot,
    // row, column triples: gmin on A[slot], gmin * x[column] on row), and
    // the lanes' last converged iterate of a ladder rung.
    const uint32_t* gstamp;
    uint32_t n_gstamp, gstamp_pad;
    double* x_good;
    uint32_t stage_mode;  // what a tile stages in shared memory (lane_smem.cuh)
    uint32_t refine_rows; // the row view is staged (FP32 refinement sweeps on)
    // The learned next-step predictor (lane_learned.cuh): the accepted
    // solution two steps back (null when neither a predictor nor a recorder
    // is attached), the learned start of each lane's next attempt (null
    // without a predictor), and the step recorder: samples of lanes l with
    // l % rec_stride == 0 past step rec_from, at most rec_cap, their features
    // (rec_x, 3 n + 1 per sample), targets (rec_y, n per sample) and tags
    // (rec_tag, 5 per sample), the next free sample in *rec_count.
    double *prev2, *xpred;
    double *rec_x, *rec_y, *rec_tag;
    uint32_t* rec_count;
    uint32_t rec_stride, rec_from, rec_cap, rec_pad;
    // Large templates (lane_levels.cuh, big = 1): the whole CTA refactors by
    // columns and solves by levels (tape.h LevelPlan). linear: no nonlinear
    // device, so a lane's A depends only on its companion coefficient and
    // gmin; fact_key (kFactKeys per lane) names, by such a key pair (the
    // ag0, or -1 without a companion, and the gmin), the A of the lane's
    // FP64 factor (words 0-1), of its FP32 factor (2-3) and the A assembled
    // in `a` (4-5). An unchanged key skips the refactor (the reference skips
    // refactoring identical values, src/solver/direct.zig:313), and the
    // gather of A's entries (the right-hand sides are still gathered).
    const uint32_t *fl_ptr, *fl_rows, *bl_ptr, *bl_rows, *rl_ptr, *rl_ent, *ru_ptr, *ru_ent;
    uint32_t n_fl, n_bl, big, linear;
    double* fact_key;
    const struct StreamDev* stream;  // the sweeps in streaming order (lane_levels.cuh), or null
    // The refactor's column levels (tape.h ColPlan; n_cl levels) and the
    // work vectors of the column groups past the first (kRefGroups - 1
    // copies of w, (n + 1) x P each; FP32 copies for a mixed handle), or null
    const uint32_t *cl_ptr, *cl_gp, *cl_cols;
    const uint4* cl_ustream;  // per U entry: its row, its L column's bounds
    uint32_t n_cl, cl_pad;
    double* wk;
    float* wk32;
};

// One sweep of a large template's solve in streaming order (tape.h
// StreamPlan), and the factor's values copied into that order: for the
// lanes of part p (tw lanes), entry e of the sweep at (p * entries + e) * tw
// + lane, so that a chunk of entries is one contiguous block per part.
struct StreamSweep {
    const uint32_t *col, *slot, *ch, *meta, *mo;
    uint32_t entries, n_chunks, max_meta, pad;
};
struct StreamDev {
    StreamSweep fw, bw;
    double *vf, *vb;    // FP64 L and U values in streaming order
    float *vf32, *vb32; // FP32 (mixed)
};

struct LaneState {
    double limit;
    double t, dt, dt_old0, dt_old1, bp_next, bp_save_dt;
    double m_prev_v, m_prev_t, m_first, m_last;
    unsigned long long attempts, nr_iters;
    uint32_t bits, pred_fallbacks, iterations, fallbacks;  // pred_fallbacks: learned starts retried linearly
    uint32_t order, steps, status, rejects;
    uint32_t bp_clamped, m_cross, m_have, event;  // event: kernels/lane.zig step_idle/attempt/accept/reject
    uint32_t s_rot, fp64, peels, pred_lin;  // pred_lin: the next attempt starts from the linear predictor
    double t_new, attempted_dt;  // the last attempt's candidate time and step
};

// LaneStep.event (src/solver/kernels/lane.zig:461-465).
constexpr uint32_t kEventIdle = 0, kEventAttempt = 1, kEventAccept = 2, kEventReject = 3;
// LaneStep.status (kernels/lane.zig:455-460).
constexpr uint32_t kStepRun = 0, kStepDone = 1, kStepUnderflow = 2, kStepParked = 3, kStepStopped = 4;

// The three history features of unknown i (f[0] = cur, f[1] the linear
// predictor's increment, f[2] the increment a step earlier). The recorder
// (k_tran's accept) and the predictor (lane_learned.cuh) compute them with this one function,
// so a sample's target y = x - (cur + f[1]) and the predictor's start
// cur + f[1] + y agree to the bit.
__host__ __device__ __forceinline__ void step_features(double cur, double prev, double prev2, double r0, double r1,
                                                       double* f) {
    f[0] = cur;
    f[1] = r0 * (cur - prev);
    f[2] = r1 * (prev - prev2);
}

// One lane's solve in a rung of the operating-point continuation ladder
// (espl_solve_op): its diagonal gmin at the template's gmin stamps (0:
// none), the scale of its independent sources, whether it solves in this
// launch and whether from a cold start.
struct LadderLane {
    double gmin, src;
    uint32_t on, init_fix;
};

struct NewtonParams {
    double reltol, abstol, vntol, gmin, residual_tol;
    // polish > 0: once a lane's step passes Newton's test, it keeps iterating
    // until the step also passes the test with every tolerance scaled by
    // `polish`, for at most polish_max further iterations
    double polish;
    uint32_t max_iter, init_fix;
    uint32_t mixed, stall_ticks;   // mixed: FP32 LU; a lane past stall_ticks refactors in FP64
    uint32_t refine;               // mixed: FP64-residual refinement sweeps per solve
    uint32_t polish_max;
    uint32_t chord;                // polish iterations reuse the previous factor (shared-memory chain)
    const LadderLane* ladder;      // per lane (all templates' lanes), or null: gmin, init_fix, all lanes
};

struct TranParams {
    double t_stop, dt, dt_min, dt_max, reltol, abstol, chgtol, trtol, vntol, residual_tol;
    double delmin, min_break;
    uint32_t method, fixed_step, max_iter, max_steps, predictor, launch_steps, polish_chord;
};

struct Companion {
    int on;
    uint32_t method;  // 0 BE, 1 trap, 2 gear-2
    double ag0, ag1, ag2;
};

#define LM(arr, i) (arr)[(size_t)(i) * P + l]

__device__ __forceinline__ uint64_t dbits(double v) { return (uint64_t)__double_as_longlong(v); }
__device__ __forceinline__ double bitsd(uint64_t b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ uint32_t fbits(float v) { return (uint32_t)__float_as_int(v); }

// ---------------------------------------------------------------------------
// LU replay of the frozen tape, FP64 (Bodies.refactor + wideMultipliers).
// 0: the replay holds; 1: a pivot failed (dead, non-finite, growth), an L/U
// entry is non-finite or a void slot filled; 2: only a multiplier past
// 1 / pivot_tol, which `replay_holds64` may still accept.
__device__ int refactor64(const GroupDev& d, uint32_t l) {
    const uint32_t P = d.P;
    const double* __restrict__ a = d.a;
    double* __restrict__ w = d.w;
    double* __restrict__ lx = d.lx;
    double* __restrict__ ux = d.ux;
    double* __restrict__ ud = d.udiag;
    for (uint32_t v = 0; v < d.n_void; v++)
        if (LM(a, d.void_slots[v]) != 0.0) return 1;
    bool bad = false;
    uint64_t nonfinite = 0;
    const double growth = 1e-12;
    for (uint32_t k = 0; k < d.n; k++) {
        uint32_t c = d.q[k];
        for (uint32_t p = d.col_ptr[c]; p < d.col_ptr[c + 1]; p++) LM(w, d.prow[p]) = LM(a, p);
        for (uint32_t p = d.up[k]; p < d.up[k + 1]; p++) {
            uint32_t i = d.ui[p];
            double uki = LM(w, i);
            LM(w, i) = 0.0;
            LM(ux, p) = uki;
            nonfinite |= dbits(uki - uki);
            for (uint32_t pl = d.lp[i]; pl < d.lp[i + 1]; pl++) LM(w, d.li[pl]) -= LM(lx, pl) * uki;
        }
        uint32_t fl = d.flags[k];
        if (fl & 1u) {
            LM(ud, k) = 1.0;
            for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) { LM(lx, p) = 0.0; LM(w, d.li[p]) = 0.0; }
            LM(w, k) = 0.0;
            for (uint32_t p = d.up[k]; p < d.up[k + 1]; p++) {
                uint32_t i = d.ui[p];
                for (uint32_t pl = d.lp[i]; pl < d.lp[i + 1]; pl++) LM(w, d.li[pl]) = 0.0;
            }
            continue;
        }
        double dk = LM(w, k);
        LM(w, k) = 0.0;
        bool dead = dk == 0.0 || !(fabs(dk) < INFINITY);
        bad |= dead;
        if (dead) dk = 1.0;
        LM(ud, k) = dk;
        if (!(fl & 2u)) {
            uint64_t cb = dbits(fabs(dk));
            for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) {
                uint32_t r = d.li[p];
                double v = LM(w, r);
                LM(w, r) = 0.0;
                uint64_t vb = dbits(fabs(v));
                cb = cb > vb ? cb : vb;
                LM(lx, p) = v / dk;
            }
            bad |= !(fabs(dk) >= growth * bitsd(cb));
        } else {
            for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) {
                uint32_t r = d.li[p];
                double lv = LM(w, r) / dk;
                nonfinite |= dbits(lv - lv);
                LM(lx, p) = lv;
                LM(w, r) = 0.0;
            }
        }
    }
    if (nonfinite || bad) return 1;
    uint64_t worst = 0;
    for (uint32_t k = 0; k < d.n; k++) {
        if (d.flags[k] & 2u) continue;
        for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) {
            uint64_t b = dbits(fabs(LM(lx, p)));
            worst = worst > b ? worst : b;
        }
    }
    return bitsd(worst) <= kWide ? 0 : 2;
}

// The same replay in FP32 with FP32 accumulation over the FP64 matrix.
__device__ bool refactor32(const GroupDev& d, uint32_t l) {
    const uint32_t P = d.P;
    const double* __restrict__ a = d.a;
    float* __restrict__ w = d.w32;
    float* __restrict__ lx = d.lx32;
    float* __restrict__ ux = d.ux32;
    float* __restrict__ ud = d.udiag32;
    for (uint32_t v = 0; v < d.n_void; v++)
        if (LM(a, d.void_slots[v]) != 0.0) return true;
    bool bad = false;
    uint32_t nonfinite = 0;
    const float growth = 1e-12f;
    for (uint32_t k = 0; k < d.n; k++) {
        uint32_t c = d.q[k];
        for (uint32_t p = d.col_ptr[c]; p < d.col_ptr[c + 1]; p++) LM(w, d.prow[p]) = (float)LM(a, p);
        for (uint32_t p = d.up[k]; p < d.up[k + 1]; p++) {
            uint32_t i = d.ui[p];
            float uki = LM(w, i);
            LM(w, i) = 0.0f;
            LM(ux, p) = uki;
            nonfinite |= fbits(uki - uki);
            for (uint32_t pl = d.lp[i]; pl < d.lp[i + 1]; pl++) LM(w, d.li[pl]) -= LM(lx, pl) * uki;
        }
        uint32_t fl = d.flags[k];
        if (fl & 1u) {
            LM(ud, k) = 1.0f;
            for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) { LM(lx, p) = 0.0f; LM(w, d.li[p]) = 0.0f; }
            LM(w, k) = 0.0f;
            for (uint32_t p = d.up[k]; p < d.up[k + 1]; p++) {
                uint32_t i = d.ui[p];
                for (uint32_t pl = d.lp[i]; pl < d.lp[i + 1]; pl++) LM(w, d.li[pl]) = 0.0f;
            }
            continue;
        }
        float dk = LM(w, k);
        LM(w, k) = 0.0f;
        bool dead = dk == 0.0f || !(fabsf(dk) < INFINITY);
        bad |= dead;
        if (dead) dk = 1.0f;
        LM(ud, k) = dk;
        float cmax = fabsf(dk);
        for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) {
            uint32_t r = d.li[p];
            float v = LM(w, r);
            LM(w, r) = 0.0f;
            cmax = fmaxf(cmax, fabsf(v));
            float lv = v / dk;
            nonfinite |= fbits(lv - lv);
            LM(lx, p) = lv;
        }
        if (!(fl & 2u)) bad |= !(fabsf(dk) >= growth * cmax) || !(cmax / fabsf(dk) <= (float)kWide);
    }
    return bad || nonfinite;
}

// dx = -A^-1 rhs through the FP64 factors (luSolve with neg).
__device__ void solve64(const GroupDev& d, uint32_t l, const double* __restrict__ rhs, double* __restrict__ out) {
    const uint32_t P = d.P;
    double* __restrict__ y = d.y;
    const double* __restrict__ lx = d.lx;
    const double* __restrict__ ux = d.ux;
    for (uint32_t r = 0; r < d.n; r++) LM(y, d.pinv[r]) = -LM(rhs, r);
    for (uint32_t k = 0; k < d.n; k++) {
        double yk = LM(y, k);
        if (yk != 0.0)
            for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) LM(y, d.li[p]) -= LM(lx, p) * yk;
    }
    for (uint32_t k = d.n; k-- > 0;) {
        double zk = LM(y, k) / LM(d.udiag, k);
        LM(y, k) = zk;
        if (zk != 0.0)
            for (uint32_t p = d.up[k]; p < d.up[k + 1]; p++) LM(y, d.ui[p]) -= LM(ux, p) * zk;
    }
    for (uint32_t j = 0; j < d.n; j++) LM(out, d.q[j]) = LM(y, j);
}

// x = A^-T b through the FP64 factors (SparseLu.solveT,
// src/solver/sparse_lu.zig:1326-1361). `y` is the work vector.
__device__ void solve_t64(const GroupDev& d, uint32_t l, const double* __restrict__ b, double* __restrict__ out) {
    const uint32_t P = d.P;
    double* __restrict__ y = d.y;
    for (uint32_t k = 0; k < d.n; k++) LM(y, k) = LM(b, d.q[k]);
    for (uint32_t k = 0; k < d.n; k++) {
        double yk = LM(y, k);
        for (uint32_t p = d.up[k]; p < d.up[k + 1]; p++) yk -= LM(d.ux, p) * LM(y, d.ui[p]);
        LM(y, k) = yk / LM(d.udiag, k);
    }
    for (uint32_t k = d.n; k-- > 0;) {
        double yk = LM(y, k);
        for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) yk -= LM(d.lx, p) * LM(y, d.li[p]);
        LM(y, k) = yk;
    }
    for (uint32_t r = 0; r < d.n; r++) LM(out, r) = LM(y, d.pinv[r]);
}

// direct.zig replayHolds (:402-447) for a replay whose only failure is a
// multiplier past 1 / pivot_tol: a probe right-hand side solved both ways
// must leave a scaled residual within replay_ratio_max / pivot_tol = 3e4.
// Scratch: rr (residual), corr (solution), x_old (row sums; free until the
// update that follows the solve).
__device__ bool replay_holds64(const GroupDev& d, uint32_t l) {
    const uint32_t P = d.P;
    const uint32_t n = d.n;
    double* __restrict__ r = d.rr;
    double* __restrict__ xs = d.corr;
    double* __restrict__ rows = d.x_old;
    for (uint32_t i = 0; i < n; i++) LM(rows, i) = 0.0;
    double norm_1 = 0.0;
    for (uint32_t j = 0; j < n; j++) {
        double col = 0.0;
        for (uint32_t p = d.col_ptr[j]; p < d.col_ptr[j + 1]; p++) {
            double av = fabs(LM(d.a, p));
            LM(rows, d.row_idx[p]) += av;
            col += av;
        }
        norm_1 = fmax(norm_1, col);
    }
    uint64_t nb = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint64_t b = dbits(fabs(LM(rows, i)));
        nb = nb > b ? nb : b;
    }
    double norm_inf = bitsd(nb);
    double den = (double)((n > 2 ? n : 2) - 1);
    for (int transpose = 0; transpose <= 1; transpose++) {
        // solve64 returns -A^-1 b, so it gets the negated probe.
        for (uint32_t i = 0; i < n; i++) {
            double mag = 1.0 + (double)i / den;
            LM(r, i) = (i % 2 == 0) ? mag : -mag;
        }
        if (transpose) {
            solve_t64(d, l, r, xs);
        } else {
            for (uint32_t i = 0; i < n; i++) LM(r, i) = -LM(r, i);
            solve64(d, l, r, xs);
            for (uint32_t i = 0; i < n; i++) LM(r, i) = -LM(r, i);
        }
        for (uint32_t j = 0; j < n; j++)
            for (uint32_t p = d.col_ptr[j]; p < d.col_ptr[j + 1]; p++) {
                uint32_t i = d.row_idx[p];
                if (transpose) LM(r, j) -= LM(d.a, p) * LM(xs, i);
                else LM(r, i) -= LM(d.a, p) * LM(xs, j);
            }
        uint64_t rm = 0, xm = 0;
        for (uint32_t i = 0; i < n; i++) {
            uint64_t b1 = dbits(fabs(LM(r, i))), b2 = dbits(fabs(LM(xs, i)));
            rm = rm > b1 ? rm : b1;
            xm = xm > b2 ? xm : b2;
        }
        double a_norm = transpose ? norm_1 : norm_inf;
        double ratio = bitsd(rm) / (a_norm * bitsd(xm) * (double)n * 2.220446049250313e-16);
        if (!(ratio <= 30.0 / 1e-3)) return false;
    }
    return true;
}

// The same through the FP32 factors; the right-hand side is rounded to
// FP32 and the result widened back.
__device__ void solve32(const GroupDev& d, uint32_t l, const double* __restrict__ rhs, double* __restrict__ out) {
    const uint32_t P = d.P;
    float* __restrict__ y = d.y32;
    const float* __restrict__ lx = d.lx32;
    const float* __restrict__ ux = d.ux32;
    for (uint32_t r = 0; r < d.n; r++) LM(y, d.pinv[r]) = (float)(-LM(rhs, r));
    for (uint32_t k = 0; k < d.n; k++) {
        float yk = LM(y, k);
        if (yk != 0.0f)
            for (uint32_t p = d.lp[k]; p < d.lp[k + 1]; p++) LM(y, d.li[p]) -= LM(lx, p) * yk;
    }
    for (uint32_t k = d.n; k-- > 0;) {
        float zk = LM(y, k) / LM(d.udiag32, k);
        LM(y, k) = zk;
        if (zk != 0.0f)
            for (uint32_t p = d.up[k]; p < d.up[k + 1]; p++) LM(y, d.ui[p]) -= LM(ux, p) * zk;
    }
    for (uint32_t j = 0; j < d.n; j++) LM(out, d.q[j]) = (double)LM(y, j);
}

// One refinement sweep of a mixed solve. The linear system is A dx = -rhs;
// r = rhs + A dx is its FP64 residual (negated), and the FP32 factors turn it
// into the correction -A^-1 r that dx takes.
__device__ void refine_mixed(const GroupDev& d, uint32_t l) {
    const uint32_t P = d.P;
    double* __restrict__ r = d.rr;
    double* __restrict__ corr = d.corr;
    for (uint32_t i = 0; i < d.n; i++) LM(r, i) = LM(d.rhs, i);
    for (uint32_t c = 0; c < d.n; c++) {
        double xc = LM(d.dx, c);
        if (xc == 0.0) continue;
        for (uint32_t p = d.col_ptr[c]; p < d.col_ptr[c + 1]; p++) LM(r, d.row_idx[p]) += LM(d.a, p) * xc;
    }
    solve32(d, l, r, corr);
    for (uint32_t i = 0; i < d.n; i++) LM(d.dx, i) += LM(corr, i);
}

// x = -A^-1 b for a lane whose replayed pivots failed, by a dense
// re-pivoting factor that takes the decisions of the host's full factor
// (SparseLu.factorPass, src/solver/sparse_lu.zig:505-581) in the tape's
// column order: per step the diagonal (or the row a hand-off gave the
// column) while |d| >= pivot_tol * column max, else the same test under row
// scaling, else the column max; the row a column loses goes to the column
// that wanted the taken row. No absolute pivot floor: only a zero or
// non-finite column fails, as there. The reference's device peel is a
// plain partial-pivoting LU with an eps^2 floor (kernels/lane.zig:310-350)
// that refuses the ill-conditioned iterates a cold operating point passes
// through; the host factor accepts them.
// The peel scratch of a template of n <= kDensePeelMax, per lane, lane-interleaved
// like every other per-lane array (element i of lane l at i * P + l):
// m[n * n] row-major, xv[n] (right-hand side, then the solution by unknown),
// rscale[n], sol[n] as doubles; want, want_of, pinv, row_of[n] as u32.
__host__ __device__ constexpr uint32_t peel_doubles(uint32_t n) { return n * n + 3 * n; }
__host__ __device__ constexpr uint32_t peel_words(uint32_t n) { return 4 * n; }

#define PM(i) pm[(size_t)(i) * P + l]
#define PI(i) pi[(size_t)(i) * P + l]

__device__ bool dense_repivot_neg(uint32_t n, const uint32_t* q, double* pm, uint32_t* pi, uint32_t P, uint32_t l) {
    const uint32_t X = n * n, RS = X + n, SOL = RS + n;
    const uint32_t WANT = 0, WOF = n, PINV = 2 * n, ROW = 3 * n;
    const double tol = 1e-3;
    const double big = 1.7976931348623157e308;
    const uint32_t none = 0xFFFFFFFFu;
    for (uint32_t r = 0; r < n; r++) {
        double mx = 0.0;
        for (uint32_t c = 0; c < n; c++) mx = fmax(mx, fabs(PM(r * n + c)));
        PM(RS + r) = (mx > 0.0 && mx <= big) ? 1.0 / mx : 1.0;
        PI(WANT + r) = r;
        PI(WOF + r) = r;
        PI(PINV + r) = none;
        PM(X + r) = -PM(X + r);
    }
    for (uint32_t k = 0; k < n; k++) {
        uint32_t c = q[k];
        double amax = 0.0, smax = 0.0;
        uint32_t piv = none;
        for (uint32_t r = 0; r < n; r++) {
            if (PI(PINV + r) != none) continue;
            double av = fabs(PM(r * n + c));
            if (av > amax) { amax = av; piv = r; }
            smax = fmax(smax, av * PM(RS + r));
        }
        if (piv == none || amax == 0.0 || !(amax <= big)) return false;
        uint32_t pr = PI(WANT + c);
        if (PI(PINV + pr) == none) {
            double dmag = fabs(PM(pr * n + c));
            if (dmag > 0.0 && (dmag >= tol * amax || dmag * PM(RS + pr) >= tol * smax)) piv = pr;
        }
        if (piv != pr) {
            uint32_t c2 = PI(WOF + piv);
            PI(WANT + c2) = pr;
            PI(WOF + pr) = c2;
        }
        PI(PINV + piv) = k;
        PI(ROW + k) = piv;
        double dv = PM(piv * n + c);
        double xp = PM(X + piv);
        for (uint32_t r = 0; r < n; r++) {
            if (PI(PINV + r) != none) continue;
            double f = PM(r * n + c) / dv;
            if (f == 0.0) continue;
            for (uint32_t kk = k + 1; kk < n; kk++) {
                uint32_t cc = q[kk];
                PM(r * n + cc) -= f * PM(piv * n + cc);
            }
            PM(X + r) -= f * xp;
        }
    }
    for (uint32_t k = n; k-- > 0;) {
        uint32_t r = PI(ROW + k);
        double acc = PM(X + r);
        for (uint32_t kk = k + 1; kk < n; kk++) acc -= PM(r * n + q[kk]) * PM(SOL + q[kk]);
        double v = acc / PM(r * n + q[k]);
        if (!(fabs(v) <= big)) return false;
        PM(SOL + q[k]) = v;
    }
    return true;
}

// A failed replay of a lane with n <= kDensePeelMax solves densely in the lane's own
// peel scratch (the place of arp_lane_peel_dense, lane_device.zig:120-147),
// re-pivoting as the host factor would; dx gets the step.
__device__ bool peel_dense(const GroupDev& d, uint32_t l, LaneState& s) {
    const uint32_t P = d.P;
    const uint32_t n = d.n;
    if (n > kDensePeelMax || d.peel_m == nullptr) return false;
    double* pm = d.peel_m;
    uint32_t* pi = d.peel_i;
    for (uint32_t i = 0; i < n * n; i++) PM(i) = 0.0;
    for (uint32_t c = 0; c < n; c++)
        for (uint32_t p = d.col_ptr[c]; p < d.col_ptr[c + 1]; p++) PM(d.row_idx[p] * n + c) += LM(d.a, p);
    for (uint32_t i = 0; i < n; i++) PM(n * n + i) = LM(d.rhs, i);
    s.peels++;
    if (!dense_repivot_neg(n, d.q, pm, pi, P, l)) return false;
    const uint32_t SOL = n * n + 2 * n;
    for (uint32_t i = 0; i < n; i++) LM(d.dx, i) = PM(SOL + i);
    return true;
}

#undef PM
#undef PI

}  // namespace espl
