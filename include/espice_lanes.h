/* espice_lanes: the GPU lane-sweep seam of ESPice, as a C ABI for B200
 * (sm_100a). Many sweep points ("lanes") of one or more circuit templates
 * run together on the GPU: per-lane device evaluation and MNA stamping,
 * numeric refactorization of a frozen Gilbert-Peierls pivot tape on the
 * BTF/AMD column order, and forward/back substitution, inside the
 * operating-point Newton loop and the transient step loop.
 *
 * Each entry point replaces one call of the reference's GPU lane driver
 * `GpuLanes` (src/analysis/gpu/lanes.zig), which the Zig host code
 * (src/analysis/dc/op.zig solveGpuLanes, src/analysis/tran/tran.zig
 * runGpuLanes, src/c_api.zig) reaches through Gompute kernel handles. Only C
 * types cross this boundary, so a Zig `extern fn` declaration binds it as is.
 *
 * Ownership: the handle owns all device memory; arrays passed in are
 * borrowed for the duration of the call only. Calls on one handle must be
 * serialized; different handles are independent.
 */
#ifndef ESPICE_LANES_H
#define ESPICE_LANES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ESPL_ABI_VERSION 3u

/* A device terminal on the datum node. Its residual row and Jacobian
 * entries are dropped, as the reference's GROUND gather does
 * (src/device/eval.zig evalRange, `gi != GROUND`). */
#define ESPL_GROUND 0xFFFFFFFFu

typedef uint32_t espl_status;
/* Mirrors the reference's lane errors (lanes.zig:165-172: NoLaneImage,
 * NoLaneTape, IncompatibleLanes) plus driver, memory and timeout codes. */
enum {
    ESPL_OK = 0,
    ESPL_INVALID_ARGUMENT = 1,
    ESPL_NO_IMAGE = 2,        /* no CUDA device or kernel image for it */
    ESPL_NO_TAPE = 3,         /* the lead lane's host factor failed */
    ESPL_INCOMPATIBLE = 4,    /* lanes the device path refuses */
    ESPL_DRIVER = 5,          /* a CUDA runtime error */
    ESPL_OUT_OF_MEMORY = 6,
    ESPL_TIMEOUT = 7,         /* a bounded device loop ran out */
    ESPL_TOO_LARGE = 8        /* a size beyond a stated maximum */
};

/* Device kinds. Terminal and parameter rows per kind:
 *   RES   term p n           param r                                   (models/resistor.va)
 *   CAP   term p n           param c                                   (models/capacitor.va)
 *   VSRC  term p n br        param dc wave v1 v2 td tr tf pw per        (models/vsource.va; br = branch-current unknown)
 *   ISRC  term p n           param dc wave v1 v2 td tr tf pw per        (models/isource.va)
 *   DIODE term a c           param is n cjo vj m fc tt                  (models/diode.va, rs = 0)
 *   MOS1  term d g s b       param type vto kp gamma phi lambda is w l  (models/mos1.va, rd = rs = 0, no TOX, no CJ)
 * wave: 0 DC, 1 PULSE. */
enum { ESPL_RES = 1, ESPL_CAP = 2, ESPL_VSRC = 3, ESPL_ISRC = 4, ESPL_DIODE = 5, ESPL_MOS1 = 6 };
#define ESPL_RES_TERMS 2u
#define ESPL_RES_PARAMS 1u
#define ESPL_CAP_TERMS 2u
#define ESPL_CAP_PARAMS 1u
#define ESPL_SRC_PARAMS 9u
#define ESPL_VSRC_TERMS 3u
#define ESPL_ISRC_TERMS 2u
#define ESPL_DIODE_TERMS 2u
#define ESPL_DIODE_PARAMS 7u
#define ESPL_MOS1_TERMS 4u
#define ESPL_MOS1_PARAMS 9u

/* One device batch of a template: `count` instances of `kind`.
 * term[i * terms + t] is the unknown of terminal t of instance i, or
 * ESPL_GROUND. param[(i * params + k) * lanes + l] is parameter k of
 * instance i in lane l (lane-major, the layout the device reads). */
typedef struct {
    uint32_t kind;
    uint32_t count;
    const uint32_t *term;
    const double *param;
} espl_batch;

/* One circuit template and its lanes. Unknown 0 is the ground row, pinned
 * by G[0,0] += 1 and F[0] += x[0] after every stamp (src/analysis/Circuit.zig
 * groundStamp). The CSC pattern must hold every diagonal and every entry the
 * devices stamp. */
typedef struct {
    uint32_t n;
    uint32_t nnz;
    const uint32_t *col_ptr; /* n + 1 */
    const uint32_t *row_idx; /* nnz */
    uint32_t n_batches;
    const espl_batch *batches;
    uint32_t lanes;
} espl_netlist;

/* Newton controls: `converger.Options` (src/solver/converger.zig) as the
 * device gates read them (`NewtonOpts`, src/solver/kernels/lane.zig:719). */
typedef struct {
    double reltol;       /* 1e-3 */
    double abstol;       /* 1e-12 A, current rows */
    double vntol;        /* 1e-6 V */
    double gmin;         /* diagonal gmin; 0 in the plain operating-point rung */
    double residual_tol; /* 1e-9 */
    uint32_t max_iter;   /* 100 */
    uint32_t init_fix;   /* 1: cold operating point (MODEINITJCT/INITFIX). This
                          * word is the reference NewtonOpts' trailing `_pad`
                          * (48 bytes either way): a host that binds the
                          * reference layout passes 0 there, a warm start. */
} espl_newton_opts;

/* Per-lane outcome: `LaneNewton` of lanes.zig. bits: 4 converged,
 * 8 singular (the lane's replay failed), 32 handed back to the host. */
typedef struct {
    uint32_t bits;
    uint32_t iterations;
    uint32_t refactor_fallbacks; /* mixed precision: FP64 refactors taken */
    uint32_t reserved;
} espl_lane_newton;

#define ESPL_CONVERGED 4u
#define ESPL_SINGULAR 8u
#define ESPL_PARKED 32u

/* Precision of the LU refactor and triangular solves. Device evaluation,
 * residuals, the Newton update and step control are FP64 in both. */
enum { ESPL_FP64 = 0, ESPL_MIXED = 1 };

typedef struct {
    uint32_t abi_version;
    uint32_t precision;      /* ESPL_FP64 or ESPL_MIXED */
    uint32_t device;         /* CUDA device ordinal */
    uint32_t lanes_per_cta;  /* 0 or 32: one 32-lane tile per CTA (the only width) */
    uint32_t refine_sweeps;  /* ESPL_MIXED: FP64-residual refinement sweeps after
                              * each FP32 solve inside Newton (0: none; each Newton
                              * iteration then refines the step against the FP64
                              * KCL residual). At most 4. */
    uint32_t polish;         /* 0: Newton publishes the iterate whose step passes
                              * the reference's test (converger.zig: |dx| <
                              * reltol |x| + vntol or abstol), as the reference does.
                              * k in 1..ESPL_POLISH_MAX_DIGITS: after that test
                              * passes, the lane keeps iterating (at most 4 more
                              * Newton iterations) until its step also passes the
                              * test with every tolerance scaled by 10^-k, and
                              * publishes that iterate. The converged point then
                              * no longer depends on where Newton started (a
                              * predicted start, a learned one, FP32 factors) to
                              * well below the Newton tolerance. Every Newton
                              * solve of the handle (operating points, the ladder,
                              * transient steps) polishes; iteration counts
                              * include the polish. */
} espl_create_opts;
#define ESPL_POLISH_MAX_DIGITS 12u

typedef struct espl_lanes espl_lanes;

uint32_t espl_abi_version(void);

/* `GpuLanes.init` / `initStatic` (lanes.zig:610, 1080) over `n_nets`
 * templates at once: each template gets its pivot tape from its lane 0
 * (`ownTape`, lanes.zig:590-603: the lead lane's matrix at x = 0, factored
 * on the host with threshold pivoting on the BTF/AMD order), and all lanes of
 * all templates run in the same launches (a lane -> tape table). For a
 * transient, `dt0` > 0 builds the tape from G + C / dt0 as `ownTape` does. */
espl_status espl_create(const espl_netlist *nets, uint32_t n_nets, const espl_create_opts *opts,
                        double dt0, espl_lanes **out);

/* `GpuLanes.deinit` (lanes.zig:1004). NULL is a no-op. */
espl_status espl_destroy(espl_lanes *h);

/* The pivot tape of template `net` (`LaneTab` + index buffer,
 * src/solver/kernels/lane.zig:17-44, buildTab :778-802), copied out:
 * q, pinv (n each), lp, up (n + 1 each), li (nnz_l), ui (nnz_u), flags (n;
 * bit 0 void, bit 1 scaled pivot). A NULL array is skipped. */
espl_status espl_tape_info(espl_lanes *h, uint32_t net, uint32_t *n, uint32_t *nnz_l, uint32_t *nnz_u);
espl_status espl_copy_tape(espl_lanes *h, uint32_t net, uint32_t *q, uint32_t *pinv, uint32_t *lp,
                           uint32_t *li, uint32_t *up, uint32_t *ui, uint32_t *flags);

/* Lane start states, point-major: x[l * n + i] for the lanes of template
 * `net` (`GpuLanes.reload` / put_x, lanes.zig:1127). cold = 1 also seeds the
 * junction limiters as `op.coldStart` does (src/analysis/dc/op.zig:28-33;
 * MOS1 vgs = vto, vds = 0, vbs = -1). */
espl_status espl_put_x(espl_lanes *h, uint32_t net, const double *x, uint32_t cold);
espl_status espl_get_x(espl_lanes *h, uint32_t net, double *x);

/* `GpuLanes.solveStatic` (lanes.zig:1171): one device Newton per lane from
 * its current x, the operating point's plain rung. out[] holds every lane
 * of every template, template-major. */
espl_status espl_solve_static(espl_lanes *h, const espl_newton_opts *opts, espl_lane_newton *out);

/* The operating point of every lane with the reference's continuation ladder
 * (`op.solve` -> solveLadder / afterPlain, src/analysis/dc/op.zig:111-330):
 * the plain rung from the cold start (x = 0, MODEINITJCT seeds), and for a
 * lane that fails it the dynamic gmin descent (gmin from 1e-3 toward 1e-12 at
 * ngspice's diagonal-gmin places, the step factor adapting to the Newton
 * count, backing off on failures, a stall exit), a clean solve without gmin,
 * then source stepping (an adaptive source scale from 0 to 1, with the
 * sources-off gmin start) and a final full-source solve. The JFNK and OPtran
 * rungs are not built: a lane that fails the final solve reports not
 * converged. Each lane runs its own ladder; the lanes still on it solve
 * together, one launch per ladder solve. iterations sums every rung's Newton
 * iterations (saturating at 65535). Uses opts' tolerances; gmin and init_fix
 * are the ladder's. */
espl_status espl_solve_op(espl_lanes *h, const espl_newton_opts *opts, espl_lane_newton *out);

/* Small-signal AC lanes (the reference's frequency-domain lanes,
 * src/solver/lane/clu.zig over src/analysis/gpu/freq.zig): every lane of
 * template `net` linearized at its current x (an operating point: call after
 * espl_solve_op or espl_solve_static), driven by a unit AC voltage on its
 * voltage source number `vsrc` (in the order of the template's ESPL_VSRC
 * batches), solved at the angular frequencies omega[n_freq]:
 * (G + j omega C) x = e. The complex values replay a real pivot tape chosen
 * on the host from the lead lane's |G| + omega_c |C| at the geometric centre
 * frequency; a lane and frequency whose pivot fails the check (max(|re|,
 * |im|) of the pivot against 1e-12 of its column) reports NaN. Out:
 * out_re/out_im[lane][freq][k] = x(omega)[rows[k]]. Leaves the lanes' limiter
 * state seeded at x. */
espl_status espl_ac(espl_lanes *h, uint32_t net, uint32_t vsrc, const double *omega, uint32_t n_freq,
                    const uint32_t *rows, uint32_t n_rows, double *out_re, double *out_im);
/* The same lanes and tape for any right-hand sides: rhs_re/rhs_im[e][n]
 * (n_rhs of them, the same on every lane), solved as (G + j omega C) x = b,
 * or with adjoint = 1 as the transpose (G + j omega C)^T z = b (the adjoint
 * solves of noise analysis: z[u] is the transfer from a current injected at
 * unknown u to the output b selects). Out: out_re/out_im[lane][freq][e][k]
 * = the solution's unknown rows[k]. espl_ac is this with b = the source's
 * branch row. */
espl_status espl_ac_solve(espl_lanes *h, uint32_t net, const double *omega, uint32_t n_freq, const double *rhs_re,
                          const double *rhs_im, uint32_t n_rhs, uint32_t adjoint, const uint32_t *rows,
                          uint32_t n_rows, double *out_re, double *out_im);

/* The white noise current densities (A^2/Hz) of every lane's noise
 * sources at its current x (an operating point), as the reference's device
 * models declare them at 27 C: resistors 4kT/R between their terminals,
 * diodes 2q|Id| (junction current, gmin shunt excluded) from anode to
 * cathode, level-1 MOS channel thermal noise 4kT (2/3)|gm| from drain to
 * source (flicker noise zero: KF = 0). Sources are the template's
 * resistors, then its diodes, then its MOS, in batch order; *n_src receives
 * their count, and psd (when not NULL) [lanes][n_src] the densities. With
 * espl_ac_solve's adjoint solve of the output row, the output noise is
 * sum_s psd[s] |z[a_s] - z[b_s]|^2. Leaves the limiter state seeded at x. */
espl_status espl_noise_sources(espl_lanes *h, uint32_t net, double *psd, uint32_t *n_src);

/* Transient lanes with device step control (`initSteps` lanes.zig:1827,
 * `deviceLaunch` :1917; the step machine `stepBegin/stepEndA/stepEndB`,
 * src/solver/kernels/lane.zig:505-700). */
typedef struct {
    double t_stop;
    double dt;        /* first (and, when fixed_step, every) step */
    double dt_min;
    double dt_max;
    double reltol, abstol, chgtol, trtol, vntol, residual_tol;
    uint32_t method;     /* 0 BE, 1 trapezoidal, 2 gear-2 (variable-step BDF2); order 1 (BE) first, then 2 */
    uint32_t fixed_step; /* 1: no LTE control, every step dt */
    uint32_t max_iter;   /* Newton iterations per step (ITL4-like) */
    uint32_t max_steps;
    uint32_t predictor;  /* 0 none (x_prev), 1 linear (SPICE xfact), 2 learned */
    uint32_t polish_chord; /* with espl_create_opts.polish: 1 lets a lane's polish
                            * iterations (those after its step passed the
                            * reference's test) reuse the factor of its previous
                            * iteration (a chord step: the residual is fresh, the
                            * LU replay is skipped) where the tile keeps its factor
                            * in shared memory; 0 refactors every iteration */
} espl_tran_opts;

/* `StepReport` (src/solver/kernels/lane.zig:441-451) per lane, with this
 * build's counters. status: 0 stepping, 1 done, 2 dt underflow, 3 parked
 * (a gate handed the lane back to the host: it keeps its state and steps no
 * further until espl_resume_lanes), 4 stopped. event: the lane's last
 * attempt in the launch, 0 idle (none), 1 attempt (under way), 2 accepted,
 * 3 rejected. */
typedef struct {
    double t;              /* the lane's time: the last accepted step's */
    double dt;             /* the next step */
    uint64_t attempts;
    uint64_t nr_iters;
    uint32_t steps;
    uint32_t rejects;
    uint32_t status;
    uint32_t learned_retries; /* attempts from a learned start (predictor 2) that did not
                               * converge and were retried from the linear predictor */
    double t_new;          /* the last attempt's candidate time t + attempted_dt */
    double attempted_dt;   /* the last attempt's step */
    uint32_t event;
    uint32_t reserved;
} espl_step_report;

espl_status espl_init_steps(espl_lanes *h, const espl_tran_opts *opts);

/* Runs up to `max_steps` accepted steps per lane (or to t_stop), all on the
 * device, then fills reports[] for every lane, template-major. */
espl_status espl_device_launch(espl_lanes *h, uint32_t max_steps, espl_step_report *reports);

/* Device-side oscillation-period measure (`arp_lane_meas`,
 * src/solver/lane_device.zig:45-72, restricted to a period pass): the mean
 * spacing of rising crossings of `level` by unknown `row` after `t_start`,
 * over crossings 1..k. Set before espl_init_steps; read after the run. */
espl_status espl_set_period_meas(espl_lanes *h, uint32_t net, uint32_t row, double level, double t_start);
espl_status espl_get_period_meas(espl_lanes *h, uint32_t net, double *period, uint32_t *crossings);

/* Streaming .meas passes over each lane's transient, on the device: every
 * pass reads unknown `row` at t = 0 (the operating point) and at every
 * accepted step, with ngspice's measure semantics as the reference streams
 * them on its lanes (src/output/scan.zig Cross, At, Extremum, Integ, Find;
 * run per lane from src/solver/lane_device.zig). Kinds:
 *   WHEN     the time `row` crosses `val` (after `td`, inside [from, to]):
 *            the `rise`-th rising, `fall`-th falling or `cross`-th crossing
 *            (ESPL_MEAS_LAST: the last one; all ESPL_MEAS_UNSET: the first);
 *            with `level_row` = 1 + u, the time `row` crosses unknown u
 *            (WHEN v(a)=v(b))
 *   FIND_AT  the value at time `at` (linear between steps); DERIV_AT the
 *            slope of the step holding `at`
 *   FIND_WHEN, DERIV_WHEN
 *            the value or slope of `row` at the event of the pass before
 *            it, which must be a WHEN pass (FIND v(x) WHEN v(y)=..., the
 *            pass's own `at` is ignored); `at` reads the event time. If
 *            that WHEN resolves only at the end of the run (LAST with no
 *            `to`), the value is NaN
 *   TARG     the TARG of a TRIG/TARG pair: the previous pass is the TRIG
 *            (a WHEN pass); this pass counts its own crossing (val or
 *            level_row, rise/fall/cross, from/to; its `td` is replaced by
 *            the TRIG event time) from the TRIG event on; value = TARG
 *            time - TRIG time, `at` = the TARG time
 *   MIN/MAX  the extremum over [from, to] (to = 0: to the end), `at` where
 *   AVG      the trapezoidal average over [from, to]
 *   INTEG    the integral over [from, to] (Simpson 3/8, Simpson, trapezoid
 *            panels as ngspice chooses them); RMS its root-mean-square
 * PP is the difference of MAX and MIN.
 * Set before espl_init_steps (at most ESPL_MEAS_MAX_PASSES per template);
 * read after the run: value and at are [lanes][n], NaN where a pass saw no
 * result. */
enum {
    ESPL_MEAS_WHEN = 1, ESPL_MEAS_FIND_AT = 2, ESPL_MEAS_MIN = 3, ESPL_MEAS_MAX = 4, ESPL_MEAS_AVG = 5,
    ESPL_MEAS_INTEG = 6, ESPL_MEAS_RMS = 7, ESPL_MEAS_DERIV_AT = 8, ESPL_MEAS_FIND_WHEN = 9,
    ESPL_MEAS_DERIV_WHEN = 10, ESPL_MEAS_TARG = 11
};
#define ESPL_MEAS_UNSET (-1)
#define ESPL_MEAS_LAST (-2)
#define ESPL_MEAS_MAX_PASSES 16u
typedef struct {
    uint32_t kind;
    uint32_t row;
    double val;                  /* WHEN: the level */
    double td;                   /* WHEN: samples before td are skipped */
    double from, to;             /* the window; to = 0 leaves it open */
    double at;                   /* FIND_AT: the time */
    int32_t rise, fall, cross;   /* WHEN: the event's count, ESPL_MEAS_UNSET or ESPL_MEAS_LAST */
    uint32_t level_row;          /* WHEN, TARG: 0 = the level is `val`; 1 + u = unknown u */
} espl_meas;
espl_status espl_set_meas(espl_lanes *h, uint32_t net, const espl_meas *passes, uint32_t n);
espl_status espl_get_meas(espl_lanes *h, uint32_t net, double *value, double *at);
/* The same passes over a table on the host, for measures of results the
 * host already holds (an AC sweep's magnitudes, a DC sweep): sample k has
 * scale x[k] and columns cols[k * n_cols + u]; a pass reads column `row`
 * (and level column level_row - 1). value/at are [n_passes]. */
espl_status espl_meas_table(const espl_meas *passes, uint32_t n_passes, const double *x, const double *cols,
                            uint32_t n_cols, uint32_t n, double *value, double *at);
/* done[lane][pass] = 1 where a pass has read its last sample (its result
 * can no longer change), between launches. */
espl_status espl_meas_done(espl_lanes *h, uint32_t net, uint8_t *done);
/* Stops every lane l of template `net` with stop[l] != 0 that is still
 * stepping before the next espl_device_launch (its report then says 4,
 * stopped); lanes already done keep their status (the reference's
 * GpuLanes.requestStop, src/analysis/gpu/lanes.zig:2059-2064). With
 * espl_meas_done this ends a lane's transient once its measures resolve. */
espl_status espl_request_stop(espl_lanes *h, uint32_t net, const uint8_t *stop);
/* Resumes every parked lane l of template `net` with resume[l] != 0 (status
 * 3 -> 0): its next launch attempts again the step it was handed back at
 * (the reference's host takes the parked step itself and re-arms the lane;
 * here the lane resumes on the device). Other lanes are left as they are. */
espl_status espl_resume_lanes(espl_lanes *h, uint32_t net, const uint8_t *resume);

/* Timing of the last solve/launch, milliseconds of device time per kernel
 * family (CUDA events on the launching stream), for roofline reporting. */
typedef struct {
    double total_ms;
    double newton_ms;
    uint64_t launches;
    uint64_t lane_iterations;
    uint64_t lane_steps;
    uint32_t dense_peels;     /* dense re-pivoting solves of failed replays, since the last reset */
    uint32_t retapes;         /* tapes rebuilt from a failing lane since create: after a solve or a
                               * launch in which, in some Newton iteration, at least half of a
                               * tile's active lanes failed the replay (the reference's stale-tape
                               * retape, lanes.zig:1573-1591,1700-1752, per tile here) */
} espl_stats;
espl_status espl_get_stats(espl_lanes *h, espl_stats *out);

/* The launch classes of the current plan, in launch order: templates
 * grouped by tile width and resident tiles per SM, one kernel launch per
 * class, each class on a stream of its own when there are several. With
 * each, the device time of its kernel in the last solve or device launch
 * (CUDA events around the launch on its stream; 0 before the first). At
 * most `cap` are written; `count` gets how many there are. The per-launch
 * counterpart of the reference driver's per-round phase split
 * (ESPICE_GPU_STATS, src/analysis/gpu/lanes.zig:372-413). */
typedef struct {
    uint32_t tiles;       /* 32-lane tiles in the class */
    uint32_t wide;        /* 1: 16-warp tiles, 0: 4-warp tiles */
    uint32_t per_sm;      /* resident tiles per SM */
    uint32_t smem_bytes;  /* dynamic shared memory per tile */
    double last_ms;       /* device time of the class's last kernel */
} espl_class_info;
espl_status espl_get_classes(espl_lanes *h, espl_class_info *out, uint32_t cap, uint32_t *count);

/* ---- The launch plan and its autotuner ----
 *
 * How a template's lanes run: in tiles of 4 warps (narrow) or 16 (wide),
 * with what staged in the tile's shared memory, and how many tiles share an
 * SM. espl_create picks these per template from the CUDA occupancy
 * calculator and a makespan rule (the automatic plan; the counterpart of
 * the reference driver's fixed lane-layout choice, src/analysis/gpu/
 * lanes.zig:92-98); espl_set_plan overrides them, and espl_autotune searches
 * them by timing short transients. No reference counterpart for the search. */
enum { ESPL_TILE_AUTO = 0, ESPL_TILE_NARROW = 1, ESPL_TILE_WIDE = 2 };
enum {
    ESPL_STAGE_AUTO = 0,
    ESPL_STAGE_LU = 1,                 /* index words, LU chain and its 16-byte records */
    ESPL_STAGE_LU_GLOBAL_RECORDS = 2,  /* index words and LU chain; records read from global memory */
    ESPL_STAGE_INDEX = 3,              /* the template's index words only */
    ESPL_STAGE_NONE = 4                /* nothing staged */
};
typedef struct {
    uint32_t tile;    /* ESPL_TILE_*; templates whose LU needs wide tiles (the
                       * banded replay, the CTA-wide LU) stay wide */
    uint32_t stage;   /* ESPL_STAGE_*; a choice that does not fit the shared
                       * memory falls back to the automatic order */
    uint32_t per_sm;  /* 0: as many resident tiles per SM as fit; k: at most k
                       * (the tile's shared memory grows to keep it so) */
    uint32_t pad;
} espl_plan_choice;

/* Re-plans the launches with one choice per template (n_nets entries; NULL:
 * all automatic). Lanes' state is kept. */
espl_status espl_set_plan(espl_lanes *h, const espl_plan_choice *choices);
/* The plan in effect, one entry per template, every field resolved (no AUTO
 * values; per_sm the resident tiles per SM of its launch class). */
espl_status espl_get_plan(espl_lanes *h, espl_plan_choice *resolved);

typedef struct {
    uint32_t trials;  /* transients timed */
    uint32_t cached;  /* 1: the plan came from the process's cache, no trial ran */
    double auto_ms;   /* the automatic plan's trial time, milliseconds */
    double best_ms;   /* the returned plan's */
} espl_tune_report;

/* Searches the launch plan of templates `nets` for the transient `tran`:
 * from the automatic plan, moves that change one launch class's templates at
 * a time (records staged or read from global memory, narrow or wide tiles,
 * one resident tile per SM fewer) are each timed on a scratch handle
 * created with `opts` and `dt0` (the operating point, then `trial_steps`
 * transient attempts of every lane; the device time of that launch), and a
 * move is kept when two timings of it (the second taken when the first is
 * at least 3 % faster) are both at least 2 % faster; at most `max_trials`
 * transients (the automatic plan's two runs included: the first warms the
 * process up). `choices` (n_nets entries) gets the best plan for
 * espl_set_plan. The result is cached for the process by the templates'
 * patterns, lane counts and device kinds, the device and the options: a
 * second call with the same inputs runs nothing. ESPL_NO_IMAGE without
 * such a device, as espl_create. A learned predictor
 * (tran->predictor 2) is timed as the linear one. */
espl_status espl_autotune(const espl_netlist *nets, uint32_t n_nets, const espl_create_opts *opts, double dt0,
                          const espl_tran_opts *tran, uint32_t trial_steps, uint32_t max_trials,
                          espl_plan_choice *choices, espl_tune_report *report);

/* Host-only symbolic seam, no GPU needed. `espl_order` is order.zig's
 * `order` (src/solver/order.zig:78): q[k] = the column factored at step k,
 * BTF sink block first, AMD or natural per block. ESPL_NO_TAPE on
 * OutOfWorkspace. */
espl_status espl_order(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q);

/* The lead lane's factor as `ownTape` runs it (lanes.zig:590-603):
 * SparseLu.factor with threshold pivoting on order q and the fill caps of
 * direct.Solver (src/solver/sparse_lu.zig:274-311, direct.zig:310-388),
 * frozen as a tape (kernels/lane.zig buildTab :778-802). ESPL_NO_TAPE when
 * the matrix is singular. Free with espl_tape_free. */
typedef struct espl_tape espl_tape;
espl_status espl_tape_build(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, const double *vals,
                            const uint32_t *q, espl_tape **out);
espl_status espl_tape_sizes(const espl_tape *t, uint32_t *nnz_l, uint32_t *nnz_u, uint32_t *n_void_slots);
/* Copies q, pinv (n), lp, up (n + 1), li (nnz_l), ui (nnz_u), flags (n),
 * prow (nnz), void_slots, and the lead lane's lx, ux, udiag. NULL skips. */
espl_status espl_tape_copy(const espl_tape *t, uint32_t *q, uint32_t *pinv, uint32_t *lp, uint32_t *li, uint32_t *up,
                           uint32_t *ui, uint32_t *flags, uint32_t *prow, uint32_t *void_slots, double *lx,
                           double *ux, double *udiag);
void espl_tape_free(espl_tape *t);

/* The last error's text, NUL-terminated (empty when none). */
espl_status espl_error_message(espl_lanes *h, char *buf, size_t cap);

/* No counterpart in the reference. Replays a host-built tape
 * (espl_tape_build) on `lanes` lanes of matrix values already on the
 * device, WITHOUT ALLOCATING: for callers that cannot allocate device memory
 * at the point of the call -- a host that sized all device memory up front,
 * or a framework whose caching allocator must not be bypassed -- and so
 * cannot create a handle. The work vector and the staged tape words live in
 * one file-scope device array of ESPL_REPLAY_SCRATCH_BYTES per device.
 *
 *   col_ptr     host, n + 1: the pattern the tape was built from
 *   vals        device, nnz x lanes, lane-interleaved (slot p of lane l at
 *               p * lanes + l)
 *   lx, ux      device, nnz_l x lanes and nnz_u x lanes, same interleaving
 *   udiag       device, n x lanes
 *   lane_status device, lanes words: 0 the replay holds, 1 a pivot failed
 *               (dead, non-finite, growth 1e-12) or a void slot filled, 2 only
 *               a multiplier past 1 / pivot_tol (kernels/lane.zig:56-125 and
 *               wideMultipliers)
 *   stream      a cudaStream_t, or NULL for the legacy default stream
 *   err         optional, err_cap bytes: the reason of a non-OK status
 *
 * ESPL_TOO_LARGE, with the sizes in `err`, when the tape words plus
 * 8 * n * lanes bytes of work vector exceed ESPL_REPLAY_SCRATCH_BYTES.
 * The results are ready when `stream` reaches the call (the launch is
 * asynchronous; the tape words are copied from host memory first).
 * The work vector must be all-zero on entry: the array starts at zero and
 * every replay leaves it at zero, so it stays so unless a launch of this
 * entry point is aborted. Calls on one device share the array: overlapping
 * calls (other streams, other host threads) race; serialize them. The first
 * call on a device resolves the array's address (cudaGetSymbolAddress, with
 * that device current) and keeps it for the life of the process; make it
 * before any stream capture begins. A device reset (cudaDeviceReset) or the
 * primary context's teardown invalidates that address: do not call this
 * entry point on the device afterwards in the same process. col_ptr must be
 * the pattern the tape was built from (col_ptr[0] = 0, non-decreasing,
 * col_ptr[n] = nnz), else ESPL_INVALID_ARGUMENT. */
#define ESPL_REPLAY_SCRATCH_BYTES (8u << 20)
espl_status espl_tape_replay_noalloc(const espl_tape *t, const uint32_t *col_ptr, const double *vals,
                                     uint32_t lanes, double *lx, double *ux, double *udiag, uint32_t *lane_status,
                                     void *stream, char *err, size_t err_cap);

#ifdef __cplusplus
}
#endif
#endif
