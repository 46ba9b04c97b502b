// Kernels of the lane sweep. One CTA per 32-lane tile of one template
// (kWarps warps, kWideWarps for large templates): the whole Newton solve of an operating point, or up to
// `launch_steps` transient attempts with device step control, in one launch.
// The tile -> template table lets one launch carry templates of different
// sizes. Every loop is bounded by max_iter / launch_steps; no kernel waits on
// another block.
#pragma once

#include <climits>
#include <type_traits>

#include "lane_band.cuh"
#include "lane_levels.cuh"

namespace espl {

// The tiles of one launch: block b runs tile tiles[b] (all tiles in order
// when tiles is null); tile_group maps a tile to its template.
struct TileMap {
    const GroupDev* groups;
    const uint32_t* tile_group;
    const uint32_t* tiles;
    uint32_t n_tiles;
};

// The Newton launches of a large template run each 32-lane tile as
// 32 >> kBigShift parts of kBigLanes lanes.
constexpr uint32_t kBigShift = 4, kBigLanes = 32u >> kBigShift;
constexpr uint32_t kBigWarps = kWideThreads / kBigLanes;  // work shares per lane of a part

// A tile-list entry: the tile in bits 0-23; in bits 24-27 the part of it
// this CTA runs and in bits 28-31 the shift s of the part's width 32 >> s
// (0: the whole tile).
constexpr uint32_t kTileBits = 0x00FFFFFFu;
__host__ __device__ inline uint32_t tile_entry(uint32_t tile, uint32_t part, uint32_t shift) {
    return tile | part << 24 | shift << 28;
}

__device__ __forceinline__ TileCtx tile_ctx(const TileMap& m) {
    TileCtx c;
    const uint32_t e = m.tiles ? m.tiles[blockIdx.x] : blockIdx.x;
    c.tile = e & kTileBits;
    const uint32_t part = (e >> 24) & 15u, shift = e >> 28;
    c.tw = 32u >> shift;
    c.d = &m.groups[m.tile_group[c.tile]];
    c.lane = threadIdx.x % c.tw;
    c.warp = threadIdx.x / c.tw;
    c.nw = blockDim.x / c.tw;
    c.l = (c.tile - c.d->tile0) * 32 + part * c.tw + c.lane;
    c.valid = c.l < c.d->lanes;
    return c;
}

// Per-tile shared state of a Newton solve and a transient attempt.
// Per-lane reductions over the warps go through shared atomics on
// order-free quantities: maxima of non-negative doubles by their bit
// patterns, minima likewise, and OR of flags.
struct TileShared {
    GroupDev gd;  // the tile's template descriptor, index arrays staged
    uint32_t active[32];
    uint32_t bits[32];
    uint32_t restore[32];  // inside a Newton solve; after it, k_tran's recorder sample (reck)
    uint32_t accf[32];
    unsigned long long acc0[32], acc1[32], acc2[32];
    double limit[32];
    double ag0[32], ag1[32], ag2[32], t[32], xfact[32];
    // The ladder's gmin and source scale of a lane live inside a Newton
    // solve (an operating-point rung); a transient's next step size lives
    // from stepEndA to the history advance, after its solve: they share.
    union {
        struct {
            double lgmin[32], lsrc[32];
        };
        double dt_next[32];
    };
    uint32_t method[32], on[32], accept[32], rot[32];  // on: bit 0 the lane attempts a step, bit 1 from xpred
    // the lane's polish iterations so far (kPitMask), and kFactorHeld: its
    // shared-memory factor is its last iteration's and held
    uint32_t pit[32];
};
constexpr uint32_t kPitMask = 0xFFFFu, kFactorHeld = 0x10000u;

constexpr uint32_t kNoRec = 0xFFFFFFFFu;

// Gate flags reduced over warps.
constexpr uint32_t kLimited = 1, kImplausible = 2, kResidualMiss = 4;

// The CTA-wide LU of a large template (lane_levels.cuh) needs, past the
// tile's staged arrays in dynamic shared memory, the refactor's per-lane
// reductions, the lanes' flags and the ring's barriers (a 4 KB header), the
// solves' partial sums (one double per thread) and, with a streaming plan
// (GroupDev stream), the ring's slots (kBigRingBytes).
constexpr uint32_t kBigScratch = 4096 + kWideThreads * 8;
constexpr uint32_t kBigRingOff = 3584;
constexpr uint32_t kBigRingBytes = ring_bytes(kBigLanes);
// The refactor runs while no chunk is staged: its window of work-vector rows
// (lvl_refactor) takes the ring's shared memory.
constexpr uint32_t kRingSpan = kBigRingBytes;
// (lvl_sweep_ring adds a row's hardware warps' sums inside one warp)
static_assert(kWideThreads / 32 * kBigLanes <= 32, "a row's warp sums fit one warp");
// (and gathers a chunk's rows' own values, one row per logical warp)
static_assert(kWideThreads / kBigLanes >= kRingRows, "a chunk's rows fit the logical warps");

template <bool MIXED>
__device__ __forceinline__ unsigned char* big_scratch(const GroupDev& d, unsigned char* dsm) {
    const uint32_t off = (smem_plan(d, d.stage_mode, MIXED).bytes + 15u) & ~15u;
    return dsm + off;
}

struct BigLaneFlags {
    uint32_t use32[32], need[32], ok[32];
};

// One Newton iteration's LU of a large template: each lane refactors when
// its A changed (a linear template's key: the companion coefficient and
// gmin; any other template every iteration) -- in FP32 on a mixed tile
// until the lane falls back to FP64 -- then solves for dx (plus the FP64
// refinement sweeps of a mixed solve). A lane whose replay fails is singular
// (no dense peel past kDensePeelMax unknowns). All threads of the CTA call it.
template <bool MIXED>
__device__ void big_lu(const GroupDev& d, const TileCtx& c, bool act, LaneState* s, TileShared& sh,
                       const NewtonParams& o, double key0, double key1, uint32_t it, unsigned char* scratch,
                       bool& failed) {
    const uint32_t lane = c.lane, warp = c.warp, nw = c.nw, l = c.l, P = d.P;
    LevelShared& ls = *reinterpret_cast<LevelShared*>(scratch);
    BigLaneFlags& bf = *reinterpret_cast<BigLaneFlags*>(scratch + sizeof(LevelShared));
    void* red = scratch + 4096;
    static_assert(sizeof(LevelShared) + sizeof(BigLaneFlags) <= kBigRingOff &&
                      kBigRingOff + sizeof(RingShared) <= 4096,
                  "the scratch header fits 4 KB");
    RingShared* ring = d.stream ? reinterpret_cast<RingShared*>(scratch + kBigRingOff) : nullptr;
    unsigned char* slots = scratch + kBigScratch;
    auto key_ok = [&](uint32_t kb) {
        return d.linear && LM(d.fact_key, kb) == key0 && LM(d.fact_key, kb + 1) == key1;
    };
    if (warp == 0) {
        const bool u32 = MIXED && act && !s->fp64;
        bf.use32[lane] = u32 ? 1u : 0u;
        bf.need[lane] = (act && !key_ok(u32 ? 2u : 0u)) ? 1u : 0u;
        bf.ok[lane] = 1u;
    }
    __syncthreads();
    if (MIXED) {
        const bool go = bf.need[lane] && bf.use32[lane];
        if (__syncthreads_or(go)) {
            const int rc = lvl_refactor<float>(d, l, lane, warp, nw, go, d.w32, d.wk32, d.lx32, d.ux32, d.udiag32, ls,
                                               d.stream ? reinterpret_cast<float*>(slots) : nullptr,
                                               kRingSpan / (kBigLanes * 4u));
            if (warp == 0 && go) {
                if (rc != 0) {
                    // the FP32 factor fails: this lane refactors in FP64 from here on
                    s->fp64 = 1;
                    s->fallbacks++;
                    LM(d.fact_key, 2) = NAN;
                    bf.use32[lane] = 0;
                    bf.need[lane] = key_ok(0) ? 0u : 1u;
                } else {
                    LM(d.fact_key, 2) = key0;
                    LM(d.fact_key, 3) = key1;
                }
            }
            if (d.stream)
                lvl_stream_store<float>(d, l, lane, warp, nw, go, d.lx32, d.ux32, d.stream->vf32, d.stream->vb32);
            __syncthreads();
        }
    }
    {
        const bool go = bf.need[lane] && !bf.use32[lane];
        if (__syncthreads_or(go)) {
            const int rc = lvl_refactor<double>(d, l, lane, warp, nw, go, d.w, d.wk, d.lx, d.ux, d.udiag, ls,
                                                d.stream ? reinterpret_cast<double*>(slots) : nullptr,
                                                kRingSpan / (kBigLanes * 8u));
            if (warp == 0 && go) {
                const bool ok = rc == 0 || (rc == 2 && replay_holds64(d, l));
                bf.ok[lane] = ok ? 1u : 0u;
                LM(d.fact_key, 0) = ok ? key0 : NAN;
                LM(d.fact_key, 1) = key1;
            }
            if (d.stream) lvl_stream_store<double>(d, l, lane, warp, nw, go, d.lx, d.ux, d.stream->vf, d.stream->vb);
            __syncthreads();
        }
    }
    if (warp == 0 && act && !bf.ok[lane]) {
        sh.bits[lane] |= kSingular;
        sh.active[lane] = 0;
        s->iterations = it;
    }
    failed = act && !bf.ok[lane];
    const bool solve = act && bf.ok[lane];
    const bool u32 = bf.use32[lane] != 0;
    if (MIXED && __syncthreads_or(solve && u32)) {
        lvl_solve<float>(d, l, lane, warp, nw, solve && u32, d.rhs, d.dx, d.y32, d.lx32, d.ux32, d.udiag32,
                         static_cast<float*>(red), ring, slots, d.stream ? d.stream->vf32 : nullptr,
                         d.stream ? d.stream->vb32 : nullptr);
        for (uint32_t r = 0; r < o.refine; r++)
            lvl_refine(d, l, lane, warp, nw, solve && u32, static_cast<float*>(red), ring, slots);
    }
    if (__syncthreads_or(solve && !u32))
        lvl_solve<double>(d, l, lane, warp, nw, solve && !u32, d.rhs, d.dx, d.y, d.lx, d.ux, d.udiag,
                          static_cast<double*>(red), ring, slots, d.stream ? d.stream->vf : nullptr,
                          d.stream ? d.stream->vb : nullptr);
    if (ring && ring->fail && act) {
        // a staged chunk never arrived: the lane's step is lost
        if (warp == 0) {
            sh.bits[lane] |= kSingular;
            sh.active[lane] = 0;
            s->iterations = it;
        }
        failed = true;
    }
}

// The ring's barriers, once per CTA of a large template with a streaming
// plan, before its first solve.
template <bool MIXED>
__device__ __forceinline__ void big_ring_init(const GroupDev& d) {
    if (d.big && d.stream) ring_init(*reinterpret_cast<RingShared*>(big_scratch<MIXED>(d, g_dsm) + kBigRingOff));
}

// One Newton solve per lane of the tile (converger.newtonLanes at W = 1 as
// the lane kernels split it: assemble, gmin, refactor, solve, update,
// limit, gates, finalize). `on` lanes take part; with `tran_companion` a
// lane's companion scalars and time come from the shared arrays. The
// instance phase of iteration k + 1 runs inside iteration k's limiter pass
// (same loads; the gather has read the cells by then); `eval0` runs
// iteration 0's instance phase first (else the caller left it in the cells).
template <bool MIXED>
__device__ __forceinline__ void newton_tile(const TileCtx& c, LaneState* s, const NewtonParams& o, int tran,
                                            bool tran_companion, bool on, TileShared& sh, unsigned char* dsm,
                                            bool eval0) {
    const GroupDev& d = *c.d;
    const uint32_t l = c.l, P = d.P, lane = c.lane, warp = c.warp, nw = c.nw;
    const uint32_t ninst = n_instances(d);
    using T = typename std::conditional<MIXED, float, double>::type;
    const bool sm = d.stage_mode == kStageLu;
    SmemTile st{};
    if (sm) st = smem_tile(dsm, smem_plan(d, kStageLu, MIXED));
    // a ladder rung's lane: its own gmin (at the gmin stamps), source scale
    // and cold or warm start
    const LadderLane* lad = (o.ladder && c.valid) ? &o.ladder[d.lane0 + l] : nullptr;
    const bool init_fix = lad ? lad->init_fix != 0 : o.init_fix != 0;
    if (warp == 0) {
        sh.active[lane] = (c.valid && on) ? 1u : 0u;
        sh.bits[lane] = (init_fix ? kInitFix : 0u);
        sh.limit[lane] = kXPlausible;
        sh.acc0[lane] = dbits(1.0);
        sh.acc1[lane] = 0;
        sh.acc2[lane] = 0;
        sh.lgmin[lane] = lad ? lad->gmin : 0.0;
        sh.lsrc[lane] = lad ? lad->src : 1.0;
        sh.pit[lane] = 0;
        if (s && on) {
            s->iterations = o.max_iter;
            // Mixed tiles factor in FP32 once Newton contracts (warm starts,
            // transient steps); a cold start (INITFIX, MODEINITJCT seeds)
            // walks through ill-conditioned iterates and runs in FP64.
            s->fp64 = (MIXED && init_fix) ? 1u : 0u;
        }
    }
    // the ladder's source scale (uniform branch: o.ladder is the launch's)
    if (o.ladder) __syncthreads();
    const double src = o.ladder ? sh.lsrc[lane] : 1.0;
    if (eval0 && c.valid && on)
        for (uint32_t t = warp; t < ninst; t += nw) inst_eval(d, l, t, tran, 0.0, cell_buf(d, 0), src);
    __syncthreads();
    for (uint32_t it = 0; it < o.max_iter; it++) {
        bool act = c.valid && sh.active[lane];
        if (!__syncthreads_or(act)) break;
        Companion cp{0, 0, 0.0, 0.0, 0.0};
        double tm = 0.0;
        if (tran_companion) {
            cp.on = 1;
            cp.method = sh.method[lane];
            cp.ag0 = sh.ag0[lane];
            cp.ag1 = sh.ag1[lane];
            cp.ag2 = sh.ag2[lane];
            tm = sh.t[lane];
        }
        const double* cells = d.cells;
        // A linear large template whose lanes' A was assembled for this
        // iteration's companion coefficient and gmin keeps it: the CTA
        // gathers only the right-hand sides.
        bool rhs_only = false;
        if (d.big && d.linear && !o.ladder) {
            const double k0 = cp.on ? cp.ag0 : -1.0;
            rhs_only = __syncthreads_and(!act || (LM(d.fact_key, 4) == k0 && LM(d.fact_key, 5) == o.gmin)) != 0;
        }
        if (act) {
            uint32_t it0, it1;
            if (rhs_only) {
                it0 = d.nnz + (uint32_t)((uint64_t)d.n * warp / nw);
                it1 = d.nnz + (uint32_t)((uint64_t)d.n * (warp + 1) / nw);
            } else if (nw == 4) {
                it0 = d.gsplit4[warp];
                it1 = d.gsplit4[warp + 1];
            } else if (nw == 16) {
                it0 = d.gsplit16[warp];
                it1 = d.gsplit16[warp + 1];
            } else if (nw == kBigWarps) {
                it0 = d.gsplit_big[warp];
                it1 = d.gsplit_big[warp + 1];
            } else {
                it0 = (uint32_t)((uint64_t)d.n_items * warp / nw);
                it1 = (uint32_t)((uint64_t)d.n_items * (warp + 1) / nw);
            }
            gather_items<T>(d, l, lane, it0, it1, cp, o.ladder ? 0.0 : o.gmin, cells,
                            sm ? static_cast<T*>(st.a) : nullptr);
            if (d.big && d.linear && !rhs_only && warp == 0) {
                // (the ladder adds its gmin to A below: no key names that A)
                LM(d.fact_key, 4) = o.ladder ? NAN : (cp.on ? cp.ag0 : -1.0);
                LM(d.fact_key, 5) = o.gmin;
            }
        }
        __syncthreads();
        if (o.ladder) {
            // the rung's gmin at ngspice's diagonal-gmin places (loadGmin,
            // converger.zig:700-717): A[slot] += gmin, rhs[row] += gmin x[col]
            const double gl = sh.lgmin[lane];
            if (warp == 0 && act && gl > 0.0)
                for (uint32_t k = 0; k < d.n_gstamp; k++) {
                    const uint32_t slot = d.gstamp[3 * k], row = d.gstamp[3 * k + 1], col = d.gstamp[3 * k + 2];
                    const double a = LM(d.a, slot) + gl;
                    LM(d.a, slot) = a;
                    if (sm) static_cast<T*>(st.a)[slot * 32 + lane] = (T)a;
                    LM(d.rhs, row) += gl * LM(d.x, col);
                }
            __syncthreads();
        }
        if (it == 0) {
            // plausibleLimit (kernels/lane.zig:202-214).
            double g = 1.0;
            unsigned long long xm = 0, fm = 0;
            if (act) {
                for (uint32_t i = warp; i < d.n; i += nw) {
                    g = fmax(g, fabs(LM(d.a, d.diag[i])));
                    unsigned long long xb = dbits(fabs(LM(d.x, i))), fb = dbits(fabs(LM(d.rhs, i)));
                    xm = xm > xb ? xm : xb;
                    fm = fm > fb ? fm : fb;
                }
                // g >= 1 and never NaN (fmax drops NaN): its bits order as it does
                atomicMax(&sh.acc0[lane], dbits(g));
                atomicMax(&sh.acc1[lane], xm);
                atomicMax(&sh.acc2[lane], fm);
            }
            __syncthreads();
            if (warp == 0 && act) {
                g = bitsd(sh.acc0[lane]);
                xm = sh.acc1[lane];
                fm = sh.acc2[lane];
                double scale = fmin(fmax(bitsd(xm), bitsd(fm) * g), 1e18);
                if (isnan(bitsd(xm)) || isnan(bitsd(fm))) scale = NAN;
                sh.limit[lane] = !(1e3 * scale > kXPlausible) ? kXPlausible : 1e3 * scale;
            }
        }
        // The LU chain: warp 0, one thread per lane; in shared memory when the
        // template fits there (FP32 tiles: only the lanes still in FP32).
        if (warp == 0) {
            sh.acc0[lane] = 0;
            sh.accf[lane] = 0;
        }
        bool failed = false;  // the lane's replay failed this iteration (it peels)
        if (d.big) {
            // the whole CTA refactors (when the lane's A changed) and solves
            const double key1 = o.ladder ? sh.lgmin[lane] : o.gmin;
            big_lu<MIXED>(d, c, act, s, sh, o, cp.on ? cp.ag0 : -1.0, key1, it, big_scratch<MIXED>(d, dsm), failed);
        } else {
            // The banded streaming replay (lane_band.cuh) of a template the
            // shared chain cannot hold: every warp takes part; it replays the
            // lanes in the tile's precision (FP32 lanes of a mixed tile, or FP64).
            int band_rc = -1;
            bool band_solved = false;
                if (!sm && d.band_ok) {
                const bool comp = warp == 0 && act && (!MIXED || !s->fp64);
                band_rc = band_refactor<T>(d, warp, lane, l, comp);
                if (!comp) band_rc = -1;
                // lanes whose replay held solve through the streamed blocks too
                band_solved = band_rc == 0;
                band_solve<T>(d, warp, lane, l, band_solved);
            }
            if (warp == 0 && act) {
                bool use32 = MIXED && !s->fp64;
                bool done = band_solved;
                if (band_solved && MIXED)
                    for (uint32_t r = 0; r < o.refine; r++) refine_mixed(d, l);
                if (sm && (use32 || !MIXED)) {
                    // a polish iteration of a chord lane keeps the factor of
                    // its previous iteration (still in shared memory)
                    const bool keep = o.chord && (sh.pit[lane] & kPitMask) > 0 && (sh.pit[lane] & kFactorHeld);
                    int rc = keep ? 0 : d.n_rec ? refactor_rec<T>(d, st, lane, l) : refactor_smem<T>(d, st, lane, l);
                    sh.pit[lane] = (sh.pit[lane] & kPitMask) | (rc == 0 ? kFactorHeld : 0u);
                    if (MIXED && rc != 0) {
                        s->fp64 = 1;
                        s->fallbacks++;
                        use32 = false;
                    } else {
                        if (!MIXED && rc == 2) {
                            spill_factor<T>(d, st, lane, l);
                            rc = replay_holds64(d, l) ? 0 : 1;
                        }
                        if (rc == 0) {
                            if (d.n_srec)
                                solve_rec<T>(d, st, lane, l);
                            else
                                solve_smem<T>(d, st, lane, l);
                            if (MIXED)
                                for (uint32_t r = 0; r < o.refine; r++) refine_smem(d, st, lane, l);
                        } else {
                            failed = true;
                            if (!peel_dense(d, l, *s)) {
                                sh.bits[lane] |= kSingular;
                                sh.active[lane] = 0;
                                s->iterations = it;
                            }
                        }
                        done = true;
                    }
                }
                if (!done) {
                    if (use32 && (band_rc >= 0 ? band_rc != 0 : refactor32(d, l))) {
                        s->fp64 = 1;
                        s->fallbacks++;
                        use32 = false;
                    }
                    bool fail = false;
                    if (!use32) {
                        int rc = (!MIXED && band_rc >= 0) ? band_rc : refactor64(d, l);
                        fail = rc == 1 || (rc == 2 && !replay_holds64(d, l));
                    }
                    if (fail) {
                        failed = true;
                        if (!peel_dense(d, l, *s)) {
                            sh.bits[lane] |= kSingular;
                            sh.active[lane] = 0;
                            s->iterations = it;
                        }
                    } else if (use32) {
                        solve32(d, l, d.rhs, d.dx);
                        for (uint32_t r = 0; r < o.refine; r++) refine_mixed(d, l);
                    } else {
                        solve64(d, l, d.rhs, d.dx);
                    }
                }
            }
        }
        // A stale tape (lanes.zig:1573-1591, per tile and iteration here):
        // when at least half of the tile's active lanes failed the replay,
        // the host rebuilds the template's tape from a failing lane's matrix
        // after the launch.
        if (warp == 0 && d.stale) {
            // the tw lanes of the CTA are threads 0 .. tw-1 of its first warp
            const unsigned mask = c.tw == 32 ? 0xffffffffu : (1u << c.tw) - 1u;
            const unsigned am = __ballot_sync(mask, act), fm = __ballot_sync(mask, act && failed);
            if (lane == 0 && fm && 2u * (unsigned)__popc(fm) >= (unsigned)__popc(am)) {
                atomicOr(&d.stale[0], 1u);
                atomicMin(&d.stale[1], c.l - lane + (uint32_t)(__ffs(fm) - 1));
            }
        }
        __syncthreads();
        act = c.valid && sh.active[lane];
        // updateNorm (kernels/lane.zig:161-179), rows split over warps.
        unsigned long long worst = 0;
        if (act)
            for (uint32_t i = warp; i < d.n; i += nw) {
                double xo = LM(d.x, i), dd = LM(d.dx, i);
                double xn = xo + dd;
                LM(d.x_old, i) = xo;
                LM(d.x, i) = xn;
                double tol = o.reltol * fmax(fabs(xn), fabs(xo)) + (d.cur_row[i] ? o.abstol : o.vntol);
                bool finite = fabs(xn) < INFINITY && fabs(dd) < INFINITY;
                double q = fabs(dd) / tol;
                double score = !finite ? INFINITY : (q == q ? q : 0.0);
                unsigned long long b = dbits(score);
                worst = worst > b ? worst : b;
            }
        // the iteration's site charges, before the limiter pass overwrites
        // the cells (a lane that converges here publishes them)
        if (act)
            for (uint32_t j = warp; j < d.n_sites; j += nw) LM(d.site_prev, j) = LM(d.cells, d.site_cell[j]);
        if (act) atomicMax(&sh.acc0[lane], worst);
        __syncthreads();
        // The limiter pass over instances (each then evaluated at its new
        // limited point for the next iteration); plausible and residual gates
        // over rows.
        uint32_t flags = 0;
        if (act) {
            double* next = d.cells;
            for (uint32_t t = warp; t < ninst; t += nw)
                if (inst_limit_eval(d, l, t, tran, tm, next, src)) flags |= kLimited;
            double lim = sh.limit[lane];
            for (uint32_t i = warp; i < d.n; i += nw) {
                double xi = LM(d.x, i);
                if (!(fabs(xi) <= lim)) flags |= kImplausible;
                const double tol = residual_gate(o.residual_tol, o.reltol, o.vntol, LM(d.a, d.diag[i]), xi);
                if (!(fabs(LM(d.rhs, i)) <= tol)) flags |= kResidualMiss;
            }
        }
        if (flags) atomicOr(&sh.accf[lane], flags);
        __syncthreads();
        if (warp == 0) {
            sh.restore[lane] = 0;
            if (act) {
                unsigned long long wb = sh.acc0[lane];
                uint32_t f = sh.accf[lane];
                double scaled = bitsd(wb);
                bool ok = !(f & kLimited) && it != 0 && !(scaled >= 1.0) && !(f & (kImplausible | kResidualMiss));
                if (ok && (sh.bits[lane] & kInitFix)) {
                    sh.bits[lane] &= ~kInitFix;
                } else if (ok && o.polish > 0.0 && !(scaled < o.polish) && (sh.pit[lane] & kPitMask) < o.polish_max) {
                    // the polish: Newton's test passed but not the tightened
                    // one; the lane goes on from x + dx
                    sh.pit[lane]++;
                } else if (ok) {
                    sh.bits[lane] |= kConverged;
                    sh.active[lane] = 0;
                    sh.restore[lane] = 1;
                    s->iterations = it + 1;
                }
                if (MIXED && sh.active[lane] && !s->fp64 && it + 1 >= o.stall_ticks) {
                    s->fp64 = 1;
                    s->fallbacks++;
                }
            }
        }
        __syncthreads();
        if (c.valid && sh.restore[lane])
            for (uint32_t i = warp; i < d.n; i += nw) LM(d.x, i) = LM(d.x_old, i);
    }
    __syncthreads();
    if (warp == 0 && s && on) s->bits = sh.bits[lane];
}


template <bool MIXED, bool WIDE>
__global__ void __launch_bounds__(WIDE ? kWideThreads : kTileThreads, WIDE ? 1 : 4)
    k_static(TileMap m, NewtonParams o, LaneState* st, int tran) {
    __shared__ TileShared sh;
    TileCtx c = tile_ctx(m);
    c.d = stage_template(*c.d, sh.gd, g_dsm, MIXED);
    big_ring_init<MIXED>(*c.d);
    LaneState* s = (c.warp == 0 && c.valid) ? &st[c.d->lane0 + c.l] : nullptr;
    const bool on = !o.ladder || (c.valid && o.ladder[c.d->lane0 + c.l].on != 0);
    newton_tile<MIXED>(c, s, o, tran, false, on, sh, g_dsm, true);
}

// The ladder's per-lane bookkeeping (action[lane0 + l]): 1 the cold start
// (x = 0 with the MODEINITJCT limiter seeds, op.zig coldStart), 2 back to the
// lane's last converged iterate of the rung (x = x_good, limiter state seeded
// there), 3 keeps the lane's iterate (x_good = x), 4 seeds the limiter
// state at the lane's x (a warm solve from where it is), 0 nothing. Warp 0
// only, one thread per lane (no barrier).
__global__ void __launch_bounds__(kTileThreads) k_ladder_x(TileMap m, const uint8_t* action) {
    TileCtx c = tile_ctx(m);
    if (!c.valid || c.warp != 0) return;
    const GroupDev& d = *c.d;
    const uint32_t P = d.P, l = c.l;
    const uint32_t a = action[d.lane0 + l];
    if (a == 0) return;
    if (a == 3) {
        for (uint32_t i = 0; i <= d.n; i++) LM(d.x_good, i) = LM(d.x, i);
        return;
    }
    if (a != 4)
        for (uint32_t i = 0; i <= d.n; i++) LM(d.x, i) = a == 1 ? 0.0 : LM(d.x_good, i);
    const uint32_t ninst = n_instances(d);
    for (uint32_t t = 0; t < ninst; t++) inst_seed(d, l, t, a == 1 ? 1 : 0, d.x);
}

// Bias-independent prep per (instance, lane) from the raw lane-major rows,
// and the constant cells (+1, -1).
__global__ void __launch_bounds__(kTileThreads) k_prep(TileMap m, const double* const* mos_raw,
                                                       const double* const* dio_raw) {
    TileCtx c = tile_ctx(m);
    const uint32_t nw = c.nw;
    if (!c.valid) return;
    const GroupDev& d = *c.d;
    const uint32_t P = d.P, l = c.l;
    uint32_t g = m.tile_group[c.tile];
    const double* mr = mos_raw[g];
    const double* dr = dio_raw[g];
    double* md = const_cast<double*>(d.mos_d);
    double* dd = const_cast<double*>(d.dio_d);
    for (uint32_t i = c.warp; i < d.n_mos; i += nw) {
        double p[9], o[Mos1Prep::count];
        for (int k = 0; k < 9; k++) p[k] = LM(mr, 9 * i + k);
        mos1_setup(p, o);
        for (int k = 0; k < Mos1Prep::count; k++) LM(md, Mos1Prep::count * i + k) = o[k];
        if (d.mos_uni && l == 0)
            for (uint32_t k = 0; k < kMosUni; k++) const_cast<double*>(d.mos_u)[kMosUni * i + k] = o[mos_uni_field(k)];
    }
    for (uint32_t i = c.warp; i < d.n_dio; i += nw) {
        double p[7], o[DiodePrep::count];
        for (int k = 0; k < 7; k++) p[k] = LM(dr, 7 * i + k);
        diode_setup(p, o);
        for (int k = 0; k < DiodePrep::count; k++) LM(dd, DiodePrep::count * i + k) = o[k];
    }
    if (c.warp == 0) {
        LM(d.cells, d.c_const) = 1.0;
        LM(d.cells, d.c_const + 1) = -1.0;
    }
}

// Limiter states for a cold (MODEINITJCT) or warm start; resets the lane's
// per-solve bookkeeping.
__global__ void __launch_bounds__(kTileThreads) k_seed(TileMap m, int cold, LaneState* st) {
    TileCtx c = tile_ctx(m);
    const uint32_t nw = c.nw;
    if (!c.valid) return;
    const GroupDev& d = *c.d;
    const uint32_t ninst = n_instances(d);
    for (uint32_t t = c.warp; t < ninst; t += nw) inst_seed(d, c.l, t, cold, d.x);
    if (c.warp == 0) {
        LaneState& s = st[d.lane0 + c.l];
        s.fp64 = 0;
        s.fallbacks = 0;
        s.peels = 0;
    }
}

// Every lane stamped at its x: A = G (+ C / dt) for the lead lane's tape
// (ownTape's matrix).
__global__ void __launch_bounds__(kTileThreads) k_assemble(TileMap m, int tran, double inv_dt) {
    TileCtx c = tile_ctx(m);
    const uint32_t nw = c.nw;
    const GroupDev& d = *c.d;
    if (c.valid)
        for (uint32_t t = c.warp; t < n_instances(d); t += nw) inst_eval(d, c.l, t, tran, 0.0, cell_buf(d, 0));
    __syncthreads();
    Companion cp{inv_dt > 0.0 ? 1 : 0, 0, inv_dt, 1.0, 0.0};
    if (c.valid)
        for (uint32_t p = c.warp; p < d.nnz; p += nw) gather_slot(d, c.l, p, cp, 0.0, cell_buf(d, 0));
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

__device__ __forceinline__ double* ring_slot(const GroupDev& d, uint32_t rot, uint32_t logical) {
    return d.sring + (size_t)((rot + logical) & 3) * d.n_sites * d.P;
}

// stepBound (kernels/lane.zig:257-297) over the sites j = j0, j0 + stride,
// ... of a lane, for the integration method m0 and, with `two`, also m1 (the
// trial order of a backward-Euler step), sharing the loads. The minimum
// over the sites is order-free, so warps can split them and take the
// minimum of their parts; a NaN in a site's inputs or bound poisons the
// method's result (bad0, bad1).
__device__ void step_bound_part(const GroupDev& d, uint32_t l, uint32_t rot, uint32_t m0, uint32_t m1, bool two,
                                uint32_t cur_method, double dt, double dt1, double dt2, double reltol, double abstol,
                                double chgtol, double trtol, double ag0, double ag1, double ag2, uint32_t j0,
                                uint32_t stride,
                                double& v0, double& v1, bool& bad0, bool& bad1) {
    const uint32_t P = d.P;
    const uint32_t ns = d.n_sites;
    double c0 = m0 == 0 ? 0.5 : m0 == 1 ? 0.08333333333 : 0.2222222222;
    double c1 = m1 == 0 ? 0.5 : m1 == 1 ? 0.08333333333 : 0.2222222222;
    double sum01 = dt + dt1, sum12 = dt1 + dt2, sum012 = dt + (dt1 + dt2);
    const double *r0 = ring_slot(d, rot, 0), *r1 = ring_slot(d, rot, 1);
    const double *r2 = ring_slot(d, rot, 2), *r3 = ring_slot(d, rot, 3);
    for (uint32_t j = j0; j < ns; j += stride) {
        double qc = LM(r0, j), qp = LM(r1, j), qp2 = LM(r2, j), qp3 = LM(r3, j), i_p = LM(d.sip, j);
        double i_new = cur_method == 1   ? ag0 * (qc - qp) - ag1 * i_p
                       : cur_method == 2 ? ag0 * (qc - qp) - ag2 * (qp - qp2)
                                         : ag0 * (qc - qp);
        double volttol = abstol + reltol * fmax(fabs(i_new), fabs(i_p));
        double chargetol = reltol * fmax(fmax(fabs(qc), fabs(qp)), chgtol) / dt;
        double tol = fmax(volttol, chargetol);
        bool in_bad = isnan((qc - qc) + (qp - qp) + (qp2 - qp2) + (i_p - i_p));
        bool bad3 = isnan(qp3 - qp3);
        double f12 = (qp - qp2) / dt1;
        double dd0 = ((qc - qp) / dt - f12) / sum01;
        double f123 = 0.0;
        if (m0 != 0 || (two && m1 != 0)) f123 = (f12 - (qp2 - qp3) / dt2) / sum12;
        double dd = m0 != 0 ? (dd0 - f123) / sum012 : dd0;
        double del = trtol * tol / fmax(abstol, c0 * fabs(dd));
        bad0 |= in_bad || (m0 != 0 && bad3) || del != del;
        v0 = fmin(v0, del);
        if (two) {
            double dd1 = m1 != 0 ? (dd0 - f123) / sum012 : dd0;
            double del1 = trtol * tol / fmax(abstol, c1 * fabs(dd1));
            bad1 |= in_bad || (m1 != 0 && bad3) || del1 != del1;
            v1 = fmin(v1, del1);
        }
    }
}

// Feeds lane l's sample at time t to every .meas pass of its template, in
// order (a pass that reads the one before it sees it after this sample).
__device__ __forceinline__ void meas_feed_all(const GroupDev& d, uint32_t l, double t) {
    const uint32_t P = d.P;
    for (uint32_t p = 0; p < d.n_mpass; p++) {
        const espl_meas& c = d.mpass[p];
        double* ms = d.mstate + (size_t)p * kMeasWords * P + l;
        const double* prev = p > 0 ? ms - (size_t)kMeasWords * P : nullptr;
        meas_feed(c, ms, P, prev, t, LM(d.x, c.row), c.level_row ? LM(d.x, c.level_row - 1) : 0.0);
    }
}

// Transient start from the operating point in x: histories, the site ring,
// the first step (tran.zig:688-699 under LTE control), breakpoints.
__global__ void __launch_bounds__(kTileThreads) k_tran_init(TileMap m, TranParams o, LaneState* st) {
    TileCtx c = tile_ctx(m);
    const uint32_t nw = c.nw;
    const GroupDev& d = *c.d;
    const uint32_t P = d.P, l = c.l;
    const uint32_t ninst = n_instances(d);
    if (c.valid)
        for (uint32_t t = c.warp; t < ninst; t += nw) {
            inst_seed(d, l, t, 0, d.x);
            inst_eval(d, l, t, 1, 0.0, cell_buf(d, 0));
        }
    __syncthreads();
    if (!c.valid) return;
    for (uint32_t i = c.warp; i < d.n; i += nw) {
        gather_charge_row(d, l, i, cell_buf(d, 0));
        LM(d.cur, i) = LM(d.x, i);
        LM(d.prev, i) = LM(d.x, i);
        if (d.prev2) LM(d.prev2, i) = LM(d.x, i);
        LM(d.q1, i) = LM(d.qrow, i);
        LM(d.q2, i) = LM(d.qrow, i);
        LM(d.ip, i) = 0.0;
    }
    for (uint32_t j = c.warp; j < d.n_sites; j += nw) {
        double q = LM(cell_buf(d, 0), d.site_cell[j]);
        for (uint32_t k = 0; k < 4; k++) LM(d.sring + (size_t)k * d.n_sites * P, j) = q;
        LM(d.sip, j) = 0.0;
    }
    if (c.warp != 0) return;
    LaneState& s = st[d.lane0 + l];
    s.s_rot = 0;
    s.t = 0.0;
    double dt;
    if (o.fixed_step) {
        dt = o.dt;
        s.dt_old0 = s.dt_old1 = o.dt;
    } else {
        dt = fmin(fmin(o.dt, o.t_stop / 100.0) / 10.0, o.dt_max);
        double bp0 = next_bp(d, l, 0.0);
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
    s.bp_next = o.fixed_step ? INFINITY : next_bp(d, l, 0.0);
    s.bp_save_dt = 0.0;
    s.bp_clamped = 0;
    s.m_cross = 0;
    s.m_have = 0;
    s.m_first = s.m_last = NAN;
    s.fp64 = 0;
    s.peels = 0;
    s.pred_lin = 0;
    s.pred_fallbacks = 0;
    s.event = kEventIdle;
    s.t_new = 0.0;
    s.attempted_dt = 0.0;
    // the .meas passes start, reading the operating point at t = 0
    for (uint32_t p = 0; p < d.n_mpass; p++) {
        double* ms = d.mstate + (size_t)p * kMeasWords * P + l;
        meas_init(d.mpass[p], ms, P);
    }
    meas_feed_all(d, l, 0.0);
}

// Up to o.launch_steps attempts per lane, each: stepBegin, the linear
// predictor, the limiter pass, Newton with the companion rows, stepEndA
// (Newton and LTE rejections, order promotion), the accepted-step history
// advance, stepEndB (breakpoints, next dt) and the period measure.
template <bool MIXED, bool WIDE>
__global__ void __launch_bounds__(WIDE ? kWideThreads : kTileThreads, WIDE ? 1 : 4)
    k_tran(TileMap m, TranParams o, NewtonParams no, LaneState* st) {
    __shared__ TileShared sh;
    TileCtx c = tile_ctx(m);
    c.d = stage_template(*c.d, sh.gd, g_dsm, MIXED);
    big_ring_init<MIXED>(*c.d);
    const GroupDev& d = *c.d;
    const uint32_t P = d.P, l = c.l, lane = c.lane, warp = c.warp, nw = c.nw;
    const uint32_t ns = d.n_sites, ninst = n_instances(d);
    LaneState* s = (warp == 0 && c.valid) ? &st[d.lane0 + l] : nullptr;
    unsigned char* dsm = g_dsm;
    NewtonParams np = no;
    np.init_fix = 0;
    np.max_iter = o.max_iter;
    np.chord = o.polish_chord;
    for (uint32_t attempt = 0; attempt < o.launch_steps; attempt++) {
        // stepBegin (kernels/lane.zig:508-545).
        if (warp == 0) {
            uint32_t on = 0, lrn = 0;
            if (s) s->event = kEventIdle;
            if (s && s->status == 0) {
                if (!(s->t < o.t_stop && !at_stop(s->t, o.t_stop) && s->steps < o.max_steps)) {
                    s->status = 1;
                } else {
                    on = 1;
                    double dt = s->dt;
                    s->attempted_dt = dt;
                    s->t_new = s->t + dt;
                    s->event = kEventAttempt;
                    uint32_t method = s->order == 1 ? 0 : o.method;
                    sh.method[lane] = method;
                    // integrator.zig coeffs (src/analysis/tran/integrator.zig:39-52)
                    sh.ag2[lane] = 0.0;
                    if (method == 0) {
                        sh.ag0[lane] = 1.0 / dt;
                        sh.ag1[lane] = 1.0;
                    } else if (method == 1) {
                        sh.ag0[lane] = 1.0 / dt / (1.0 - 0.5);
                        sh.ag1[lane] = 0.5 / (1.0 - 0.5);
                    } else {  // gear-2, the variable-step BDF2
                        const double r = dt / s->dt_old0;
                        sh.ag0[lane] = (1.0 + 2.0 * r) / ((1.0 + r) * dt);
                        sh.ag2[lane] = r * r / ((1.0 + r) * dt);
                        sh.ag1[lane] = 1.0;
                    }
                    sh.t[lane] = s->t + dt;
                    sh.xfact[lane] = dt / s->dt_old0;
                    sh.rot[lane] = s->s_rot;
                    s->fp64 = 0;
                    lrn = (o.predictor == 2 && d.xpred && s->steps >= 3 && !s->pred_lin) ? 1u : 0u;
                }
            }
            sh.on[lane] = on | (lrn << 1);
        }
        __syncthreads();
        bool on = c.valid && sh.on[lane];
        if (!__syncthreads_or(on)) break;
        // The predictor: the learned start (k_step_predict wrote it before
        // this attempt), else the linear one (predictor 1, and 2 until the
        // lane has three accepted steps or after a learned start failed),
        // else the last accepted point.
        if (on) {
            double xf = sh.xfact[lane];
            const bool lrn = (sh.on[lane] & 2u) != 0;
            for (uint32_t i = warp; i < d.n; i += nw) {
                double cu = LM(d.cur, i);
                LM(d.x, i) = lrn ? LM(d.xpred, i) : o.predictor != 0 ? cu + xf * (cu - LM(d.prev, i)) : cu;
            }
        }
        __syncthreads();
        // The limiter state restarts from the accepted point, then limits the
        // predicted iterate and evaluates the instances there (the instance
        // phase of Newton's iteration 0, into the cells).
        if (on)
            for (uint32_t t = warp; t < ninst; t += nw) {
                inst_seed(d, l, t, 0, d.cur);
                inst_limit_eval(d, l, t, 1, sh.t[lane], cell_buf(d, 0));
            }
        __syncthreads();
        newton_tile<MIXED>(c, s, np, 1, true, on, sh, dsm, false);
        // The last eval ran at the published x: its site charges are the
        // point's, logical slot 0 of the ring.
        bool conv = on && (sh.bits[lane] & kConverged);
        if (warp == 0) {
            sh.acc1[lane] = dbits(INFINITY);
            sh.acc2[lane] = dbits(INFINITY);
            sh.accf[lane] = 0;
        }
        if (conv) {
            double* r0 = ring_slot(d, sh.rot[lane], 0);
            for (uint32_t j = warp; j < ns; j += nw) LM(r0, j) = LM(d.site_prev, j);
        }
        __syncthreads();
        // The LTE bound of a converged LTE-controlled step, its sites split
        // over the warps (minima in acc1 / acc2, poison bits in accf).
        {
            double v0 = INFINITY, v1 = INFINITY;
            bool b0 = false, b1 = false;
            if (conv && !o.fixed_step && ns > 0) {
                const LaneState& ls = st[d.lane0 + l];
                if (ls.steps > 0) {
                    uint32_t method = sh.method[lane];
                    step_bound_part(d, l, ls.s_rot, method, o.method, method == 0, method, ls.dt, ls.dt_old0,
                                    ls.dt_old1, o.reltol, o.abstol, o.chgtol, o.trtol, sh.ag0[lane], sh.ag1[lane], sh.ag2[lane],
                                    warp, nw, v0, v1, b0, b1);
                }
            }
            // the bounds are >= 0 (NaN ones only poison): their bits order as they do
            if (v0 < INFINITY) atomicMin(&sh.acc1[lane], dbits(v0));
            if (v1 < INFINITY) atomicMin(&sh.acc2[lane], dbits(v1));
            if (b0 || b1) atomicOr(&sh.accf[lane], (b0 ? 1u : 0u) | (b1 ? 2u : 0u));
        }
        __syncthreads();
        // stepEndA (kernels/lane.zig:563-654).
        if (warp == 0) {
            uint32_t acc = 0;
            uint32_t rk = kNoRec;
            if (s && on) {
                double dt = s->dt;
                uint32_t method = sh.method[lane];
                const bool lrn = (sh.on[lane] & 2u) != 0;
                if (!lrn) s->pred_lin = 0;
                s->attempts++;
                if (!(sh.bits[lane] & kSingular)) s->nr_iters += s->iterations < o.max_iter ? s->iterations : o.max_iter;
                if (sh.bits[lane] & kParked) {
                    // a gate that hands the lane back to the host (the
                    // reference's reject_at / $bound_step, kernels/lane.zig
                    // :565-573): the lane stops, its state kept, until the
                    // host resumes it
                    s->status = kStepParked;
                    s->event = kEventIdle;
                } else if (!conv && lrn) {
                    // plain Newton is the fallback: the same step again from
                    // the linear predictor, not a rejected step
                    s->pred_lin = 1;
                    s->pred_fallbacks++;
                } else if (!conv) {
                    s->rejects++;
                    s->order = 1;
                    s->event = kEventReject;
                    if (o.fixed_step) {
                        s->status = 2;
                    } else {
                        double ndt = dt / 8.0;
                        if (ndt < o.dt_min && dt > o.dt_min && s->t + o.dt_min > s->t) ndt = o.dt_min;
                        s->dt = ndt;
                        if (ndt < o.dt_min) s->status = 2;
                    }
                } else {
                    double dt_next = s->steps == 0 ? dt : fmin(dt * 2.0, o.dt_max);
                    bool reject = false;
                    if (o.fixed_step) {
                        dt_next = dt;
                        if (s->order == 1 && o.method != 0) s->order = 2;
                    } else if (ns > 0 && s->steps > 0) {
                        double v0 = bitsd(sh.acc1[lane]), v1 = bitsd(sh.acc2[lane]);
                        uint32_t bad = sh.accf[lane];
                        double del = (bad & 1u) ? NAN : method == 0 ? v0 : sqrt(v0);
                        double del2 = method == 0 ? ((bad & 2u) ? NAN : o.method == 0 ? v1 : sqrt(v1)) : del;
                        if (!(del >= 0.9 * dt)) {
                            reject = true;
                            s->rejects++;
                            s->event = kEventReject;
                            double ndt;
                            if (isnan(del)) { s->order = 1; ndt = dt / 8.0; }
                            else ndt = del;
                            if (ndt < o.dt_min && dt > o.dt_min && s->t + o.dt_min > s->t) ndt = o.dt_min;
                            s->dt = ndt;
                            if (ndt < o.dt_min) s->status = 2;
                        } else {
                            dt_next = fmin(fmin(fmax(del, o.dt_min), 2 * dt), o.dt_max);
                            if (s->order == 1) {
                                double trial = o.method == method ? del : del2;
                                if (!isnan(trial)) {
                                    double nd2 = fmin(2.0 * dt, trial);
                                    if (nd2 > 1.05 * dt) s->order = 2;
                                    dt_next = fmin(fmax(nd2, o.dt_min), o.dt_max);
                                }
                            }
                        }
                    }
                    if (!reject) {
                        acc = 1;
                        s->event = kEventAccept;
                        sh.dt_next[lane] = dt_next;
                        // the step recorder's sample of this accepted step
                        if (d.rec_count && l % d.rec_stride == 0 && s->steps >= d.rec_from && s->steps >= 3) {
                            const uint32_t k = atomicAdd(d.rec_count, 1u);
                            if (k < d.rec_cap) {
                                rk = k;
                                double* tg = d.rec_tag + 5 * (size_t)k;
                                tg[0] = (double)l;
                                tg[1] = (double)s->steps;
                                tg[2] = dt;
                                tg[3] = s->dt_old0;
                                tg[4] = s->dt_old1;
                                d.rec_x[(size_t)k * (3 * d.n + 1) + 3 * d.n] = dt / o.dt_max;
                            }
                        }
                    }
                }
            }
            sh.accept[lane] = acc;
            sh.restore[lane] = rk;
        }
        __syncthreads();
        // Accept (lane_device.zig accept): row histories and companion currents.
        bool acc = c.valid && sh.accept[lane];
        if (acc) {
            double ag0 = sh.ag0[lane], ag1 = sh.ag1[lane], ag2 = sh.ag2[lane];
            uint32_t method = sh.method[lane];
            // a recorded step: its features and target, before the histories shift
            const uint32_t rk = sh.restore[lane];
            double* fx = nullptr;
            double* fy = nullptr;
            double r0 = 0.0, r1 = 0.0;
            if (rk != kNoRec) {
                const LaneState& ls = st[d.lane0 + l];
                fx = d.rec_x + (size_t)rk * (3 * d.n + 1);
                fy = d.rec_y + (size_t)rk * d.n;
                r0 = sh.xfact[lane];
                r1 = ls.dt / ls.dt_old1;
            }
            for (uint32_t i = warp; i < d.n; i += nw) {
                const double q1 = LM(d.q1, i);
                double dq = ag0 * (LM(d.qrow, i) - q1);
                LM(d.ip, i) = method == 1 ? dq - ag1 * LM(d.ip, i) : method == 2 ? dq - ag2 * (q1 - LM(d.q2, i)) : dq;
                LM(d.q2, i) = q1;
                LM(d.q1, i) = LM(d.qrow, i);
                if (d.prev2) {
                    const double cu = LM(d.cur, i), pv = LM(d.prev, i);
                    if (fx) {
                        double f[3];
                        step_features(cu, pv, LM(d.prev2, i), r0, r1, f);
                        fx[i] = f[0];
                        fx[d.n + i] = f[1];
                        fx[2 * d.n + i] = f[2];
                        fy[i] = LM(d.x, i) - (cu + f[1]);
                    }
                    LM(d.prev2, i) = pv;
                }
                LM(d.prev, i) = LM(d.cur, i);
                LM(d.cur, i) = LM(d.x, i);
            }
            const double* q0 = ring_slot(d, sh.rot[lane], 0);
            const double* q1 = ring_slot(d, sh.rot[lane], 1);
            const double* q2 = ring_slot(d, sh.rot[lane], 2);
            for (uint32_t j = warp; j < ns; j += nw) {
                double dq = ag0 * (LM(q0, j) - LM(q1, j));
                LM(d.sip, j) = method == 1   ? dq - ag1 * LM(d.sip, j)
                               : method == 2 ? dq - ag2 * (LM(q1, j) - LM(q2, j))
                                             : dq;
            }
        }
        __syncthreads();
        if (warp == 0 && s && acc) {
            double dt = s->dt;
            double dt_next = sh.dt_next[lane];
            s->s_rot = (s->s_rot + 3) & 3;  // rotate right: new logical k = old k - 1
            s->dt_old1 = s->dt_old0;
            s->dt_old0 = dt;
            double t_new = s->t + dt;
            s->steps++;
            if (d.meas_row != 0xFFFFFFFFu && t_new >= d.meas_t0) {
                double v = LM(d.x, d.meas_row);
                if (s->m_have && s->m_prev_v < d.meas_level && v >= d.meas_level) {
                    double tc = s->m_prev_t + (d.meas_level - s->m_prev_v) * (t_new - s->m_prev_t) / (v - s->m_prev_v);
                    if (s->m_cross == 0) s->m_first = tc;
                    s->m_last = tc;
                    s->m_cross++;
                }
                s->m_prev_v = v;
                s->m_prev_t = t_new;
                s->m_have = 1;
            }
            meas_feed_all(d, l, t_new);
            // stepEndB (kernels/lane.zig:667-700).
            s->t = t_new;
            if (!o.fixed_step) {
                double nb = next_bp(d, l, t_new + o.min_break);
                if (s->bp_next != INFINITY) {
                    double bp = s->bp_next;
                    bool landed = s->bp_clamped ? fabs(t_new - bp) <= o.min_break
                                                : (bp - t_new <= o.delmin || almost_equal_ulps(t_new, bp, 100));
                    if (landed) {
                        s->order = 1;
                        double shrink = s->bp_save_dt;
                        if (nb != INFINITY) shrink = fmin(shrink, nb - t_new);
                        dt_next = fmin(dt_next, 0.1 * shrink);
                    }
                }
                s->bp_next = nb;
                s->bp_clamped = 0;
                if (nb != INFINITY) {
                    double to_bp = nb - t_new;
                    if (to_bp < dt_next) {
                        s->bp_save_dt = dt_next;
                        dt_next = to_bp;
                        s->bp_clamped = 1;
                    }
                }
            }
            s->dt = dt_next;
            if (t_new + s->dt > o.t_stop) s->dt = o.t_stop - t_new;
        }
        __syncthreads();
    }
}

#undef LM

}  // namespace espl
