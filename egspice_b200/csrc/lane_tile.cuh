// The 32-lane tile: a CTA of kWarps warps owns 32 lanes of one template.
// The element-parallel work of a Newton iteration (device evaluation, the
// stamp gather, the update, limiter and gates) is spread over all warps;
// the sequential LU chain runs on warp 0, one thread per lane.
//
// Device evaluation is split in two, the way the reference's GPU sink
// writes per-contribution staging cells and reduces them into the planes
// (src/device/eval.zig LaneSink :3732, hub reduce, lane_device.zig:77-98):
// the instance phase writes each instance's contributions into its own
// cells, then the gather phase sums, per Jacobian slot and per residual or
// charge row, the cells that stamp there, in the order the host stamping
// adds them (Circuit.zig stamp -> eval.zig evalRange), so a slot's sum is
// the reference's sum bit for bit. No atomics, no races between warps.
#pragma once

#include "lane_engine.cuh"

namespace espl {

constexpr int kWarps = 4;
constexpr int kTileThreads = kWarps * 32;
// Tiles of large templates (the banded replay's) run 16 warps: their
// instance, gather and update phases split over four times the threads.
constexpr int kWideWarps = 16;
constexpr int kWideThreads = kWideWarps * 32;
constexpr uint32_t kNeg = 0x80000000u;
// Entries of the flat gather list (GroupDev gi_ent): bit 31 negates, bits
// 28-30 the kind, bits 0-27 a cell, or for a row's q1 / ip / x value the row.
constexpr uint32_t kGiKindShift = 28;
constexpr uint32_t kGiIdx = 0x0fffffffu;
enum : uint32_t { kGiCell = 0, kGiCellC = 1, kGiQ1 = 2, kGiIp = 3, kGiX = 4, kGiNop = 5, kGiQ2 = 6 };
constexpr uint32_t kGiChunk = 12;  // entries whose loads are in flight together

// Cells per instance.
constexpr uint32_t kResCells = 2;   // g, current
constexpr uint32_t kCapCells = 2;   // c, q
constexpr uint32_t kVsrcCells = 2;  // ib, branch residual
constexpr uint32_t kIsrcCells = 1;  // value
constexpr uint32_t kDioCells = 4;   // g, f, c, q
constexpr uint32_t kMosCells = 15;  // fd, fs, fb, jd[4], js[4], jb[4]

// A CTA runs the lanes of one 32-lane tile, or of one part of it: the
// Newton launches of a large template split each tile into 32 / tw parts
// of tw lanes (tile_ctx), so that more SMs share its LU. Thread t works on
// lane t % tw of the part; t / tw ("warp") chooses its share of the
// per-lane work, nw such shares per lane.
struct TileCtx {
    const GroupDev* d;
    uint32_t tile;   // tile index over all templates
    uint32_t l;      // lane in the template
    uint32_t lane;   // 0..tw-1
    uint32_t warp;   // 0..nw-1
    uint32_t nw;     // work shares per lane (blockDim / tw)
    uint32_t tw;     // lanes of the CTA: 32, or a part of a tile
    bool valid;      // l < lanes
};

// ---------------------------------------------------------------------------
// Instance phase: one instance of one kind at the lane's x, its limiter
// state giving the linearization point (eval.zig:826-874).

// Diode i's cells at its terminal voltage vd, linearized at the limited vl.
__device__ __forceinline__ void diode_cells(const GroupDev& d, uint32_t l, uint32_t i, double vd, double vl,
                                            double* __restrict__ cells) {
    const uint32_t P = d.P;
    const double* dd = d.dio_d;
    uint32_t b = DiodePrep::count * i;
    double id, gd, qd, cd;
    diode_core(LM(dd, b + DiodePrep::is), LM(dd, b + DiodePrep::vte), LM(dd, b + DiodePrep::gmin),
               LM(dd, b + DiodePrep::cjo), LM(dd, b + DiodePrep::cjo_t), LM(dd, b + DiodePrep::vj_t),
               LM(dd, b + DiodePrep::mt), LM(dd, b + DiodePrep::fc), LM(dd, b + DiodePrep::tt), vl, id, gd, qd, cd);
    uint32_t c = d.c_dio + kDioCells * i;
    LM(cells, c) = gd;
    LM(cells, c + 1) = id + gd * (vd - vl);
    bool charge = LM(dd, b + DiodePrep::cjo) > 0.0 || LM(dd, b + DiodePrep::tt) > 0.0;
    LM(cells, c + 2) = charge ? cd : 0.0;
    LM(cells, c + 3) = charge ? qd + cd * (vd - vl) : 0.0;
}

// MOS i's cells at its terminal voltages (normalized frame vgs, vds, vbs),
// linearized at the limited (lgs, lds, lbs).
struct MosPrep {
    double ty, vt, beta, lambda, gamma, phit, von0, isat, gmin, vcrit;
};

__device__ __forceinline__ MosPrep mos_prep(const GroupDev& d, uint32_t l, uint32_t i) {
    const uint32_t P = d.P;
    const double* md = d.mos_d;
    uint32_t b = Mos1Prep::count * i;
    if (d.mos_uni) {
        const double* u = d.mos_u + kMosUni * i;
        return MosPrep{__ldg(u + 0), __ldg(u + 1), LM(md, b + Mos1Prep::beta), __ldg(u + 2), __ldg(u + 3),
                       __ldg(u + 4), LM(md, b + Mos1Prep::von0), __ldg(u + 5), __ldg(u + 7), __ldg(u + 6)};
    }
    return MosPrep{LM(md, b + Mos1Prep::type),  LM(md, b + Mos1Prep::vt),    LM(md, b + Mos1Prep::beta),
                   LM(md, b + Mos1Prep::lambda), LM(md, b + Mos1Prep::gamma), LM(md, b + Mos1Prep::phit),
                   LM(md, b + Mos1Prep::von0),   LM(md, b + Mos1Prep::isat),  LM(md, b + Mos1Prep::gmin),
                   LM(md, b + Mos1Prep::vcrit)};
}

__device__ __forceinline__ void mos_cells(const GroupDev& d, uint32_t l, uint32_t i, const MosPrep& m, double vgs,
                                          double vds, double vbs, double lgs, double lds, double lbs,
                                          double* __restrict__ cells) {
    const uint32_t P = d.P;
    const double ty = m.ty;
    Mos1Out o;
    mos1_core(ty, m.vt, m.beta, m.lambda, m.gamma, m.phit, m.von0, m.isat, m.gmin, lgs, lds, lbs, o);
    double dgs = vgs - lgs, dds = vds - lds, dbs = vbs - lbs;
    double gm = o.mode * o.gm, gds = o.mode * o.gds, gmbs = o.mode * o.gmbs;
    double ich = o.mode * o.id + gm * dgs + gds * dds + gmbs * dbs;
    double ibd = o.ibd + o.gbd * (dbs - dds);
    double ibs = o.ibs + o.gbs * dbs;
    double gsum = gm + gds + gmbs;
    uint32_t c = d.c_mos + kMosCells * i;
    LM(cells, c + 0) = ty * ich - ty * ibd;
    LM(cells, c + 1) = -ty * ich - ty * ibs;
    LM(cells, c + 2) = ty * ibd + ty * ibs;
    LM(cells, c + 3) = gds + o.gbd;
    LM(cells, c + 4) = gm;
    LM(cells, c + 5) = -gsum;
    LM(cells, c + 6) = gmbs - o.gbd;
    LM(cells, c + 7) = -gds;
    LM(cells, c + 8) = -gm;
    LM(cells, c + 9) = gsum + o.gbs;
    LM(cells, c + 10) = -gmbs - o.gbs;
    LM(cells, c + 11) = -o.gbd;
    LM(cells, c + 12) = 0.0;
    LM(cells, c + 13) = -o.gbs;
    LM(cells, c + 14) = o.gbd + o.gbs;
}

// `src` scales the independent sources (source stepping; 1 otherwise).
__device__ __forceinline__ void inst_eval(const GroupDev& d, uint32_t l, uint32_t t, int tran, double tm,
                                          double* __restrict__ cells, double src = 1.0) {
    const uint32_t P = d.P;
    const double* __restrict__ x = d.x;
    uint32_t i = t;
    if (i < d.n_res) {
        uint32_t tp = d.res_t[2 * i], tn = d.res_t[2 * i + 1];
        double v = LM(x, tp) - LM(x, tn);
        double r = LM(d.res_r, i);
        uint32_t c = d.c_res + kResCells * i;
        LM(cells, c) = 1.0 / r;
        LM(cells, c + 1) = v / r;
        return;
    }
    i -= d.n_res;
    if (i < d.n_cap) {
        uint32_t tp = d.cap_t[2 * i], tn = d.cap_t[2 * i + 1];
        double v = LM(x, tp) - LM(x, tn);
        double cc = LM(d.cap_c, i);
        uint32_t c = d.c_cap + kCapCells * i;
        LM(cells, c) = cc;
        LM(cells, c + 1) = cc * v;
        return;
    }
    i -= d.n_cap;
    if (i < d.n_vsrc) {
        uint32_t tp = d.vsrc_t[3 * i], tn = d.vsrc_t[3 * i + 1], tb = d.vsrc_t[3 * i + 2];
        const double* pp = d.vsrc_p;
        uint32_t b9 = 9 * i;
        double val = source_value(LM(pp, b9 + 0), LM(pp, b9 + 1), LM(pp, b9 + 2), LM(pp, b9 + 3), LM(pp, b9 + 4),
                                  LM(pp, b9 + 5), LM(pp, b9 + 6), LM(pp, b9 + 7), LM(pp, b9 + 8), tran, tm);
        uint32_t c = d.c_vsrc + kVsrcCells * i;
        LM(cells, c) = LM(x, tb);
        LM(cells, c + 1) = (LM(x, tp) - LM(x, tn)) - val * src;
        return;
    }
    i -= d.n_vsrc;
    if (i < d.n_isrc) {
        const double* pp = d.isrc_p;
        uint32_t b9 = 9 * i;
        LM(cells, d.c_isrc + i) = source_value(LM(pp, b9 + 0), LM(pp, b9 + 1), LM(pp, b9 + 2), LM(pp, b9 + 3),
                                               LM(pp, b9 + 4), LM(pp, b9 + 5), LM(pp, b9 + 6), LM(pp, b9 + 7),
                                               LM(pp, b9 + 8), tran, tm) * src;
        return;
    }
    i -= d.n_isrc;
    if (i < d.n_dio) {
        uint32_t ta = d.dio_t[2 * i], tc = d.dio_t[2 * i + 1];
        diode_cells(d, l, i, LM(x, ta) - LM(x, tc), LM(d.lim_dio, i), cells);
        return;
    }
    i -= d.n_dio;
    if (i < d.n_mos) {
        const uint32_t* tmv = d.mos_t + 4 * i;
        const MosPrep m = mos_prep(d, l, i);
        double xd = LM(x, tmv[0]), xg = LM(x, tmv[1]), xs = LM(x, tmv[2]), xb = LM(x, tmv[3]);
        double vgs = m.ty * (xg - xs), vds = m.ty * (xd - xs), vbs = m.ty * (xb - xs);
        mos_cells(d, l, i, m, vgs, vds, vbs, LM(d.lim_mos, 3 * i), LM(d.lim_mos, 3 * i + 1), LM(d.lim_mos, 3 * i + 2),
                  cells);
        return;
    }
    i -= d.n_mos;
    if (i == 0) LM(cells, d.c_pin) = LM(x, 0);  // the ground pin's residual term
}

__device__ __forceinline__ uint32_t n_instances(const GroupDev& d) {
    return d.n_res + d.n_cap + d.n_vsrc + d.n_isrc + d.n_dio + d.n_mos + 1;
}

// Limiter state of instance t (MOS1 or diode) at the seeds (cold) or at
// the image of `xs` (warm). Other kinds have none.
__device__ __forceinline__ void inst_seed(const GroupDev& d, uint32_t l, uint32_t t, int cold, const double* xs) {
    const uint32_t P = d.P;
    uint32_t base = d.n_res + d.n_cap + d.n_vsrc + d.n_isrc;
    if (t < base) return;
    uint32_t i = t - base;
    if (i < d.n_dio) {
        LM(d.lim_dio, i) = LM(xs, d.dio_t[2 * i]) - LM(xs, d.dio_t[2 * i + 1]);
        return;
    }
    i -= d.n_dio;
    if (i >= d.n_mos) return;
    const uint32_t* tmv = d.mos_t + 4 * i;
    uint32_t b = Mos1Prep::count * i;
    const double* md = d.mos_d;
    if (cold) {
        LM(d.lim_mos, 3 * i) = LM(md, b + Mos1Prep::vgs_seed);
        LM(d.lim_mos, 3 * i + 1) = 0.0;
        LM(d.lim_mos, 3 * i + 2) = -1.0;
    } else {
        double ty = LM(md, b + Mos1Prep::type);
        double xsrc = LM(xs, tmv[2]);
        LM(d.lim_mos, 3 * i) = ty * (LM(xs, tmv[1]) - xsrc);
        LM(d.lim_mos, 3 * i + 1) = ty * (LM(xs, tmv[0]) - xsrc);
        LM(d.lim_mos, 3 * i + 2) = ty * (LM(xs, tmv[3]) - xsrc);
    }
}

// The limiter pass of instance t with snapLimited (eval.zig:1115-1171),
// then the instance evaluated at its new limited point into `cells` (what
// the next Newton iteration's instance phase would compute), on one load of
// the instance's state: true when the limiter clamped.
__device__ __forceinline__ bool inst_limit_eval(const GroupDev& d, uint32_t l, uint32_t t, int tran, double tm,
                                                double* __restrict__ cells, double src = 1.0) {
    const uint32_t P = d.P;
    const double* x = d.x;
    const double eps16 = 16 * 2.220446049250313e-16;
    uint32_t base = d.n_res + d.n_cap + d.n_vsrc + d.n_isrc;
    if (t < base) {
        inst_eval(d, l, t, tran, tm, cells, src);
        return false;
    }
    uint32_t i = t - base;
    if (i < d.n_dio) {
        double xa = LM(x, d.dio_t[2 * i]), xc = LM(x, d.dio_t[2 * i + 1]);
        double vd = xa - xc;
        uint32_t b = DiodePrep::count * i;
        double v = pnjlim(vd, LM(d.lim_dio, i), LM(d.dio_d, b + DiodePrep::vte), LM(d.dio_d, b + DiodePrep::vcrit));
        if (fabs(v - vd) <= eps16 * fmax(fabs(xa), fabs(xc))) v = vd;
        LM(d.lim_dio, i) = v;
        diode_cells(d, l, i, vd, v, cells);
        return v != vd;
    }
    i -= d.n_dio;
    if (i >= d.n_mos) {
        inst_eval(d, l, t, tran, tm, cells, src);
        return false;
    }
    const uint32_t* tmv = d.mos_t + 4 * i;
    const MosPrep m = mos_prep(d, l, i);
    double xd = LM(x, tmv[0]), xg = LM(x, tmv[1]), xs = LM(x, tmv[2]), xb = LM(x, tmv[3]);
    double cgs = m.ty * (xg - xs), cds = m.ty * (xd - xs), cbs = m.ty * (xb - xs);
    double vgs = cgs, vds = cds, vbs = cbs;
    mos1_limit(m.vt, m.gamma, m.phit, m.von0, m.vcrit, LM(d.lim_mos, 3 * i), LM(d.lim_mos, 3 * i + 1),
               LM(d.lim_mos, 3 * i + 2), vgs, vds, vbs);
    double tol = eps16 * fmax(fmax(fabs(xd), fabs(xg)), fmax(fabs(xs), fabs(xb)));
    if (fabs(vgs - cgs) <= tol) vgs = cgs;
    if (fabs(vds - cds) <= tol) vds = cds;
    if (fabs(vbs - cbs) <= tol) vbs = cbs;
    LM(d.lim_mos, 3 * i) = vgs;
    LM(d.lim_mos, 3 * i + 1) = vds;
    LM(d.lim_mos, 3 * i + 2) = vbs;
    mos_cells(d, l, i, m, cgs, cds, cbs, vgs, vds, vbs, cells);
    return (vgs != cgs) | (vds != cds) | (vbs != cbs);
}

__device__ __forceinline__ double gather_sum(const double* __restrict__ cells, uint32_t P, uint32_t l,
                                             const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ list,
                                             uint32_t k) {
    double s = 0.0;
    for (uint32_t e = ptr[k]; e < ptr[k + 1]; e++) {
        uint32_t c = list[e];
        double v = cells[(size_t)(c & ~kNeg) * P + l];
        s += (c & kNeg) ? -v : v;
    }
    return s;
}

// One slot of A = G + ag0 C (gmin on a diagonal) from the per-slot lists
// (the retape's assembly; Newton gathers through gather_items).
__device__ __forceinline__ double slot_value(const GroupDev& d, uint32_t l, uint32_t p, const Companion& cp,
                                             double gmin, const double* __restrict__ cells) {
    const uint32_t P = d.P;
    double g = gather_sum(cells, P, l, d.g_ptr, d.g_cell, p);
    double a = g;
    if (cp.on) {
        double c = gather_sum(cells, P, l, d.c_ptr, d.c_cell, p);
        a = g + cp.ag0 * c;
    }
    if (gmin > 0.0 && d.slot_diag[p]) a += gmin;
    return a;
}

__device__ __forceinline__ double gather_slot(const GroupDev& d, uint32_t l, uint32_t p, const Companion& cp,
                                              double gmin, const double* __restrict__ cells) {
    const uint32_t P = d.P;
    double a = slot_value(d, l, p, cp, gmin, cells);
    LM(d.a, p) = a;
    return a;
}

// The gather of Newton's items it0 .. it1 (slots, then rows) from the flat
// list: per slot A = G + ag0 C (+ gmin on a diagonal), per row the residual
// with its companion and gmin terms and the row charge, term for term in the
// order the host stamping adds them, with the loads of kGiChunk entries in
// flight at a time instead of one sum's.
// Slot values also go to `sa` (the shared LU chain's A) when it is given.
template <typename T>
__device__ __forceinline__ void gather_items(const GroupDev& d, uint32_t l, uint32_t lane, uint32_t it0, uint32_t it1,
                                             const Companion& cp, double gmin, const double* __restrict__ cells,
                                             T* __restrict__ sa) {
    if (it0 >= it1) return;
    const uint32_t P = d.P;
    const uint32_t* __restrict__ ptr = d.gi_ptr;
    const uint32_t* __restrict__ ent = d.gi_ent;
    const uint32_t e_end = ptr[it1];
    uint32_t it = it0, nxt = ptr[it0 + 1];
    double s0 = 0.0, s1 = 0.0, xq1 = 0.0, xip = 0.0, xx = 0.0, xq2 = 0.0;
    for (uint32_t e = ptr[it0]; e < e_end; e += kGiChunk) {
        uint32_t w[kGiChunk];
        double v[kGiChunk];
#pragma unroll
        for (int j = 0; j < (int)kGiChunk; j++) w[j] = e + j < e_end ? ent[e + j] : (kGiNop << kGiKindShift);
#pragma unroll
        for (int j = 0; j < (int)kGiChunk; j++) {
            const uint32_t k = (w[j] >> kGiKindShift) & 7u;
            const double* b = k == kGiQ1 ? d.q1 : k == kGiIp ? d.ip : k == kGiX ? d.x : k == kGiQ2 ? d.q2 : cells;
            v[j] = b[(size_t)(w[j] & kGiIdx) * P + l];
        }
        // every entry is consumed without a branch (padding is a no-op
        // kind past the last item, which no item boundary reaches), so the
        // chunk's loads stay ahead of their uses
#pragma unroll
        for (int j = 0; j < (int)kGiChunk; j++) {
            const uint32_t k = (w[j] >> kGiKindShift) & 7u;
            const double vj = (w[j] & kNeg) ? -v[j] : v[j];
            s0 = k == kGiCell ? s0 + vj : s0;
            s1 = k == kGiCellC ? s1 + vj : s1;
            xq1 = k == kGiQ1 ? vj : xq1;
            xip = k == kGiIp ? vj : xip;
            xx = k == kGiX ? vj : xx;
            xq2 = k == kGiQ2 ? vj : xq2;
            if (e + j + 1 == nxt) {
                if (it < d.nnz) {
                    double a = s0;
                    if (cp.on) a = s0 + cp.ag0 * s1;
                    if (gmin > 0.0 && d.slot_diag[it]) a += gmin;
                    LM(d.a, it) = a;
                    if (sa) sa[it * 32 + lane] = (T)a;
                } else {
                    const uint32_t i = it - d.nnz;
                    double r = s0;
                    if (cp.on) {
                        const double q = s1;
                        LM(d.qrow, i) = q;
                        double dq = cp.ag0 * (q - xq1);
                        double base = r + dq;
                        r = cp.method == 1 ? base - cp.ag1 * xip : cp.method == 2 ? base - cp.ag2 * (xq1 - xq2) : base;
                    }
                    if (gmin > 0.0) r += gmin * xx;
                    LM(d.rhs, i) = r;
                }
                s0 = 0.0;
                s1 = 0.0;
                it++;
                nxt = it < it1 ? ptr[it + 1] : 0xFFFFFFFFu;
            }
        }
    }
}

// Row charges without a Newton (the transient start and the tape's charge
// planes are read from them).
__device__ __forceinline__ void gather_charge_row(const GroupDev& d, uint32_t l, uint32_t i,
                                                  const double* __restrict__ cells) {
    const uint32_t P = d.P;
    LM(d.qrow, i) = gather_sum(cells, P, l, d.q_ptr, d.q_cell, i);
}

// The cells of a template: an iteration's instance phase writes them, its
// gather reads them, and its limiter pass (after the gather) overwrites them
// with the next iteration's instance phase. One buffer: the only values of
// an iteration still needed after that pass, its site charges, are kept in
// site_prev by the update phase before it.
__device__ __forceinline__ double* cell_buf(const GroupDev& d, uint32_t) { return d.cells; }

}  // namespace espl
