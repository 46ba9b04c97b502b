// Device-model math of the lane kernels, FP64, one thread per lane.
//
// Restated from the reference's Verilog-A (the reference runs VerA-generated
// code through its forward-mode AD; the partials here are hand-derived from
// the same expressions):
//   models/mos1.va:19-500  Shichman-Hodges MOS1 (rd = rs = 0, no TOX, no CJ):
//                          jcur (:106), sbody with the frozen-copy slope above
//                          vbx = 0 (:120, :328-334), mode swap, the three
//                          regions (:336-346), mos1load.c's limiting order
//                          (:290-308);
//   models/diode.va:119-376 Shockley diode, 80*vte tangent continuation,
//                          -3*vte cubic tail, gmin shunt, depletion and
//                          diffusion charge;
//   models/vsource.va, models/isource.va PULSE waveform (waveform 1).
// The `$limit` functions follow ngspice devsup.c (DEVpnjlim, DEVfetlim,
// DEVlimvds), named by models/mos1.va:14 and models/diode.va:13-17.
#pragma once

#include <cstdint>

namespace espl {

// ngspice const.h (CODATA 2014), as mos1.va and diode.va use them.
constexpr double kBoltz = 1.38064852e-23;
constexpr double kQ = 1.6021766208e-19;
constexpr double kTnomK = 27.0 + 273.15;
constexpr double kGminDevice = 1e-12;  // $simparam("gmin"), the .options default

// Derived per-(instance, lane) MOS1 constants: the bias-independent prep of
// mos1.va:138-259 at the device temperature = tnom.
struct Mos1Prep {
    enum { type, vt, beta, lambda, gamma, phit, von0, isat, vcrit, gmin, vgs_seed, count };
};
// The lane-uniform MOS prep values (GroupDev mos_u), in this order.
constexpr uint32_t kMosUni = 8;
__host__ __device__ constexpr int mos_uni_field(uint32_t k) {
    return k == 0 ? Mos1Prep::type : k == 1 ? Mos1Prep::vt : k == 2 ? Mos1Prep::lambda : k == 3 ? Mos1Prep::gamma
         : k == 4 ? Mos1Prep::phit : k == 5 ? Mos1Prep::isat : k == 6 ? Mos1Prep::vcrit : Mos1Prep::gmin;
}
struct DiodePrep {
    enum { is, vte, vcrit, gmin, cjo, cjo_t, vj_t, mt, fc, tt, count };
};

__host__ __device__ inline void mos1_setup(const double p[9], double out[Mos1Prep::count]) {
    double type = p[0], vto = p[1], kp = p[2], gamma = p[3], phi = p[4], lambda = p[5], is = p[6], w = p[7], l = p[8];
    double tnomk = kTnomK;
    double vtnom = tnomk * (kBoltz / kQ);
    double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
    double tk = kTnomK;
    double vt = tk * (kBoltz / kQ);
    double fact1 = tnomk / 300.15, fact2 = tk / 300.15;
    double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
    double arg1 = -egfet1 / (2.0 * kBoltz * tnomk) + 1.1150877 / (2.0 * kBoltz * 300.15);
    double argt = -egfet / (2.0 * kBoltz * tk) + 1.1150877 / (2.0 * kBoltz * 300.15);
    double pbfact1 = -2.0 * vtnom * (1.5 * log(fact1) + kQ * arg1);
    double pbfact = -2.0 * vt * (1.5 * log(fact2) + kQ * argt);
    double ratio4 = (tk / tnomk) * sqrt(tk / tnomk);
    double kpt = kp / ratio4;
    double phio = (phi - pbfact1) / fact1;
    double phit = fact2 * phio + pbfact;
    double vbit = vto - type * (gamma * sqrt(phi)) + 0.5 * (egfet1 - egfet) + type * 0.5 * (phit - phi);
    double ist = is * exp(-egfet / vt + egfet1 / vtnom);
    double leff = l < 1.0e-10 ? 1.0e-10 : l;
    out[Mos1Prep::type] = type;
    out[Mos1Prep::vt] = vt;
    out[Mos1Prep::beta] = kpt * 1.0 * w / leff;
    out[Mos1Prep::lambda] = lambda;
    out[Mos1Prep::gamma] = gamma;
    out[Mos1Prep::phit] = phit;
    out[Mos1Prep::von0] = vbit * type;
    out[Mos1Prep::isat] = ist;
    out[Mos1Prep::vcrit] = vt * log(vt / (1.4142135623730951 * ist));
    out[Mos1Prep::gmin] = kGminDevice;
    out[Mos1Prep::vgs_seed] = type * vbit + gamma * sqrt(phit);
}

__host__ __device__ inline void diode_setup(const double p[7], double out[DiodePrep::count]) {
    double is = p[0], n = p[1], cjo = p[2], vj = p[3], m = p[4], fc = p[5], tt = p[6];
    double tk = kTnomK, tnomk = kTnomK;
    double ratio = tk / tnomk;
    double vt = kBoltz / kQ * tk, vtnom = kBoltz / kQ * tnomk;
    double vte = n * vt;
    double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
    double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
    double fact1 = tnomk / 300.15, fact2 = tk / 300.15;
    double arg1 = -egfet1 / (2.0 * kBoltz * tnomk) + 1.1150877 / (2.0 * kBoltz * 300.15);
    double argt = -egfet / (2.0 * kBoltz * tk) + 1.1150877 / (2.0 * kBoltz * 300.15);
    double pbfact1 = -2.0 * vtnom * (1.5 * log(fact1) + kQ * arg1);
    double pbfact = -2.0 * vt * (1.5 * log(fact2) + kQ * argt);
    double pbo = (vj - pbfact1) / fact1;
    double gmaold = (vj - pbo) / pbo;
    double vj_t = pbfact + fact2 * pbo;
    double gmanew = (vj_t - pbo) / pbo;
    double cjo_t = cjo * (1.0 + m * (400e-6 * (tk - 300.15) - gmanew)) / (1.0 + m * (400e-6 * (tnomk - 300.15) - gmaold));
    double is_t = is * 1.0 * exp((ratio - 1.0) * 1.11 / vte + (3.0 / n) * log(ratio));
    out[DiodePrep::is] = is_t;
    out[DiodePrep::vte] = vte;
    out[DiodePrep::vcrit] = vte * log(vte / (1.4142135623730951 * is_t));
    out[DiodePrep::gmin] = kGminDevice;
    out[DiodePrep::cjo] = cjo;
    out[DiodePrep::cjo_t] = cjo_t;
    out[DiodePrep::vj_t] = vj_t;
    out[DiodePrep::mt] = m;
    out[DiodePrep::fc] = fc;
    out[DiodePrep::tt] = tt;
}

__device__ __forceinline__ double pnjlim(double vnew, double vold, double vt, double vcrit) {
    if (vnew > vcrit && fabs(vnew - vold) > vt + vt) {
        if (vold > 0) {
            double arg = 1 + (vnew - vold) / vt;
            vnew = arg > 0 ? vold + vt * log(arg) : vcrit;
        } else {
            vnew = vt * log(vnew / vt);
        }
    } else if (vnew < 0) {
        double arg = vold > 0 ? -1 * vold - 1 : 2 * vold - 1;
        if (vnew < arg) vnew = arg;
    }
    return vnew;
}

__device__ __forceinline__ double fetlim(double vnew, double vold, double vto) {
    double vtsthi = fabs(2 * (vold - vto)) + 2;
    double vtstlo = fabs(vold - vto) + 1;
    double vtox = vto + 3.5;
    double delv = vnew - vold;
    if (vold >= vto) {
        if (vold >= vtox) {
            if (delv <= 0) {
                if (vnew >= vtox) {
                    if (-delv > vtstlo) vnew = vold - vtstlo;
                } else {
                    vnew = fmax(vnew, vto + 2);
                }
            } else if (delv >= vtsthi) {
                vnew = vold + vtsthi;
            }
        } else {
            vnew = delv <= 0 ? fmax(vnew, vto - .5) : fmin(vnew, vto + 4);
        }
    } else {
        if (delv <= 0) {
            if (-delv > vtsthi) vnew = vold - vtsthi;
        } else {
            double vtemp = vto + .5;
            if (vnew <= vtemp) {
                if (delv > vtstlo) vnew = vold + vtstlo;
            } else {
                vnew = vtemp;
            }
        }
    }
    return vnew;
}

__device__ __forceinline__ double limvds(double vnew, double vold) {
    if (vold >= 3.5) {
        if (vnew > vold) vnew = fmin(vnew, 3 * vold + 2);
        else if (vnew < 3.5) vnew = fmax(vnew, 2.0);
    } else {
        vnew = vnew > vold ? fmin(vnew, 4.0) : fmax(vnew, -.5);
    }
    return vnew;
}

__device__ __forceinline__ void jcur(double v, double isat, double vtx, double gm, double& i, double& g) {
    if (v > -3.0 * vtx) {
        double r = v / vtx;
        double u = fmin(r, 80.0);
        double e = exp(u);
        i = isat * (e * (1.0 + (r - u)) - 1.0) + gm * v;
        g = isat * e / vtx + gm;
    } else {
        i = gm * v - isat;
        g = gm;
    }
}

__device__ __forceinline__ void sbody(double vbx, double phit, double& s, double& ds) {
    if (vbx <= 0.0) {
        s = sqrt(phit - vbx);
        ds = -0.5 / s;
    } else {
        double sp = sqrt(phit);
        double v = sp - vbx / (2.0 * sp);
        if (v > 0.0) {
            s = v;
            ds = -1.0 / (2.0 * v);
        } else {
            s = 0.0;
            ds = 0.0;
        }
    }
}

struct Mos1Out {
    double mode, id, gm, gds, gmbs, ibs, gbs, ibd, gbd;
};

// Channel current (normalized frame) and bulk junctions at (vgs, vds, vbs).
__device__ __forceinline__ void mos1_core(double type_unused, double vt, double beta, double lambda, double gamma,
                                          double phit, double von0, double isat, double gmin, double vgs, double vds,
                                          double vbs, Mos1Out& o) {
    double vbd = vbs - vds, vgd = vgs - vds;
    jcur(vbs, isat, vt, gmin, o.ibs, o.gbs);
    jcur(vbd, isat, vt, gmin, o.ibd, o.gbd);
    double mode, vbx, vgsx, vdsx;
    if (vds >= 0.0) {
        mode = 1.0; vbx = vbs; vgsx = vgs; vdsx = vds;
    } else {
        mode = -1.0; vbx = vbd; vgsx = vgd; vdsx = -vds;
    }
    double sarg, dsarg;
    sbody(vbx, phit, sarg, dsarg);
    double von = von0 + gamma * sarg;
    double dvon = gamma * dsarg;
    double vgst = vgsx - von;
    double bp = beta * (1.0 + lambda * vdsx);
    double id, dg, dd, db;
    if (vgst <= 0.0) {
        id = dg = dd = db = 0.0;
    } else if (vgst <= vdsx) {
        id = 0.5 * bp * vgst * vgst;
        dg = bp * vgst;
        dd = 0.5 * vgst * vgst * beta * lambda;
        db = -bp * vgst * dvon;
    } else {
        id = bp * vdsx * (vgst - 0.5 * vdsx);
        dg = bp * vdsx;
        dd = bp * (vgst - vdsx) + beta * lambda * vdsx * (vgst - 0.5 * vdsx);
        db = -bp * vdsx * dvon;
    }
    o.mode = mode;
    o.id = id;
    o.gm = dg;
    o.gmbs = db;
    o.gds = mode > 0 ? dd : -dg - dd - db;
}

// mos1load.c's limiting sequence in the normalized frame; von is the
// threshold at the previous (limited) iterate.
__device__ __forceinline__ void mos1_limit(double vt, double gamma, double phit, double von0, double vcrit,
                                           double vgs_o, double vds_o, double vbs_o, double& vgs, double& vds,
                                           double& vbs) {
    double vgd = vgs - vds, vbd = vbs - vds;  // from the unlimited iterate
    double vgdo = vgs_o - vds_o, vbdo = vbs_o - vds_o;
    double s, ds;
    sbody(vds_o >= 0.0 ? vbs_o : vbdo, phit, s, ds);
    double von = von0 + gamma * s;
    if (vds_o >= 0.0) {
        vgs = fetlim(vgs, vgs_o, von);
        vds = vgs - vgd;
        vds = limvds(vds, vds_o);
    } else {
        vgd = fetlim(vgd, vgdo, von);
        vds = vgs - vgd;
        vds = -limvds(-vds, -vds_o);
        vgs = vgd + vds;
    }
    if (vds >= 0.0) {
        vbs = pnjlim(vbs, vbs_o, vt, vcrit);
    } else {
        vbd = pnjlim(vbd, vbdo, vt, vcrit);
        vbs = vbd + vds;
    }
}

__device__ __forceinline__ void diode_core(double is, double vte, double gmin, double cjo, double cjo_t, double vj,
                                           double mt, double fc, double tt, double vd, double& i, double& g,
                                           double& q, double& c) {
    double id, gd;
    if (vd >= -3.0 * vte) {
        double u = vd / vte;
        double ul = fmin(u, 80.0);
        double e = exp(ul);
        id = is * (e * (1.0 + (u - ul)) - 1.0);
        gd = is * e / vte;
    } else {
        double a = 3.0 * vte / (vd * 2.718281828459045);
        double a3 = a * a * a;
        id = -is * (1.0 + a3);
        gd = 3.0 * is * a3 / vd;
    }
    i = id + gmin * vd;
    g = gd + gmin;
    double qj = 0.0, cj = 0.0;
    if (cjo > 0.0) {
        double vfc = fc * vj;
        if (vd < vfc) {
            double base = 1.0 - vd / vj;
            qj = cjo_t * vj * (1.0 - pow(base, 1.0 - mt)) / (1.0 - mt);
            cj = cjo_t * pow(base, -mt);
        } else {
            double f1 = vj * (1.0 - pow(1.0 - fc, 1.0 - mt)) / (1.0 - mt);
            double f2 = pow(1.0 - fc, 1.0 + mt);
            double f3 = 1.0 - fc * (1.0 + mt);
            qj = cjo_t * (f1 + (1.0 / f2) * (f3 * (vd - vfc) + (mt / (2.0 * vj)) * (vd * vd - vfc * vfc)));
            cj = cjo_t * (1.0 / f2) * (f3 + (mt / vj) * vd);
        }
    }
    if (tt > 0.0) {
        qj += tt * (id + gmin * vd);
        cj += tt * (gd + gmin);
    }
    q = qj;
    c = cj;
}

// vsource.va / isource.va: DC, or PULSE in a transient (its operating point
// included, where the pulse is read at t = 0).
__host__ __device__ inline double source_value(double dc, double wave, double v1, double v2, double td, double tr,
                                               double tf, double pw, double per, int tran, double t) {
    if (!tran || wave != 1.0) return dc;
    double p_tr = tr > 1.0e-12 ? tr : 1.0e-12;
    double p_tf = tf > 1.0e-12 ? tf : 1.0e-12;
    double p_pw = (pw > 0.0 ? pw : 0.0) + (-pw > 0.0 ? -pw : 0.0) * 1.0e30;
    double minper = p_tr + p_pw + p_tf + 1.0e-12;
    double p_per = per > minper ? per : minper;
    double t_rel = t - td;
    double t_mod = t_rel + (0.0 / 360.0) * p_per;
    t_mod = t_mod - floor(t_mod / p_per) * p_per;
    t_mod = t_mod > 0.0 ? t_mod : 0.0;
    if (t_rel < 0.0) return v1;
    if (t_mod < p_tr) return v1 + (v2 - v1) * (t_mod / p_tr);
    if (t_mod < p_tr + p_pw) return v2;
    if (t_mod < p_tr + p_pw + p_tf) return v2 - (v2 - v1) * ((t_mod - (p_tr + p_pw)) / p_tf);
    return v1;
}

// The next PULSE corner strictly after t (the four timer events of
// vsource.va each period), +inf for none.
__host__ __device__ inline double source_next_bp(double wave, double td, double tr, double tf, double pw, double per,
                                                 double t) {
    if (wave != 1.0) return INFINITY;
    double p_tr = tr > 1.0e-12 ? tr : 1.0e-12;
    double p_tf = tf > 1.0e-12 ? tf : 1.0e-12;
    double p_pw = (pw > 0.0 ? pw : 0.0) + (-pw > 0.0 ? -pw : 0.0) * 1.0e30;
    double minper = p_tr + p_pw + p_tf + 1.0e-12;
    double p_per = per > minper ? per : minper;
    double corners[4] = {td, td + p_tr, td + p_tr + p_pw, td + p_tr + p_pw + p_tf};
    double best = INFINITY;
    double k0 = floor((t - td) / p_per);
    if (k0 < 0) k0 = 0;
    for (int kk = 0; kk < 2; kk++) {
        double base = (k0 + kk) * p_per;
        for (int c = 0; c < 4; c++) {
            double tc = corners[c] + base;
            if (tc > t && tc < best) best = tc;
        }
    }
    return best;
}

}  // namespace espl
