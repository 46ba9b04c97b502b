/* ORACLE (test infrastructure only; never linked into the product).
 *
 * Device models of the lane-sweep configurations, restated from the
 * reference's Verilog-A in plain FP64 C with hand-derived derivatives (the
 * reference differentiates by VerA's forward AD; the partials are the same
 * functions):
 *   resistor  models/resistor.va:49-56   I(p,n) = V(p,n) / r
 *   capacitor models/capacitor.va:13     I(p,n) = c ddt(V(p,n))
 *   vsource   models/vsource.va (waveform 0 DC, 1 PULSE), V(p,n) <+ out
 *   isource   models/isource.va (same waveforms), I(p,n) <+ out
 *   diode     models/diode.va:119-376 (tlev 0, rs 0, no breakdown, no
 *             ikf/isr): Shockley current with the 80*vte tangent
 *             continuation and the -3*vte cubic tail, gmin shunt, pnjlim,
 *             depletion + diffusion charge
 *   mos1      models/mos1.va:19-500 (rd = rs = 0, TOX and CJ not given, so
 *             no Meyer or junction charge): Shichman-Hodges current with
 *             mode swap and body effect, bulk junctions jcur, and the
 *             mos1load.c limiting sequence (fetlim, limvds, pnjlim)
 * The limiters follow ngspice devsup.c (DEVpnjlim, DEVfetlim, DEVlimvds),
 * which models/mos1.va:14,290-308 and models/diode.va:13-17 name; VerA's
 * own code for them is not vendored, so this boundary is unpinned.
 */
#include "devices.h"

#include <float.h>
#include <math.h>
#include <string.h>

/* ngspice const.h CODATA 2014, as mos1.va and diode.va use them. */
#define K_BOLTZ 1.38064852e-23
#define Q_CHARGE 1.6021766208e-19
#define TNOM_K 300.15
#define GMIN_DEFAULT 1e-12

double orc_pnjlim(double vnew, double vold, double vt, double vcrit, int *icheck) {
    /* ngspice devsup.c DEVpnjlim */
    if (vnew > vcrit && fabs(vnew - vold) > vt + vt) {
        if (vold > 0) {
            double arg = 1 + (vnew - vold) / vt;
            if (arg > 0) vnew = vold + vt * log(arg);
            else vnew = vcrit;
        } else {
            vnew = vt * log(vnew / vt);
        }
        *icheck = 1;
    } else {
        if (vnew < 0) {
            double arg = vold > 0 ? -1 * vold - 1 : 2 * vold - 1;
            if (vnew < arg) {
                vnew = arg;
                *icheck = 1;
            } else {
                *icheck = 0;
            }
        } else {
            *icheck = 0;
        }
    }
    return vnew;
}

double orc_fetlim(double vnew, double vold, double vto) {
    /* ngspice devsup.c DEVfetlim */
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
                    vnew = vnew > vto + 2 ? vnew : vto + 2;
                }
            } else {
                if (delv >= vtsthi) vnew = vold + vtsthi;
            }
        } else {
            if (delv <= 0) vnew = vnew > vto - .5 ? vnew : vto - .5;
            else vnew = vnew < vto + 4 ? vnew : vto + 4;
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

double orc_limvds(double vnew, double vold) {
    /* ngspice devsup.c DEVlimvds */
    if (vold >= 3.5) {
        if (vnew > vold) {
            double c = 3 * vold + 2;
            vnew = vnew < c ? vnew : c;
        } else if (vnew < 3.5) {
            vnew = vnew > 2 ? vnew : 2;
        }
    } else {
        if (vnew > vold) vnew = vnew < 4 ? vnew : 4;
        else vnew = vnew > -.5 ? vnew : -.5;
    }
    return vnew;
}

/* ---------------- setup: bias-independent prep per (instance, lane) ----- */

void dev_setup_diode(const double *p, dev_diode *d) {
    /* diode.va:119-258 at tk = tnom = 300.15 K, area 1, tlev 0, tlevc 0. */
    double is = p[0], n = p[1], cjo = p[2], vj = p[3], m = p[4], fc = p[5], tt = p[6];
    double tk = TNOM_K, tnomk = 27.0 + 273.15;
    double ratio = tk / tnomk;
    double vt = K_BOLTZ / Q_CHARGE * tk;
    double vtnom = K_BOLTZ / Q_CHARGE * tnomk;
    double vte = n * vt;
    double egp = 1.11;
    double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
    double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
    double mt = m;
    double fact1 = tnomk / 300.15, fact2 = tk / 300.15;
    double arg1 = -egfet1 / (2.0 * K_BOLTZ * tnomk) + 1.1150877 / (2.0 * K_BOLTZ * 300.15);
    double argt = -egfet / (2.0 * K_BOLTZ * tk) + 1.1150877 / (2.0 * K_BOLTZ * 300.15);
    double pbfact1 = -2.0 * vtnom * (1.5 * log(fact1) + Q_CHARGE * arg1);
    double pbfact = -2.0 * vt * (1.5 * log(fact2) + Q_CHARGE * argt);
    double pbo = (vj - pbfact1) / fact1;
    double gmaold = (vj - pbo) / pbo;
    double vj_t = pbfact + fact2 * pbo;
    double gmanew = (vj_t - pbo) / pbo;
    double cjo_t = cjo * (1.0 + mt * (400e-6 * (tk - 300.15) - gmanew)) / (1.0 + mt * (400e-6 * (tnomk - 300.15) - gmaold));
    double xti = 3.0;
    double is_t = is * 1.0 * exp((ratio - 1.0) * egp / vte + (xti / n) * log(ratio));
    d->is_t = is_t;
    d->vte = vte;
    d->vcrit = vte * log(vte / (1.4142135623730951 * is_t));
    d->gmin = GMIN_DEFAULT;
    d->cjo = cjo;
    d->cjo_t = cjo_t;
    d->vj_t = vj_t;
    d->mt = mt;
    d->fc = fc;
    d->tt = tt;
}

void dev_setup_mos1(const double *p, dev_mos1 *m) {
    /* mos1.va:138-259 with TOX, NSUB not given, rd = rs = 0, ld = 0,
     * tk = tnom. */
    double type = p[0], vto = p[1], kp = p[2], gamma = p[3], phi = p[4], lambda = p[5], is = p[6], w = p[7], l = p[8];
    double tnomk = 27.0 + 273.15;
    double vtnom = tnomk * (K_BOLTZ / Q_CHARGE);
    double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
    double phix = phi, gammax = gamma, vtox = vto, kpx = kp;
    double tk = TNOM_K;
    double vt = tk * (K_BOLTZ / Q_CHARGE);
    double fact1 = tnomk / 300.15, fact2 = tk / 300.15;
    double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
    double arg1 = -egfet1 / (2.0 * K_BOLTZ * tnomk) + 1.1150877 / (2.0 * K_BOLTZ * 300.15);
    double argt = -egfet / (2.0 * K_BOLTZ * tk) + 1.1150877 / (2.0 * K_BOLTZ * 300.15);
    double pbfact1 = -2.0 * vtnom * (1.5 * log(fact1) + Q_CHARGE * arg1);
    double pbfact = -2.0 * vt * (1.5 * log(fact2) + Q_CHARGE * argt);
    double ratio4 = (tk / tnomk) * sqrt(tk / tnomk);
    double kpt = kpx / ratio4;
    double phio = (phix - pbfact1) / fact1;
    double phit = fact2 * phio + pbfact;
    double vbit = vtox - type * (gammax * sqrt(phix)) + 0.5 * (egfet1 - egfet) + type * 0.5 * (phit - phix);
    double ist = is * exp(-egfet / vt + egfet1 / vtnom);
    double leff = l;
    if (leff < 1.0e-10) leff = 1.0e-10;
    double beta = kpt * 1.0 * w / leff;
    double isat = ist * 1.0;
    m->type = type;
    m->vt = vt;
    m->beta = beta;
    m->lambda = lambda;
    m->gamma = gammax;
    m->phit = phit;
    m->sqrt_phit = sqrt(phit);
    m->von0 = vbit * type; /* `vbit * type` of von = vbit*type + gamma*sarg */
    m->isat = isat;
    m->vcrit = vt * log(vt / (1.4142135623730951 * isat));
    m->gmin = GMIN_DEFAULT;
    /* MODEINITJCT seed of the limited vgs: type*vbit + gamma*sqrt(phit). */
    m->vgs_seed = type * vbit + gammax * sqrt(phit);
}

/* ---------------- bias-dependent evaluation ---------------- */

/* mos1.va jcur: value and slope. */
static void jcur(double v, double isat, double vtx, double gm, double *i, double *g) {
    if (v > -3.0 * vtx) {
        double r = v / vtx;
        double u = r < 80.0 ? r : 80.0;
        double e = exp(u);
        *i = isat * (e * (1.0 + (r - u)) - 1.0) + gm * v;
        *g = isat * e / vtx + gm;
    } else {
        *i = gm * v - isat;
        *g = gm;
    }
}

/* mos1.va sbody with the frozen-copy slope above vbx = 0. */
static void sbody(double vbx, double phit, double *s, double *ds) {
    if (vbx <= 0.0) {
        *s = sqrt(phit - vbx);
        *ds = -0.5 / *s;
    } else {
        double sp = sqrt(phit);
        double v = sp - vbx / (2.0 * sp);
        if (v > 0.0) {
            *s = v;
            *ds = -1.0 / (2.0 * v);
        } else {
            *s = 0.0;
            *ds = 0.0;
        }
    }
}

/* Channel current in the normalized frame at (vgs, vds, vbs): id (drain to
 * source, normalized sign) and its partials. */
void dev_mos1_core(const dev_mos1 *m, double vgs, double vds, double vbs, dev_mos1_out *o) {
    double vbd = vbs - vds, vgd = vgs - vds;
    jcur(vbs, m->isat, m->vt, m->gmin, &o->ibs, &o->gbs);
    jcur(vbd, m->isat, m->vt, m->gmin, &o->ibd, &o->gbd);
    double mode, vbx, vgsx, vdsx;
    if (vds >= 0.0) {
        mode = 1.0;
        vbx = vbs;
        vgsx = vgs;
        vdsx = vds;
    } else {
        mode = -1.0;
        vbx = vbd;
        vgsx = vgd;
        vdsx = -vds;
    }
    double sarg, dsarg;
    sbody(vbx, m->phit, &sarg, &dsarg);
    double von = m->von0 + m->gamma * sarg;
    double dvon = m->gamma * dsarg;
    double vgst = vgsx - von;
    double bp = m->beta * (1.0 + m->lambda * vdsx);
    double id, d_g, d_d, d_b; /* partials wrt vgsx, vdsx, vbx */
    if (vgst <= 0.0) {
        id = d_g = d_d = d_b = 0.0;
    } else if (vgst <= vdsx) {
        id = 0.5 * bp * vgst * vgst;
        d_g = bp * vgst;
        d_d = 0.5 * vgst * vgst * m->beta * m->lambda;
        d_b = -bp * vgst * dvon;
    } else {
        id = bp * vdsx * (vgst - 0.5 * vdsx);
        d_g = bp * vdsx;
        d_d = bp * (vgst - vdsx) + m->beta * m->lambda * vdsx * (vgst - 0.5 * vdsx);
        d_b = -bp * vdsx * dvon;
    }
    /* Back to the unswapped normalized frame. */
    o->mode = mode;
    o->id = id;
    if (mode > 0) {
        o->gm = d_g;
        o->gds = d_d;
        o->gmbs = d_b;
    } else {
        o->gm = d_g;
        o->gmbs = d_b;
        o->gds = -d_g - d_d - d_b;
    }
    o->von = von;
}

/* The limiting sequence of mos1load.c as models/mos1.va:290-308 spells it,
 * in the normalized frame. old: limited (vgs, vds, vbs) of the previous
 * iterate. cur: the new iterate. out: limited values. */
void dev_mos1_limit(const dev_mos1 *m, const double old[3], const double cur[3], double out[3]) {
    double vgs = cur[0], vds = cur[1], vbs = cur[2];
    double vgs_o = old[0], vds_o = old[1], vbs_o = old[2];
    double vbd = vbs - vds, vgd = vgs - vds;
    double vgdo = vgs_o - vds_o, vbdo = vbs_o - vds_o;
    /* The threshold the previous load stored: von at the old iterate. */
    double vbx_o = vds_o >= 0.0 ? vbs_o : vbdo;
    double s, ds;
    sbody(vbx_o, m->phit, &s, &ds);
    double von = m->von0 + m->gamma * s;
    if (vds_o >= 0.0) {
        vgs = orc_fetlim(vgs, vgs_o, von);
        vds = vgs - vgd;
        vds = orc_limvds(vds, vds_o);
        vgd = vgs - vds;
    } else {
        vgd = orc_fetlim(vgd, vgdo, von);
        vds = vgs - vgd;
        vds = -orc_limvds(-vds, -vds_o);
        vgs = vgd + vds;
    }
    int check;
    if (vds >= 0.0) {
        vbs = orc_pnjlim(vbs, vbs_o, m->vt, m->vcrit, &check);
        vbd = vbs - vds;
    } else {
        vbd = orc_pnjlim(vbd, vbdo, m->vt, m->vcrit, &check);
        vbs = vbd + vds;
    }
    (void)vbd;
    out[0] = vgs;
    out[1] = vds;
    out[2] = vbs;
}

/* Diode current and charge at vd. */
void dev_diode_core(const dev_diode *d, double vd, double *i, double *g, double *q, double *c) {
    double vte = d->vte, is = d->is_t;
    double id, gd;
    if (vd >= -3.0 * vte) {
        double u = vd / vte;
        double ul = u < 80.0 ? u : 80.0;
        double e = exp(ul);
        id = is * (e * (1.0 + (u - ul)) - 1.0);
        gd = is * e / vte;
    } else {
        double a = 3.0 * vte / (vd * 2.718281828459045);
        double a3 = a * a * a;
        id = -is * (1.0 + a3);
        gd = 3.0 * is * a3 / vd;
    }
    *i = id + d->gmin * vd;
    *g = gd + d->gmin;
    double qj = 0.0, cj = 0.0;
    if (d->cjo > 0.0) {
        double vj = d->vj_t, mt = d->mt, fc = d->fc;
        double vfc = fc * vj;
        if (vd < vfc) {
            double base = 1.0 - vd / vj;
            qj = d->cjo_t * vj * (1.0 - pow(base, 1.0 - mt)) / (1.0 - mt);
            cj = d->cjo_t * pow(base, -mt);
        } else {
            double f1 = vj * (1.0 - pow(1.0 - fc, 1.0 - mt)) / (1.0 - mt);
            double f2 = pow(1.0 - fc, 1.0 + mt);
            double f3 = 1.0 - fc * (1.0 + mt);
            qj = d->cjo_t * (f1 + (1.0 / f2) * (f3 * (vd - vfc) + (mt / (2.0 * vj)) * (vd * vd - vfc * vfc)));
            cj = d->cjo_t * (1.0 / f2) * (f3 + (mt / vj) * vd);
        }
    }
    if (d->tt > 0.0) {
        qj += d->tt * (id + d->gmin * vd);
        cj += d->tt * (gd + d->gmin);
    }
    *q = qj;
    *c = cj;
}

/* vsource.va / isource.va waveform value. `tran`: the analysis is a
 * transient (its operating point included), where a PULSE is read at t. */
double dev_source_value(const double *p, int tran, double t) {
    double dc = p[0];
    if (!tran || p[1] != 1.0) return dc;
    double v1 = p[2], v2 = p[3], td = p[4], tr = p[5], tf = p[6], pw = p[7], per = p[8];
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

/* The next PULSE corner strictly after t (timer events of vsource.va:
 * td, td+tr, td+tr+pw, td+tr+pw+tf, each every period), inf for none. */
double dev_source_next_bp(const double *p, double t) {
    if (p[1] != 1.0) return INFINITY;
    double td = p[4], tr = p[5], tf = p[6], pw = p[7], per = p[8];
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
