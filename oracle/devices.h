/* ORACLE (test infrastructure only): device-model restatements. */
#ifndef ESPICE_ORACLE_DEVICES_H
#define ESPICE_ORACLE_DEVICES_H

#include "oracle.h"

typedef struct {
    double is_t, vte, vcrit, gmin, cjo, cjo_t, vj_t, mt, fc, tt;
} dev_diode;

typedef struct {
    double type, vt, beta, lambda, gamma, phit, sqrt_phit, von0, isat, vcrit, gmin, vgs_seed;
} dev_mos1;

typedef struct {
    double mode, id, gm, gds, gmbs, von;
    double ibs, gbs, ibd, gbd;
} dev_mos1_out;

void dev_setup_diode(const double *p, dev_diode *d);
void dev_setup_mos1(const double *p, dev_mos1 *m);
void dev_mos1_core(const dev_mos1 *m, double vgs, double vds, double vbs, dev_mos1_out *o);
void dev_mos1_limit(const dev_mos1 *m, const double old[3], const double cur[3], double out[3]);
void dev_diode_core(const dev_diode *d, double vd, double *i, double *g, double *q, double *c);
double dev_source_value(const double *p, int tran, double t);
double dev_source_next_bp(const double *p, double t);

#endif
