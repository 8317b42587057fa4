/*
 * Oracle (test infrastructure): FP64 restatement of radmod.f90's column pass
 * -- solarini band split (:166-376), solang (:1336-1444), mko3 (:1451-1524),
 * swr (:1530-2116), lwr (:2122-2456) and radstep's heating rates
 * (:927-1110).  The reference evaluates each statement over all NHOR columns
 * (array syntax with WHERE masks); columns never interact except through the
 * ndcycle=0 zonal mean, so the restatement runs the same statements column by
 * column.  Entropy diagnostics (dftue1/2, dftu0, dftd0) and the aerosol block
 * (l_aerorad=1) are not restated: they do not feed the fluxes or heating
 * rates of the default configuration.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "exo_oracle.h"

#define PI_PUMA 3.14159265359          /* plasimmod.f90:119 */
#define TWOPI_PUMA (PI_PUMA + PI_PUMA)

void oracle_radpar_default(oracle_radpar *p, int nlev, int nhor, int nlon,
                           const double *sigma, const double *sigmah,
                           const double *dsigma) {
    memset(p, 0, sizeof(*p));
    p->nlev = nlev; p->nhor = nhor; p->nlon = nlon;
    p->sigma = sigma; p->sigmah = sigmah; p->dsigma = dsigma;
    /* p_earth.f90:41-58 and plasim.f90:1317-1318 */
    p->ga = 9.80665; p->gascon = 287.0;
    p->acpd = p->gascon / 0.286;
    p->adv = 1870.0 / p->acpd - 1.0;
    /* radmod.f90:27-100 */
    p->gsol0 = 1367.0; p->gdist2 = 1.0;
    p->zsolar1 = 0.517; p->zsolar2 = 0.483; p->rcoeff = 1.0;
    p->tswr1 = 0.077; p->tswr2 = 0.065; p->tswr3 = 0.0055;
    p->tpofmt = 1.0; p->acllwr = 0.1; p->th2oc = 0.024; p->clgray = -1.0;
    p->a0o3 = 0.25; p->a1o3 = 0.11; p->aco3 = 0.08; p->bo3 = 20000.0;
    p->co3 = 5000.0; p->toffo3 = 0.25; p->o3scale = 1.0;
    p->rcl1[0] = 0.15; p->rcl1[1] = 0.30; p->rcl1[2] = 0.60;
    p->rcl2[0] = 0.15; p->rcl2[1] = 0.30; p->rcl2[2] = 0.60;
    p->acl2[0] = 0.05; p->acl2[1] = 0.10; p->acl2[2] = 0.20;
    p->ndcycle = 1; p->no3 = 1; p->nswrcl = 1; p->nclouds = 1; p->nrscat = 1;
    p->newrsc = 0; p->necham = 1; p->necham6 = 0; p->nstartemp = 0;
    p->npbroaden = 1; p->nswr = 1; p->nlwr = 1; p->nsol = 1;
    p->nfixed = 0; p->ncstsol = 0; p->ngenkeplerian = 0;
    p->zdecl = 0.0; p->zmins = 0.0; p->zrtim = TWOPI_PUMA / 1440.0; p->rasc = 0.0;
    p->dawn = 0.0; p->solclat = 1.0; p->solcdec = 1.0; p->zcday = 0.0;
}

/* SUBROUTINE SOLARINI band split, radmod.f90:166-376 (blackbody branch) */
void oracle_solarini(double starbbtemp, double minwavel,
                     double *zsolar1, double *zsolar2, double *rcoeff) {
    const double cst = 0.0143877735383;
    double wv1[1024], wv2[1024], wvm1[1024], wvm2[1024];
    double bb1[1024], bb2[1024], bbg1[1024], bbg2[1024];
    double constg = cst / 5772.0;
    double wmin = minwavel;     /* metres: radini scales the namelist nm value by 1e-9 (radmod.f90:738) */
    double lwmin = log10(wmin);
    double hinge = log10(7.5e-7);
    double dl1 = (hinge - lwmin) / 1024.0;
    double dl2 = (-4 - hinge) / 1024.0;
    for (int k = 1; k <= 1024; k++) {
        wv1[k - 1] = pow(10.0, lwmin + (k - 1) * dl1);
        wv2[k - 1] = pow(10.0, hinge + (k - 1) * dl2);
    }
    for (int k = 0; k < 1024; k++) {
        wvm1[k] = pow(1.0e6 * wv1[k], 5);
        wvm2[k] = pow(1.0e6 * wv2[k], 5);
    }
    for (int k = 0; k < 1024; k++) {
        bbg1[k] = 1.0 / wvm1[k] * 1.0 / (exp(constg / wv1[k]) - 1);
        bbg2[k] = 1.0 / wvm2[k] * 1.0 / (exp(constg / wv2[k]) - 1);
    }
    double const2 = cst / starbbtemp;
    for (int k = 0; k < 1024; k++) {
        bb1[k] = 1.0 / wvm1[k] * 1.0 / (exp(const2 / wv1[k]) - 1);
        bb2[k] = 1.0 / wvm2[k] * 1.0 / (exp(const2 / wv2[k]) - 1);
    }
    double z1 = 0, z2 = 0, zg1 = 0, zg2 = 0, zc1 = 0, zc2 = 0, zgc1 = 0, zgc2 = 0;
    for (int k = 0; k < 1023; k++) {
        z1 = z1 + 0.5 * (bb1[k] + bb1[k + 1]) * (wv1[k + 1] - wv1[k]);
        z2 = z2 + 0.5 * (bb2[k] + bb2[k + 1]) * (wv2[k + 1] - wv2[k]);
        zg1 = zg1 + 0.5 * (bbg1[k] + bbg1[k + 1]) * (wv1[k + 1] - wv1[k]);
        zg2 = zg2 + 0.5 * (bbg2[k] + bbg2[k + 1]) * (wv2[k + 1] - wv2[k]);
        zc1 = zc1 + 0.5 * (bb1[k] / pow(wv1[k] * 1.0e6, 4) + bb1[k + 1] / pow(wv1[k + 1] * 1.0e6, 4)) * (wv1[k + 1] - wv1[k]);
        zc2 = zc2 + 0.5 * (bb2[k] / pow(wv2[k] * 1.0e6, 4) + bb2[k + 1] / pow(wv2[k + 1] * 1.0e6, 4)) * (wv2[k + 1] - wv2[k]);
        zgc1 = zgc1 + 0.5 * (bbg1[k] / pow(wv1[k] * 1.0e6, 4) + bbg1[k + 1] / pow(wv1[k + 1] * 1.0e6, 4)) * (wv1[k + 1] - wv1[k]);
        zgc2 = zgc2 + 0.5 * (bbg2[k] / pow(wv2[k] * 1.0e6, 4) + bbg2[k + 1] / pow(wv2[k + 1] * 1.0e6, 4)) * (wv2[k + 1] - wv2[k]);
    }
    z1 = z1 + 0.5 * (bb1[1023] + bb2[0]) * (wv2[0] - wv1[1023]);
    zc1 = zc1 + 0.5 * (bb1[1023] / pow(wv1[1023] * 1.0e6, 4) + bb2[0] / pow(wv2[0] * 1.0e6, 4)) * (wv2[0] - wv1[1023]);
    zg1 = zg1 + 0.5 * (bbg1[1023] + bbg2[0]) * (wv2[0] - wv1[1023]);
    zgc1 = zgc1 + 0.5 * (bbg1[1023] / pow(wv1[1023] * 1.0e6, 4) + bbg2[0] / pow(wv2[0] * 1.0e6, 4)) * (wv2[0] - wv1[1023]);
    double zg = zg1 + zg2, zgcross = zgc1 + zgc2;
    double zchi = zgcross / zg;
    /* rcoeff uses the module default zsolar1 = 0.517 at this point */
    *rcoeff = (zc1 + zc2) * 0.517 / z1 / zchi;
    double znet = z1 + z2;
    z1 = z1 / znet;
    *zsolar1 = z1;
    *zsolar2 = 1.0 - z1;
}

/* SUBROUTINE SOLANG zenith-angle part, radmod.f90:1380-1436 */
void oracle_solang_range(const oracle_radpar *p, const double *sid, const double *cola,
                         double *gmu0, int j0, int j1) {
    int nlon = p->nlon;
    double zdawn = sin(p->dawn * PI_PUMA / 180.0);
    double zrlon = TWOPI_PUMA / nlon;
    double zrtim = p->zrtim, zmins = p->zmins, zdecl = p->zdecl;
    for (int jhor = j0; jhor < j1; jhor++) {
        int jlat = jhor / nlon, jlon = jhor % nlon;
        {
            double zmuz;
            gmu0[jhor] = 0.0;
            if (p->ncstsol == 0) {
                double zhangle = zmins * zrtim + jlon * zrlon - PI_PUMA;
                if (p->ngenkeplerian == 1) zhangle = zhangle - p->rasc;
                if (zhangle < -PI_PUMA) zhangle = zhangle + TWOPI_PUMA;
                if (zhangle > PI_PUMA) zhangle = zhangle - TWOPI_PUMA;
                if (p->nfixed == 1) zhangle = zhangle + PI_PUMA;
                zmuz = sin(zdecl) * sid[jlat] + cola[jlat] * cos(zdecl) * cos(zhangle);
            } else {
                double solclatcdec = p->solclat * p->solcdec;
                double solslat = sqrt(1 - p->solclat * p->solclat);
                double solsdec = sqrt(1 - p->solcdec * p->solcdec);
                double solslatsdec = solslat * solsdec;
                if (p->ndcycle == 1) {
                    double zhangle = zmins * zrtim - PI_PUMA;
                    zmuz = solslatsdec + solclatcdec * cos(zhangle);
                } else {
                    zmuz = solslatsdec + solclatcdec / PI_PUMA;
                }
            }
            if (zmuz > zdawn) gmu0[jhor] = zmuz;
        }
    }
}
void oracle_solang(const oracle_radpar *p, const double *sid, const double *cola,
                   double *gmu0) {
    oracle_solang_range(p, sid, cola, gmu0, 0, p->nhor);
}

/* SUBROUTINE MKO3 (no3 == 1), radmod.f90:1489-1522 */
void oracle_mko3_range(const oracle_radpar *p, const double *sid, const double *dt,
                       const double *dp, double *dqo3, int j0, int j1) {
    int nlev = p->nlev, nhor = p->nhor, nlon = p->nlon;
    const double zro3 = 2.14, zfo3 = 100.0 / zro3;
    const double *sigmah = p->sigmah, *dsigma = p->dsigma;
    double zconst = exp(-p->bo3 / p->co3);
    for (int j = j0; j < j1; j++) {
        double s = sid[j / nlon];
        double za = p->a0o3 + p->a1o3 * fabs(s) + p->aco3 * s * cos(TWOPI_PUMA * (p->zcday - p->toffo3));
        double zo3t = za, zh = 0.0;
        for (int jlev = nlev; jlev >= 2; jlev--) {
            zh = zh - dt[(size_t)(jlev - 1) * nhor + j] * p->gascon / p->ga * log(sigmah[jlev - 2] / sigmah[jlev - 1]);
            double zo3 = -(za + za * zconst) / (1. + exp((zh - p->bo3) / p->co3)) + zo3t;
            dqo3[(size_t)(jlev - 1) * nhor + j] = zo3 * p->ga / (zfo3 * dsigma[jlev - 1] * dp[j]);
            zo3t = zo3t - zo3;
        }
        dqo3[j] = zo3t * p->ga / (zfo3 * dsigma[0] * dp[j]);
        if (p->o3scale != 1.0)
            for (int jlev = 0; jlev < nlev; jlev++) dqo3[(size_t)jlev * nhor + j] *= p->o3scale;
    }
}
void oracle_mko3(const oracle_radpar *p, const double *sid, const double *dt,
                 const double *dp, double *dqo3) {
    oracle_mko3_range(p, sid, dt, dp, dqo3, 0, p->nhor);
}

/* ozone and water-vapour broadband absorptions of swr (radmod.f90:1907-1913, 1992-1993) */
static double ao3(double x) {
    return 0.02118 * x / (1. + 0.042 * x + 0.000323 * (x * x))
         + 1.082 * x / pow(1. + 138.6 * x, 0.805)
         + 0.0658 * x / (1. + (103.6 * x) * (103.6 * x) * (103.6 * x));
}
static double awv(double x) { return 2.9 * x / (pow(1. + 141.5 * x, 0.635) + 5.925 * x); }

/* SUBROUTINE SWR for one column, radmod.f90:1530-2116 (l_aerorad = 0) */
static void swr_col(const oracle_radpar *p, int nlev, double zmu0, double zmu1,
                    double dp, double *dalb, double dsalb[2], double dls, double dicec,
                    const double *dq, const double *dql, const double *dcc,
                    const double *dqo3, const double *dt,
                    double *dfu, double *dfd, double *dswfl) {
    const double zero = 1.e-6, zbetta = 1.66, zmbar = 1.9, zro3 = 2.14, zfo3 = 100. / zro3;
    const double aa = 0.2542857142857143, bb = 0.8229693877551021, c0 = 0.14997959183673468;
    const double *sigma = p->sigma, *dsigma = p->dsigma;
    const double ga = p->ga;
    int nlep = nlev + 1;
    double zt1[nlep], zt2[nlep], zr1s[nlep], zr2s[nlep], zrl1[nlep], zrl2[nlep], zrl1s[nlep], zrl2s[nlep];
    double ztb1[nlev], ztb2[nlev], ztb1u[nlev], ztb2u[nlev], zrb1[nlev], zrb2[nlev], zrb1s[nlev], zrb2s[nlev];
    double zo3l[nlev], zxo3l[nlev], zwvl[nlev], zywvl[nlev], zrcs[nlev], zrcsu[nlev];
    double zrcl1[nlev], zrcl2[nlev], zrcl1s[nlev], zrcl2s[nlev], ztcl2[nlev], ztcl2s[nlev];
    int nclouds = p->nclouds;
    for (int k = 0; k < nlep; k++) { dfu[k] = 0.0; dfd[k] = 0.0; dswfl[k] = 0.0; }

    double zftop1 = p->zsolar1 * p->gsol0 * p->gdist2 * zmu1;
    double zftop2 = p->zsolar2 * p->gsol0 * p->gdist2 * zmu1;
    int losun = (zftop1 + zftop2 > zero);

    double zcs = 1.0, zmu00 = 0.5;
    double zb3 = p->tswr1 * sqrt(zmu00) / zmu00;
    double zb4 = p->tswr2 * sqrt(zmu00);
    double zb5 = p->tswr3 * zmu00 * zmu00;
    if (nclouds == 1) {
        if (p->nswrcl == 0) {
            for (int jl = 0; jl < nlev; jl++) {
                int r = (sigma[jl] <= 1. / 3.) ? 0 : ((sigma[jl] > 1. / 3. && sigma[jl] <= 2. / 3.) ? 1 : 2);
                zrcl1s[jl] = p->rcl1[r] / (p->rcl1[r] + zmu00);
                zrcl1[jl] = zcs * p->rcl1[r] / (p->rcl1[r] + zmu0) + (1. - zcs) * zrcl1s[jl];
                zrcl2s[jl] = fmin(1. - p->acl2[r], p->rcl2[r] / (p->rcl2[r] + zmu00));
                zrcl2[jl] = fmin(1. - p->acl2[r], zcs * p->rcl2[r] / (p->rcl2[r] + zmu0) + (1. - zcs) * zrcl2s[jl]);
                ztcl2s[jl] = 1. - zrcl2s[jl] - p->acl2[r];
                ztcl2[jl] = 1. - zrcl2[jl] - p->acl2[r];
                zcs = zcs * (1. - dcc[jl]);
            }
        } else {
            for (int jl = 0; jl < nlev; jl++) {
                zrcl1[jl] = 0.0; zrcl2[jl] = 0.0; ztcl2[jl] = 1.0;
                zrcl1s[jl] = 0.0; zrcl2s[jl] = 0.0; ztcl2s[jl] = 1.0;
            }
            for (int jl = 0; jl < nlev; jl++) {
                if (losun && dcc[jl] > 0.) {
                    double zlwp = fmin(1000.0, 1000. * dql[jl] * dp / ga * dsigma[jl]);
                    double ztau = 2.0 * pow(log10(zlwp + 1.5), 3.9);
                    double zlog = log(1000.0 / ztau);
                    double zb2 = zb4 / log(3. + 0.1 * ztau);
                    double zom0 = fmin(0.9999, 1.0 - zb5 * zlog);
                    double zun = 1.0 - zom0;
                    double zuz = zun + 2.0 * zb2 * zom0;
                    double zu = sqrt(zuz / zun);
                    double zexp = exp(fmin(25.0, ztau * sqrt(zuz * zun) / zmu00));
                    double zr = (zu + 1.) * (zu + 1.) * zexp - (zu - 1.) * (zu - 1.) / zexp;
                    zrcl1s[jl] = 1. - 1. / (1. + zb3 * ztau);
                    ztcl2s[jl] = 4. * zu / zr;
                    zrcl2s[jl] = (zu * zu - 1.) / zr * (zexp - 1. / zexp);
                    double zb1 = p->tswr1 * sqrt(zmu0);
                    zb2 = p->tswr2 * sqrt(zmu0) / log(3. + 0.1 * ztau);
                    zom0 = fmin(0.9999, 1. - p->tswr3 * zmu0 * zmu0 * zlog);
                    zun = 1.0 - zom0;
                    zuz = zun + 2.0 * zb2 * zom0;
                    zu = sqrt(zuz / zun);
                    zexp = exp(fmin(25.0, ztau * sqrt(zuz * zun) / zmu0));
                    zr = (zu + 1.) * (zu + 1.) * zexp - (zu - 1.) * (zu - 1.) / zexp;
                    zrcl1[jl] = 1. - 1. / (1. + zb1 * ztau / zmu0);
                    ztcl2[jl] = 4. * zu / zr;
                    zrcl2[jl] = (zu * zu - 1.) / zr * (zexp - 1. / zexp);
                    zrcl1[jl] = zcs * zrcl1[jl] + (1. - zcs) * zrcl1s[jl];
                    ztcl2[jl] = zcs * ztcl2[jl] + (1. - zcs) * ztcl2s[jl];
                    zrcl2[jl] = zcs * zrcl2[jl] + (1. - zcs) * zrcl2s[jl];
                }
                zcs = zcs * (1. - dcc[jl]);
            }
        }
    }
    if (!losun) return;

    double zm = 35. / sqrt(1. + 1224. * zmu0 * zmu0);
    zcs = 1.;
    double zo3t = 0., zxo3t = 0., zwvt = 0., zywvt = 0.;
    for (int jl = 0; jl < nlev; jl++) {
        double zo3 = zfo3 * dsigma[jl] * dp * dqo3[jl] / ga;
        zo3t = zo3t + zo3;
        zxo3t = zcs * (zxo3t + zm * zo3) + (1. - zcs) * (zxo3t + zmbar * zo3);
        zo3l[jl] = zo3t;
        zxo3l[jl] = zxo3t;
        double zwv = 0.1 * dsigma[jl] * dq[jl] * dp / ga * sqrt(273. / dt[jl]) * sigma[jl] * dp / 100000.;
        zwvt = zwvt + zwv;
        zywvt = zcs * (zywvt + zm * zwv) + (1. - zcs) * (zywvt + zbetta * zwv);
        zwvl[jl] = zwvt;
        zywvl[jl] = zywvt;
        zcs = zcs * (1. - dcc[jl] * nclouds);
        zrcs[jl] = (aa / (1. + bb * zmu0) * zcs + c0 * (1. - zcs - dcc[nlev - 1] * nclouds))
                 * dsigma[jl] * (dp / 101100.0) * (9.80665 / ga) * p->nrscat * p->newrsc;
        zrcsu[jl] = c0 * (1. - dcc[nlev - 1]) * dsigma[jl] * (dp / 101100.0) * (9.80665 / ga) * p->nrscat * p->newrsc;
    }

    double zta1 = 1., zta1s = 1., zra1 = 0., zra1s = 0.;
    double zta2 = 1., zta2s = 1., zra2 = 0., zra2s = 0.;
    double zto3t = 1.;
    double zo3 = zxo3t + zmbar * zo3t;
    double zto3tu = 1. - ao3(zo3) / p->zsolar1;
    double ztwvt = 1.;
    double zwv = zywvt + zbetta * zwvt;
    double ztwvtu = 1. - awv(zwv) / p->zsolar2;
    int newrsc = p->newrsc, nrscat = p->nrscat;
    zrcs[nlev - 1] = zrcs[nlev - 1] * newrsc;
    zrcsu[nlev - 1] = zrcsu[nlev - 1] * newrsc;
    double zscf = p->rcoeff * dp / 101100.0 * 9.80665 / ga;
    zrcsu[nlev - 1] = zrcsu[nlev - 1] + (1.0 - exp(zscf * log(1.0 - 0.144)))
                    * (1 - newrsc) * nrscat * (1 - dcc[nlev - 1] * nclouds);
    zrcs[nlev - 1] = zrcs[nlev - 1] + (1.0 - exp(zscf * log(1.0 - (0.219 / (1. + 0.816 * zmu0)))))
                   * zcs * (1 - newrsc) * nrscat
                   + (1.0 - exp(zscf * log(1.0 - 0.144))) * (1. - zcs - dcc[nlev - 1]) * nrscat * (1 - newrsc);

    for (int jl = 0; jl < nlev; jl++) {
        zt1[jl] = zta1; zt2[jl] = zta2; zr1s[jl] = zra1s; zr2s[jl] = zra2s;
        zrb1[jl] = zrcs[jl] + zrcl1[jl] * dcc[jl] * nclouds;
        zrb1s[jl] = zrcsu[jl] + zrcl1s[jl] * dcc[jl] * nclouds;
        zo3 = zxo3l[jl];
        double zto3 = (1. - ao3(zo3) / p->zsolar1) / zto3t;
        zto3t = zto3t * zto3;
        zo3 = zxo3t + zmbar * (zo3t - zo3l[jl]);
        double zto3u = zto3tu / (1. - ao3(zo3) / p->zsolar1);
        zto3tu = zto3tu / zto3u;
        ztb1[jl] = 1. - (1. - zto3) * (1. - dcc[jl]) - zrb1[jl];
        ztb1u[jl] = 1. - (1. - zto3u) * (1. - dcc[jl]) - zrb1s[jl];
        double z1mrabr = 1. / (1. - zra1s * zrb1s[jl]);
        zra1 = zra1 + zta1 * zrb1[jl] * zta1s * z1mrabr;
        zta1 = zta1 * ztb1[jl] * z1mrabr;
        zra1s = zrb1s[jl] + ztb1u[jl] * zra1s * ztb1[jl] * z1mrabr;
        zta1s = ztb1u[jl] * zta1s * z1mrabr;

        zrb2[jl] = zrcl2[jl] * dcc[jl] * nclouds;
        zrb2s[jl] = zrcl2s[jl] * dcc[jl] * nclouds;
        zwv = zywvl[jl];
        double ztwv = (1. - awv(zwv) / p->zsolar2) / ztwvt;
        ztwvt = ztwvt * ztwv;
        zwv = zywvt + zbetta * (zwvt - zwvl[jl]);
        double ztwvu = ztwvtu / (1. - awv(zwv) / p->zsolar2);
        ztwvtu = ztwvtu / ztwvu;
        ztb2[jl] = 1. - (1. - ztwv) * (1. - dcc[jl] * nclouds) - (1. - ztcl2[jl]) * dcc[jl] * nclouds;
        ztb2u[jl] = 1. - (1. - ztwvu) * (1. - dcc[jl] * nclouds) - (1. - ztcl2s[jl]) * dcc[jl] * nclouds;
        z1mrabr = 1. / (1. - zra2s * zrb2s[jl]);
        zra2 = zra2 + zta2 * zrb2[jl] * zta2s * z1mrabr;
        zta2 = zta2 * ztb2[jl] * z1mrabr;
        zra2s = zrb2s[jl] + ztb2u[jl] * zra2s * ztb2[jl] * z1mrabr;
        zta2s = ztb2u[jl] * zta2s * z1mrabr;
    }
    zt1[nlev] = zta1; zt2[nlev] = zta2; zr1s[nlev] = zra1s; zr2s[nlev] = zra2s;

    int nst = p->nstartemp, ne = p->necham, ne6 = p->necham6;
    zra1s = *dalb * (1 - nst) + dsalb[0] * nst;
    zra2s = *dalb * (1 - nst) + dsalb[1] * nst;
    double ocean3 = fmin(0.05 / (zmu0 + 0.15), 0.15);
    double ocean6 = (0.026 / (pow(zmu0, 1.7) + 0.065) + 0.15 * (zmu0 - 1) * (zmu0 - 0.5) * (zmu0 - 0.1) + 0.0082);
    for (int b = 0; b < 2; b++) {
        dsalb[b] = dls * dsalb[b] + (1. - dls) * dicec * dsalb[b]
                 + (1. - dls) * (1. - dicec) * ocean3 * ne * (1 - ne6)
                 + (1. - dls) * (1. - dicec) * (1 - ne) * ne6 * ocean6
                 + (1. - dls) * (1. - dicec) * (1. - ne) * (1 - ne6) * dsalb[b];
    }
    /* zsolars(1:2) hold the solarini split (radmod.f90:358-359) */
    *dalb = (p->zsolar1 * dsalb[0] + p->zsolar2 * dsalb[1]) * nst
          + (dls * *dalb + (1. - dls) * dicec * *dalb
             + (1. - dls) * (1. - dicec) * ocean3 * ne * (1 - ne6)
             + (1. - dls) * (1. - dicec) * (1 - ne) * ne6 * ocean6
             + (1. - dls) * (1. - dicec) * (1. - ne) * (1 - ne6) * *dalb) * (1 - nst);
    zra1 = dsalb[0] * nst + *dalb * (1 - nst);
    zra2 = dsalb[1] * nst + *dalb * (1 - nst);

    for (int jl = nlev - 1; jl >= 0; jl--) {
        zrl1[jl + 1] = zra1; zrl2[jl + 1] = zra2; zrl1s[jl + 1] = zra1s; zrl2s[jl + 1] = zra2s;
        zra1 = zrb1[jl] + ztb1[jl] * zra1 * ztb1u[jl] / (1. - zra1s * zrb1s[jl]);
        zra1s = zrb1s[jl] + ztb1u[jl] * zra1s * ztb1u[jl] / (1. - zra1s * zrb1s[jl]);
        zra2 = zrb2[jl] + ztb2[jl] * zra2 * ztb2u[jl] / (1. - zra2s * zrb2s[jl]);
        zra2s = zrb2s[jl] + ztb2u[jl] * zra2s * ztb2u[jl] / (1. - zra2s * zrb2s[jl]);
    }
    zrl1[0] = zra1; zrl2[0] = zra2; zrl1s[0] = zra1s; zrl2s[0] = zra2s;

    for (int jl = 0; jl < nlep; jl++) {
        double z1mrabr = 1. / (1. - zr1s[jl] * zrl1s[jl]);
        double zfd1 = zt1[jl] * z1mrabr;
        double zfu1 = -zt1[jl] * zrl1[jl] * z1mrabr;
        z1mrabr = 1. / (1. - zr2s[jl] * zrl2s[jl]);
        double zfd2 = zt2[jl] * z1mrabr;
        double zfu2 = -zt2[jl] * zrl2[jl] * z1mrabr;
        dfu[jl] = zfu1 * zftop1 + zfu2 * zftop2;
        dfd[jl] = zfd1 * zftop1 + zfd2 * zftop2;
        dswfl[jl] = dfu[jl] + dfd[jl];
    }
}

/* SUBROUTINE LWR for one column, radmod.f90:2122-2456 */
static void lwr_col(const oracle_radpar *p, int nlev, double dp, double dls,
                    const double *dt, const double *dq, const double *dcc,
                    const double *dql, const double *dqo3, const double *dqco2,
                    double *dftu, double *dftd, double *dlwfl) {
    const double SBK = 5.67e-8;
    const double zmmair = 0.0289644, zmmco2 = 0.0440098, zpv2pm = zmmco2 / zmmair;
    const double zrco2 = 1.9635, zro3 = 2.14, zttop = 0.;
    const double zfh2o = 0.1, zfco2 = 100. / zrco2, zfo3 = 100. / zro3;
    const double *sigma = p->sigma, *sigmah = p->sigmah, *dsigma = p->dsigma;
    const double ga = p->ga;
    int nlep = nlev + 1, nlem = nlev - 1;
    double zbu[nlep + 1], zbd[nlep + 1]; /* index 0..NLEP */
    double zst4h[nlep], zst4[nlep];
    double ztau[nlev], zq[nlev], zqo3[nlev], zqco2[nlev], ztausf[nlev], ztaucs[nlev], ztaucc0[nlev];
    double zsigh2[nlep];
    const double zero = 1.e-6;
    double zao30 = 0.209 * pow(7.e-5, 0.436);
    double zco20 = 0.0676 * pow(0.01022, 0.421);
    double zh2o0a = 0.846 * pow(3.59e-5, 0.243);
    double zh2o0 = 0.832 * pow(0.0286, 0.26);
    double zao3c = 0.209 * pow(0.01 + 7.e-5, 0.436) - zao30 - 0.0212 * log10(0.01);
    double zaco2c = 0.0676 * pow(1.01022, 0.421) - zco20;
    double zah2oc = 0.846 * pow(0.01 + 3.59e-5, 0.243) - zh2o0a - 0.24 * log10(0.02);
    double zth2oc = 1. - (0.832 * pow(2. + 0.0286, 0.26) - zh2o0) + 0.1196 * log(2. - 0.6931);
    zsigh2[0] = 0.;
    for (int k = 1; k < nlep; k++) zsigh2[k] = sigmah[k - 1] * sigmah[k - 1];
    (void)zsigh2;
    double zps2 = (p->npbroaden > 0.5) ? dp * dp : 101100.0 * 101100.0;

    for (int k = 0; k < nlep; k++) { dftu[k] = 0.; dftd[k] = 0.; }
    for (int k = 0; k < nlep; k++) { double t2 = dt[k] * dt[k]; zst4[k] = SBK * (t2 * t2); }
    /* Fortran 1-based: zst4h(1) .. zst4h(NLEP) -> index k-1 */
    zst4h[0] = zst4[0] - (zst4[0] - zst4[1]) * sigma[0] / (sigma[0] - sigma[1]);
    for (int jlev = 2; jlev <= nlev; jlev++) {
        int jlem = jlev - 1;
        zst4h[jlev - 1] = (zst4[jlev - 1] * (sigma[jlem - 1] - sigmah[jlem - 1])
                         + zst4[jlem - 1] * (sigmah[jlem - 1] - sigma[jlev - 1]))
                        / (sigma[jlem - 1] - sigma[jlev - 1]);
    }
    if ((zst4[nlev - 1] - zst4h[nlev - 1]) * (zst4[nlev - 1] - zst4[nlep - 1]) > 0.)
        zst4h[nlep - 1] = zst4[nlep - 1];
    else
        zst4h[nlep - 1] = zst4[nlev - 1] + (zst4[nlev - 1] - zst4[nlem - 1]) * (1. - sigma[nlev - 1])
                                          / (sigma[nlev - 1] - sigma[nlem - 1]);

    zbd[0] = SBK * (zttop * zttop * zttop * zttop);
    double zeps = dls + 0.98 * (1. - dls);
    zbu[nlep] = zeps * zst4[nlep - 1];

    for (int jlev = 1; jlev <= nlev; jlev++) {
        double zzf1 = sigma[jlev - 1] * dsigma[jlev - 1] / ga / 100000.;
        double zzf2 = zpv2pm * 1.e-6;
        double zzf3 = -1.66 * p->acllwr * 1000. * dsigma[jlev - 1] / ga;
        double zsfac = zzf1 * zps2;
        zq[jlev - 1] = zfh2o * zsfac * dq[jlev - 1];
        zqo3[jlev - 1] = zfo3 * zsfac * dqo3[jlev - 1];
        zqco2[jlev - 1] = zfco2 * zzf2 * zsfac * dqco2[jlev - 1];
        if (p->clgray > 0) ztaucc0[jlev - 1] = 1. - dcc[jlev - 1] * p->clgray;
        else ztaucc0[jlev - 1] = 1. - dcc[jlev - 1] * (1. - exp(zzf3 * dql[jlev - 1] * dp));
    }

    for (int jlev = 1; jlev <= nlev; jlev++) {
        int jlem = jlev - 1;
        double ztaucc = 1., zsumwv = 0., zsumo3 = 0., zsumco2 = 0.;
        for (int jlev2 = jlev; jlev2 <= nlev; jlev2++) {
            zsumwv = zsumwv + zq[jlev2 - 1];
            zsumo3 = zsumo3 + zqo3[jlev2 - 1];
            zsumco2 = zsumco2 + zqco2[jlev2 - 1];
            double zah2o, zaco2, zth2o, zao3;
            if (zsumwv <= 0.01) zah2o = 0.846 * pow(zsumwv + 3.59e-5, 0.243) - zh2o0a;
            else zah2o = 0.24 * log10(zsumwv + 0.01) + zah2oc;
            if (p->th2oc > 0.) zah2o = fmin(zah2o + (1. - exp(-p->th2oc * zsumwv)), 1.);
            if (zsumco2 <= 1.0) zaco2 = 0.0676 * pow(zsumco2 + 0.01022, 0.421) - zco20;
            else zaco2 = 0.0546 * log10(zsumco2) + zaco2c;
            if (zsumwv <= 2.) zth2o = 1. - (0.832 * pow(zsumwv + 0.0286, 0.26) - zh2o0);
            else zth2o = fmax(0., zth2oc - 0.1196 * log(zsumwv - 0.6931));
            if (zsumo3 <= 0.01) zao3 = 0.209 * pow(zsumo3 + 7.e-5, 0.436) - zao30;
            else zao3 = 0.0212 * log10(zsumo3) + zao3c;
            double tcs = 1. - zah2o - zao3 - zaco2 * zth2o;
            tcs = fmin(1. - zero, fmax(zero, tcs));
            ztaucs[jlev2 - 1] = tcs;
            ztaucc = ztaucc * ztaucc0[jlev2 - 1];
            ztau[jlev2 - 1] = tcs * ztaucc;
        }
        if (jlev == 1) {
            double ztau0 = 1. - zero;
            for (int jlev2 = 1; jlev2 <= nlev; jlev2++) {
                int jlep2 = jlev2 + 1;
                ztau0 = ztaucs[jlev2 - 1] / ztau0 * ztaucc0[jlev2 - 1] * p->tpofmt;
                ztau0 = fmin(1. - zero, fmax(zero, ztau0));
                if ((zst4[jlev2 - 1] - zst4h[jlev2 - 1]) * (zst4[jlev2 - 1] - zst4h[jlep2 - 1]) > 0.) {
                    zbd[jlev2] = 0.5 * zst4[jlev2 - 1] + 0.25 * (zst4h[jlev2 - 1] + zst4h[jlep2 - 1]);
                    zbu[jlev2] = zbd[jlev2];
                } else {
                    zbd[jlev2] = (zst4h[jlep2 - 1] - ztau0 * zst4h[jlev2 - 1]) / (1. - ztau0)
                               - (zst4h[jlev2 - 1] - zst4h[jlep2 - 1]) / log(ztau0);
                    zbu[jlev2] = zst4h[jlev2 - 1] + zst4h[jlep2 - 1] - zbd[jlev2];
                }
                ztau0 = ztaucs[jlev2 - 1];
            }
        }
        dftu[jlev - 1] = dftu[jlev - 1] - zbu[jlev];
        dftd[jlev - 1] = dftd[jlev - 1] + zbd[jlem];
        double zbdl = zbd[jlem] - zbd[jlev];
        for (int jlev2 = jlev; jlev2 <= nlev; jlev2++) {
            int jlep2 = jlev2 + 1;
            dftu[jlev - 1] = dftu[jlev - 1] - (zbu[jlep2] - zbu[jlev2]) * ztau[jlev2 - 1];
            dftd[jlep2 - 1] = dftd[jlep2 - 1] + zbdl * ztau[jlev2 - 1];
        }
        ztausf[jlev - 1] = ztau[nlev - 1];
    }
    dftu[nlep - 1] = dftu[nlep - 1] - zbu[nlep];
    dftd[nlep - 1] = dftd[nlep - 1] + zbd[nlev];
    zeps = (1. - zeps) * dftd[nlep - 1];
    for (int jlev = 1; jlev <= nlev; jlev++) dftu[jlev - 1] = dftu[jlev - 1] - ztausf[jlev - 1] * zeps;
    for (int k = 0; k < nlep; k++) dlwfl[k] = dftu[k] + dftd[k];
}

/* SUBROUTINE RADSTEP, radmod.f90:927-1110 (ndiagcf = 0, nradice = 1), for
 * columns j0..j1-1; with ndcycle = 0 the range must cover whole latitude rows */
void oracle_radstep_range(const oracle_radpar *p, oracle_radio *io, int j0, int j1) {
    int nlev = p->nlev, nhor = p->nhor, nlon = p->nlon, nlep = nlev + 1;
    if (p->nsol == 1) oracle_solang_range(p, io->sid, io->cola, io->gmu0, j0, j1);
    if (p->no3 == 1) oracle_mko3_range(p, io->sid, io->dt, io->dp, io->dqo3, j0, j1);
    double *zmu0 = malloc(sizeof(double) * nhor), *zmu1 = malloc(sizeof(double) * nhor);
    if (p->ndcycle == 0) { /* zonal means, radmod.f90:1650-1665 */
        for (int js = j0; js < j1; js += nlon) {
            int icnt = 0;
            double zsum = 0.0;
            for (int j = js; j < js + nlon; j++) if (io->gmu0[j] > 0.0) icnt++;
            for (int j = js; j < js + nlon; j++) zsum += io->gmu0[j];
            for (int j = js; j < js + nlon; j++) {
                zmu0[j] = icnt > 0 ? zsum / icnt : 0.0;
                zmu1[j] = icnt > 0 ? zsum / nlon : 0.0;
            }
        }
    } else {
        for (int j = j0; j < j1; j++) { zmu0[j] = io->gmu0[j]; zmu1[j] = io->gmu0[j]; }
    }
    double c_dt[nlep], c_dq[nlep], c_dcc[nlep], c_dql[nlep], c_o3[nlev], c_co2[nlev];
    double fu[nlep], fd[nlep], sw[nlep], ftu[nlep], ftd[nlep], lw[nlep];
    for (int j = j0; j < j1; j++) {
        for (int k = 0; k < nlep; k++) {
            c_dt[k] = io->dt[(size_t)k * nhor + j];
            c_dq[k] = io->dq[(size_t)k * nhor + j];
            c_dcc[k] = io->dcc[(size_t)k * nhor + j];
            c_dql[k] = io->dql[(size_t)k * nhor + j];
        }
        for (int k = 0; k < nlev; k++) {
            c_o3[k] = io->dqo3[(size_t)k * nhor + j];
            c_co2[k] = io->dqco2[(size_t)k * nhor + j];
        }
        double dp = io->dp[j];
        for (int k = 0; k < nlep; k++) { fu[k] = fd[k] = sw[k] = ftu[k] = ftd[k] = lw[k] = 0.0; }
        if (p->nswr == 1)
            swr_col(p, nlev, zmu0[j], zmu1[j], dp, &io->dalb[j], &io->dsalb[2 * j], io->dls[j], io->dicec[j],
                    c_dq, c_dql, c_dcc, c_o3, c_dt, fu, fd, sw);
        if (p->nlwr == 1)
            lwr_col(p, nlev, dp, io->dls[j], c_dt, c_dq, c_dcc, c_dql, c_o3, c_co2, ftu, ftd, lw);
        double fl[nlep], zdh[nlev];
        for (int k = 0; k < nlep; k++) fl[k] = lw[k] + sw[k];
        for (int jlev = nlev; jlev >= 2; jlev--)
            zdh[jlev - 1] = -c_dt[jlev - 1] * p->gascon / p->ga * log(p->sigmah[jlev - 2] / p->sigmah[jlev - 1]);
        zdh[0] = -c_dt[0] * p->gascon / p->ga * log(p->sigma[0] / p->sigmah[0]) * 0.5;
        for (int k = 0; k < nlep; k++) {
            size_t o = (size_t)k * nhor + j;
            io->dfu[o] = fu[k]; io->dfd[o] = fd[k]; io->dswfl[o] = sw[k];
            io->dftu[o] = ftu[k]; io->dftd[o] = ftd[k]; io->dlwfl[o] = lw[k];
            io->dflux[o] = fl[k];
        }
        for (int jlev = 1; jlev <= nlev; jlev++) {
            int jlep = jlev + 1;
            size_t o = (size_t)(jlev - 1) * nhor + j;
            double den = p->dsigma[jlev - 1] * dp * p->acpd * (1. + p->adv * c_dq[jlev - 1]);
            double zdtdt = -(p->ga * (fl[jlep - 1] - fl[jlev - 1]) / den);
            io->dtdt[o] = io->dtdt[o] + zdtdt;
            io->dtdtswr[o] = -(p->ga * (sw[jlep - 1] - sw[jlev - 1]) / den);
            io->dtdtlwr[o] = -(p->ga * (lw[jlep - 1] - lw[jlev - 1]) / den);
            io->dconv[o] = (fl[jlev - 1] - fl[jlep - 1]) / (zdh[jlev - 1] + 1.0e-9);
        }
    }
    free(zmu0);
    free(zmu1);
}

void oracle_radstep(const oracle_radpar *p, oracle_radio *io) {
    oracle_radstep_range(p, io, 0, p->nhor);
}
