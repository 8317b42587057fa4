/*
 * Oracle (test infrastructure): FP64 restatement of gaussmod.f90, legmod.f90,
 * fftmod.f90 and the fft991mod.f90 transform contract.  Loop order and
 * operation order follow the reference so that FP64 rounding agrees with an
 * 8-byte (-fdefault-real-8) build to the last few ulps.  Compiled with
 * -O2 -ffp-contract=off; never linked into the product library.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "exo_oracle.h"

/* ===================== gaussmod.f90 ===================== */

/* FUNCTION QL, gaussmod.f90:46-69 */
static double ql(int k, double p) {
    double z0 = acos(p), z1 = 1.0, z2 = 0.0, z3 = 0.0, z4;
    for (int j = k; j >= 0; j -= 2) {
        z3 = z1 * cos(z0 * j);
        z2 = z2 + z3;
        z4 = (double)((k - j + 1) * (k + j)) * 0.5;
        z1 = z1 * z4 / (z4 + (j - 1));
    }
    if (k % 2 == 0) z2 = z2 - 0.5 * z3;
    z0 = sqrt(2.0);
    for (int j = 1; j <= k; j++) z0 = z0 * sqrt(1.0 - 0.25 / (double)(j * j));
    return z0 * z2;
}

/* FUNCTION QLD, gaussmod.f90:75-86 */
static double qld(int k, double p) {
    double z = p * ql(k, p) - sqrt((k + k + 1.0) / (k + k - 1.0)) * ql(k - 1, p);
    return (p * p - 1.0) / (k * z);
}

/* SUBROUTINE INIGAU, gaussmod.f90:5-40 */
void oracle_inigau(int klat, double *pz0, double *pzw) {
    const double PI = 3.14159265358979;
    const double ZEPS = 1.0e-16;
    double z0 = PI / (2 * klat + 1);
    double z1 = 1.0 / (double)(klat * klat * 8);
    double z4 = 2.0 / (double)(klat * klat);
    for (int jlat = 1; jlat <= klat / 2; jlat++) {
        double z2 = z0 * (2 * jlat - 0.5);
        z2 = cos(z2 + z1 / tan(z2));
        for (int jiter = 1; jiter <= 50; jiter++) {
            double z3 = ql(klat, z2) * qld(klat, z2);
            z2 = z2 - z3;
            if (fabs(z3) < ZEPS) break;
        }
        double z5 = ql(klat - 1, z2) / sqrt(klat - 0.5);
        pz0[jlat - 1] = z2;
        pzw[jlat - 1] = z4 * (1.0 - z2 * z2) / (z5 * z5);
        pz0[klat - jlat] = -z2;
        pzw[klat - jlat] = pzw[jlat - 1];
    }
}

/* ===================== legmod.f90 ===================== */

/* SUBROUTINE LEGINI, legmod.f90:30-171 (tables for all NLPP = NLAT rows) */
int oracle_legini(oracle_leg *L, int nlat, int nfilter, int ngptfilter,
                  int nspvfilter, double landhoskn0, double filterkappa,
                  int nfilterexp, int pyfft_nfs) {
    int nlon = 2 * nlat, ntru = (nlon - 1) / 3, ntp1 = ntru + 1;
    int ncsp = (ntru + 1) * (ntru + 2) / 2;
    memset(L, 0, sizeof(*L));
    L->ntru = ntru; L->nlat = nlat; L->nlon = nlon; L->ncsp = ncsp;
    L->sid = malloc(sizeof(double) * nlat);
    L->gwd = malloc(sizeof(double) * nlat);
    double **tabs[8] = {&L->qi, &L->qj, &L->qc, &L->qe, &L->qm, &L->qq, &L->qu, &L->qv};
    for (int t = 0; t < 8; t++) *tabs[t] = malloc(sizeof(double) * (size_t)ncsp * nlat);
    L->skgpsp = malloc(sizeof(double) * ntp1);
    L->skspgp = malloc(sizeof(double) * ntp1);
    oracle_inigau(nlat, L->sid, L->gwd);

    double *zpli = malloc(sizeof(double) * ncsp);
    double *zpld = malloc(sizeof(double) * ncsp);
#define ZPLI(i) zpli[(i) - 1]
#define ZPLD(i) zpld[(i) - 1]
    for (int jlat = 1; jlat <= nlat; jlat++) {
        double zgwd = L->gwd[jlat - 1];
        double zsin = L->sid[jlat - 1];
        double zcsq = 1.0 - zsin * zsin;
        double zgwdcsq = zgwd / zcsq;
        double f1m = sqrt(1.5), f2m, amsq, z1, z2, z3;
        ZPLI(1) = sqrt(0.5);
        ZPLI(2) = f1m * zsin;
        ZPLD(1) = 0.0;
        int lm = 2;
        for (int m = 0; m <= ntru; m++) {
            if (m > 0) {
                lm = lm + 1;
                f2m = -f1m * sqrt(zcsq / (double)(m + m));
                f1m = f2m * sqrt(m + m + 3.0);
                ZPLI(lm) = f2m;
                if (lm < ncsp) {
                    lm = lm + 1;
                    ZPLI(lm) = f1m * zsin;
                    ZPLD(lm - 1) = -m * f2m * zsin;
                }
            }
            amsq = (double)(m * m);
            for (int n = m + 2; n <= ntru; n++) {
                lm = lm + 1;
                z1 = sqrt(((n - 1) * (n - 1) - amsq) / (double)(4 * (n - 1) * (n - 1) - 1));
                z2 = zsin * ZPLI(lm - 1) - z1 * ZPLI(lm - 2);
                ZPLI(lm) = z2 * sqrt((4 * n * n - 1) / (n * n - amsq));
                ZPLD(lm - 1) = (1 - n) * z2 + n * z1 * ZPLI(lm - 2);
            }
            if (lm < ncsp) {
                z3 = sqrt((ntru * ntru - amsq) / (double)(4 * ntru * ntru - 1));
                ZPLD(lm) = -ntru * zsin * ZPLI(lm) + (ntru + ntru + 1) * ZPLI(lm - 1) * z3;
            } else {
                ZPLD(lm) = -ntru * zsin * ZPLI(lm);
            }
        }
        lm = 0;
        size_t off = (size_t)(jlat - 1) * ncsp;
        for (int m = 0; m <= ntru; m++) {
            for (int n = m; n <= ntru; n++) {
                lm = lm + 1;
                double znn1 = 0.0;
                if (n > 0) znn1 = 1.0 / (double)(n * (n + 1));
                L->qi[off + lm - 1] = ZPLI(lm);
                L->qj[off + lm - 1] = ZPLD(lm);
                L->qc[off + lm - 1] = ZPLI(lm) * zgwd;
                L->qu[off + lm - 1] = ZPLI(lm) * znn1 * m;
                L->qv[off + lm - 1] = ZPLD(lm) * znn1;
                L->qe[off + lm - 1] = ZPLD(lm) * zgwdcsq;
                L->qq[off + lm - 1] = ZPLI(lm) * zgwdcsq * n * (n + 1) * 0.5;
                L->qm[off + lm - 1] = ZPLI(lm) * zgwdcsq * m;
            }
        }
    }
#undef ZPLI
#undef ZPLD
    free(zpli);
    free(zpld);

    /* physics filters, legmod.f90:124-155; index n is 1-based as in Fortran */
    for (int n = 1; n <= ntp1; n++) {
        double g = 1.0, s = 1.0, rn = (double)n;
        if (pyfft_nfs >= 0) {
            /* pyfft.f90:152-156: the pyfft module is compiled without
             * -fdefault-real-8, so real(n) and the exponential are 4-byte */
            float x = (float)n / (float)ntru;
            float x2 = x * x, x4 = x2 * x2, x8 = x4 * x4;
            float f = expf(-8.0f * x8);
            g = s = (double)(1 - pyfft_nfs) * 1.0 + (double)pyfft_nfs * (double)f;
        } else if (nfilter == 1) {
            g = (1 - ngptfilter) * g + ngptfilter * (1.0 - rn / ntp1);
            s = (1 - nspvfilter) * s + nspvfilter * (1.0 - rn / ntp1);
        } else if (nfilter == 2) {
            g = (1 - ngptfilter) * g + ngptfilter * exp(-filterkappa * pow(rn / ntru, nfilterexp));
            s = (1 - nspvfilter) * s + nspvfilter * exp(-filterkappa * pow(rn / ntru, nfilterexp));
        } else if (nfilter == 3) {
            double r = rn * (double)(n + 1) / (landhoskn0 * (landhoskn0 + 1));
            g = (1 - ngptfilter) * g + ngptfilter * exp(-(r * r));
            s = (1 - nspvfilter) * s + nspvfilter * exp(-(r * r));
        } else if (nfilter == 4) {
            double r = 1.0 - rn / ntp1;
            g = (1 - ngptfilter) * g + ngptfilter * (r * r);
            s = (1 - nspvfilter) * s + nspvfilter * (r * r);
        }
        L->skgpsp[n - 1] = g;
        L->skspgp[n - 1] = s;
    }
    return 0;
}

void oracle_legfree(oracle_leg *L) {
    free(L->sid); free(L->gwd);
    free(L->qi); free(L->qj); free(L->qc); free(L->qe);
    free(L->qm); free(L->qq); free(L->qu); free(L->qv);
    free(L->skgpsp); free(L->skspgp);
    memset(L, 0, sizeof(*L));
}

/* index helpers, 1-based like the Fortran */
#define FC(a, c, m, l) (a)[(size_t)((l) - 1) * nlon + 2 * ((m) - 1) + (c) - 1]
#define FC4(a, c, m, l, v) (a)[((size_t)((v) - 1) * nlat + ((l) - 1)) * nlon + 2 * ((m) - 1) + (c) - 1]
#define SP(a, c, w) (a)[2 * ((w) - 1) + (c) - 1]
#define SP3(a, c, w, v) (a)[(size_t)((v) - 1) * nrsp + 2 * ((w) - 1) + (c) - 1]
#define Q(t, w, l) (t)[(size_t)((l) - 1) * ncsp + (w) - 1]

/* SUBROUTINE SP2FC, legmod.f90:230-255 (and SP2FCDMU :262-287 with qj) */
static void sp2fc_tab(const oracle_leg *L, const double *tab, const double *sp, double *fc) {
    int nlat = L->nlat, nlon = L->nlon, ncsp = L->ncsp, ntp1 = L->ntru + 1;
    memset(fc, 0, sizeof(double) * (size_t)nlat * nlon);
    for (int l = 1; l <= nlat; l++) {
        int w = 1;
        for (int m = 1; m <= ntp1; m++)
            for (int n = m; n <= ntp1; n++) {
                FC(fc, 1, m, l) = FC(fc, 1, m, l) + Q(tab, w, l) * SP(sp, 1, w) * L->skspgp[n - 1];
                FC(fc, 2, m, l) = FC(fc, 2, m, l) + Q(tab, w, l) * SP(sp, 2, w) * L->skspgp[n - 1];
                w = w + 1;
            }
    }
}
void oracle_sp2fc(const oracle_leg *L, const double *sp, double *fc) { sp2fc_tab(L, L->qi, sp, fc); }
void oracle_sp2fcdmu(const oracle_leg *L, const double *sp, double *fc) { sp2fc_tab(L, L->qj, sp, fc); }

/* SUBROUTINE FC2SP, legmod.f90:178-223 */
void oracle_fc2sp(const oracle_leg *L, const double *fc, double *sp, int folded) {
    int nlat = L->nlat, nlon = L->nlon, ncsp = L->ncsp, ntp1 = L->ntru + 1;
    const double *qc = L->qc, *f = L->skgpsp;
    memset(sp, 0, sizeof(double) * 2 * (size_t)ncsp);
    if (!folded) {
        for (int l = 1; l <= nlat; l++) {
            int w = 1;
            for (int m = 1; m <= ntp1; m++)
                for (int n = m; n <= ntp1; n++) {
                    SP(sp, 1, w) = SP(sp, 1, w) + Q(qc, w, l) * FC(fc, 1, m, l) * f[n - 1];
                    SP(sp, 2, w) = SP(sp, 2, w) + Q(qc, w, l) * FC(fc, 2, m, l) * f[n - 1];
                    w = w + 1;
                }
        }
    } else {
        for (int l = 1; l <= nlat / 2; l++) {
            int w = 1, k = nlat + 1 - l;
            for (int m = 1; m <= ntp1; m++)
                for (int n = m; n <= ntp1; n++) {
                    if ((m + n) % 2 == 0) {
                        SP(sp, 1, w) = SP(sp, 1, w) + Q(qc, w, l) * (FC(fc, 1, m, l) + FC(fc, 1, m, k)) * f[n - 1];
                        SP(sp, 2, w) = SP(sp, 2, w) + Q(qc, w, l) * (FC(fc, 2, m, l) + FC(fc, 2, m, k)) * f[n - 1];
                    } else {
                        SP(sp, 1, w) = SP(sp, 1, w) + Q(qc, w, l) * (FC(fc, 1, m, l) - FC(fc, 1, m, k)) * f[n - 1];
                        SP(sp, 2, w) = SP(sp, 2, w) + Q(qc, w, l) * (FC(fc, 2, m, l) - FC(fc, 2, m, k)) * f[n - 1];
                    }
                    w = w + 1;
                }
        }
    }
}

/* SUBROUTINE DV2UV, legmod.f90:312-349 */
void oracle_dv2uv(const oracle_leg *L, const double *pd, double *pz,
                  double *pu, double *pv, int nlev, double plavor) {
    int nlat = L->nlat, nlon = L->nlon, ncsp = L->ncsp, ntp1 = L->ntru + 1, nrsp = 2 * ncsp;
    const double *qu = L->qu, *qv = L->qv, *f = L->skspgp;
    memset(pu, 0, sizeof(double) * (size_t)nlat * nlon * nlev);
    memset(pv, 0, sizeof(double) * (size_t)nlat * nlon * nlev);
    for (int v = 1; v <= nlev; v++) {
        double zsave = SP3(pz, 1, 2, v);
        SP3(pz, 1, 2, v) = zsave - plavor;
        for (int l = 1; l <= nlat; l++) {
            int w = 1;
            for (int m = 1; m <= ntp1; m++)
                for (int n = m; n <= ntp1; n++) {
                    double fn = f[n - 1];
                    FC4(pu, 1, m, l, v) = FC4(pu, 1, m, l, v) + Q(qv, w, l) * SP3(pz, 1, w, v) * fn + Q(qu, w, l) * SP3(pd, 2, w, v) * fn;
                    FC4(pu, 2, m, l, v) = FC4(pu, 2, m, l, v) + Q(qv, w, l) * SP3(pz, 2, w, v) * fn - Q(qu, w, l) * SP3(pd, 1, w, v) * fn;
                    FC4(pv, 1, m, l, v) = FC4(pv, 1, m, l, v) + Q(qu, w, l) * SP3(pz, 2, w, v) * fn - Q(qv, w, l) * SP3(pd, 1, w, v) * fn;
                    FC4(pv, 2, m, l, v) = FC4(pv, 2, m, l, v) - Q(qu, w, l) * SP3(pz, 1, w, v) * fn - Q(qv, w, l) * SP3(pd, 2, w, v) * fn;
                    w = w + 1;
                }
        }
        SP3(pz, 1, 2, v) = zsave;
    }
}

/* SUBROUTINE UV2DV, legmod.f90:356-426 */
void oracle_uv2dv(const oracle_leg *L, const double *pu, const double *pv,
                  double *pd, double *pz, int nlev, int folded) {
    int nlat = L->nlat, nlon = L->nlon, ncsp = L->ncsp, ntp1 = L->ntru + 1, nrsp = 2 * ncsp;
    const double *qe = L->qe, *qm = L->qm, *f = L->skgpsp;
    memset(pd, 0, sizeof(double) * (size_t)nrsp * nlev);
    memset(pz, 0, sizeof(double) * (size_t)nrsp * nlev);
    for (int v = 1; v <= nlev; v++) {
        if (!folded) {
            for (int l = 1; l <= nlat; l++) {
                int w = 1;
                for (int m = 1; m <= ntp1; m++)
                    for (int n = m; n <= ntp1; n++) {
                        double fn = f[n - 1];
                        SP3(pz, 1, w, v) = SP3(pz, 1, w, v) + Q(qe, w, l) * FC4(pu, 1, m, l, v) * fn - Q(qm, w, l) * FC4(pv, 2, m, l, v) * fn;
                        SP3(pz, 2, w, v) = SP3(pz, 2, w, v) + Q(qe, w, l) * FC4(pu, 2, m, l, v) * fn + Q(qm, w, l) * FC4(pv, 1, m, l, v) * fn;
                        SP3(pd, 1, w, v) = SP3(pd, 1, w, v) - Q(qe, w, l) * FC4(pv, 1, m, l, v) * fn - Q(qm, w, l) * FC4(pu, 2, m, l, v) * fn;
                        SP3(pd, 2, w, v) = SP3(pd, 2, w, v) - Q(qe, w, l) * FC4(pv, 2, m, l, v) * fn + Q(qm, w, l) * FC4(pu, 1, m, l, v) * fn;
                        w = w + 1;
                    }
            }
        } else {
            for (int l = 1; l <= nlat / 2; l++) {
                int k = nlat + 1 - l, w = 1;
                for (int m = 1; m <= ntp1; m++)
                    for (int n = m; n <= ntp1; n++) {
                        double fn = f[n - 1];
                        if ((m + n) % 2 == 0) {
                            SP3(pz, 1, w, v) = SP3(pz, 1, w, v) + Q(qe, w, l) * (FC4(pu, 1, m, l, v) - FC4(pu, 1, m, k, v)) * fn
                                                                - Q(qm, w, l) * (FC4(pv, 2, m, l, v) + FC4(pv, 2, m, k, v)) * fn;
                            SP3(pz, 2, w, v) = SP3(pz, 2, w, v) + Q(qe, w, l) * (FC4(pu, 2, m, l, v) - FC4(pu, 2, m, k, v)) * fn
                                                                + Q(qm, w, l) * (FC4(pv, 1, m, l, v) + FC4(pv, 1, m, k, v)) * fn;
                            SP3(pd, 1, w, v) = SP3(pd, 1, w, v) - Q(qe, w, l) * (FC4(pv, 1, m, l, v) - FC4(pv, 1, m, k, v)) * fn
                                                                - Q(qm, w, l) * (FC4(pu, 2, m, l, v) + FC4(pu, 2, m, k, v)) * fn;
                            SP3(pd, 2, w, v) = SP3(pd, 2, w, v) - Q(qe, w, l) * (FC4(pv, 2, m, l, v) - FC4(pv, 2, m, k, v)) * fn
                                                                + Q(qm, w, l) * (FC4(pu, 1, m, l, v) + FC4(pu, 1, m, k, v)) * fn;
                        } else {
                            SP3(pz, 1, w, v) = SP3(pz, 1, w, v) + Q(qe, w, l) * (FC4(pu, 1, m, l, v) + FC4(pu, 1, m, k, v)) * fn
                                                                - Q(qm, w, l) * (FC4(pv, 2, m, l, v) - FC4(pv, 2, m, k, v)) * fn;
                            SP3(pz, 2, w, v) = SP3(pz, 2, w, v) + Q(qe, w, l) * (FC4(pu, 2, m, l, v) + FC4(pu, 2, m, k, v)) * fn
                                                                + Q(qm, w, l) * (FC4(pv, 1, m, l, v) - FC4(pv, 1, m, k, v)) * fn;
                            SP3(pd, 1, w, v) = SP3(pd, 1, w, v) - Q(qe, w, l) * (FC4(pv, 1, m, l, v) + FC4(pv, 1, m, k, v)) * fn
                                                                - Q(qm, w, l) * (FC4(pu, 2, m, l, v) - FC4(pu, 2, m, k, v)) * fn;
                            SP3(pd, 2, w, v) = SP3(pd, 2, w, v) - Q(qe, w, l) * (FC4(pv, 2, m, l, v) + FC4(pv, 2, m, k, v)) * fn
                                                                + Q(qm, w, l) * (FC4(pu, 1, m, l, v) - FC4(pu, 1, m, k, v)) * fn;
                        }
                        w = w + 1;
                    }
            }
        }
    }
}

/* SUBROUTINE QTEND, legmod.f90:433-499 */
void oracle_qtend(const oracle_leg *L, double *q, const double *qn,
                  const double *uq, const double *vq, int nlev, int folded) {
    int nlat = L->nlat, nlon = L->nlon, ncsp = L->ncsp, ntp1 = L->ntru + 1, nrsp = 2 * ncsp;
    const double *qe = L->qe, *qm = L->qm, *qc = L->qc, *f = L->skgpsp;
    memset(q, 0, sizeof(double) * (size_t)nrsp * nlev);
    for (int v = 1; v <= nlev; v++) {
        if (!folded) {
            for (int l = 1; l <= nlat; l++) {
                int w = 1;
                for (int m = 1; m <= ntp1; m++)
                    for (int n = m; n <= ntp1; n++) {
                        double fn = f[n - 1];
                        SP3(q, 1, w, v) = SP3(q, 1, w, v) + Q(qe, w, l) * FC4(vq, 1, m, l, v) * fn
                                        + Q(qc, w, l) * FC4(qn, 1, m, l, v) * fn + Q(qm, w, l) * FC4(uq, 2, m, l, v) * fn;
                        SP3(q, 2, w, v) = SP3(q, 2, w, v) + Q(qe, w, l) * FC4(vq, 2, m, l, v) * fn
                                        + Q(qc, w, l) * FC4(qn, 2, m, l, v) * fn - Q(qm, w, l) * FC4(uq, 1, m, l, v) * fn;
                        w = w + 1;
                    }
            }
        } else {
            for (int l = 1; l <= nlat / 2; l++) {
                int k = nlat + 1 - l, w = 1;
                for (int m = 1; m <= ntp1; m++)
                    for (int n = m; n <= ntp1; n++) {
                        double fn = f[n - 1];
                        if ((m + n) % 2 == 0) {
                            SP3(q, 1, w, v) = SP3(q, 1, w, v) + Q(qe, w, l) * (FC4(vq, 1, m, l, v) - FC4(vq, 1, m, k, v)) * fn
                                            + Q(qc, w, l) * (FC4(qn, 1, m, l, v) + FC4(qn, 1, m, k, v)) * fn
                                            + Q(qm, w, l) * (FC4(uq, 2, m, l, v) + FC4(uq, 2, m, k, v)) * fn;
                            SP3(q, 2, w, v) = SP3(q, 2, w, v) + Q(qe, w, l) * (FC4(vq, 2, m, l, v) - FC4(vq, 2, m, k, v)) * fn
                                            + Q(qc, w, l) * (FC4(qn, 2, m, l, v) + FC4(qn, 2, m, k, v)) * fn
                                            - Q(qm, w, l) * (FC4(uq, 1, m, l, v) + FC4(uq, 1, m, k, v)) * fn;
                        } else {
                            SP3(q, 1, w, v) = SP3(q, 1, w, v) + Q(qe, w, l) * (FC4(vq, 1, m, l, v) + FC4(vq, 1, m, k, v)) * fn
                                            + Q(qc, w, l) * (FC4(qn, 1, m, l, v) - FC4(qn, 1, m, k, v)) * fn
                                            + Q(qm, w, l) * (FC4(uq, 2, m, l, v) - FC4(uq, 2, m, k, v)) * fn;
                            SP3(q, 2, w, v) = SP3(q, 2, w, v) + Q(qe, w, l) * (FC4(vq, 2, m, l, v) + FC4(vq, 2, m, k, v)) * fn
                                            + Q(qc, w, l) * (FC4(qn, 2, m, l, v) - FC4(qn, 2, m, k, v)) * fn
                                            - Q(qm, w, l) * (FC4(uq, 1, m, l, v) - FC4(uq, 1, m, k, v)) * fn;
                        }
                        w = w + 1;
                    }
            }
        }
    }
}

/* SUBROUTINE MKTEND, legmod.f90:505-606 */
void oracle_mktend(const oracle_leg *L, double *d, double *t, double *z,
                   const double *tn, const double *fu, const double *fv,
                   const double *ke, const double *ut, const double *vt,
                   int nlev, int folded) {
    int nlat = L->nlat, nlon = L->nlon, ncsp = L->ncsp, ntp1 = L->ntru + 1, nrsp = 2 * ncsp;
    const double *qe = L->qe, *qm = L->qm, *qc = L->qc, *qq = L->qq, *f = L->skgpsp;
    memset(d, 0, sizeof(double) * (size_t)nrsp * nlev);
    memset(t, 0, sizeof(double) * (size_t)nrsp * nlev);
    memset(z, 0, sizeof(double) * (size_t)nrsp * nlev);
    for (int v = 1; v <= nlev; v++) {
        if (!folded) {
            for (int l = 1; l <= nlat; l++) {
                int w = 1;
                for (int m = 1; m <= ntp1; m++)
                    for (int n = m; n <= ntp1; n++) {
                        double fn = f[n - 1];
                        SP3(d, 1, w, v) = SP3(d, 1, w, v) + Q(qq, w, l) * FC4(ke, 1, m, l, v) * fn
                                        - Q(qe, w, l) * FC4(fv, 1, m, l, v) * fn - Q(qm, w, l) * FC4(fu, 2, m, l, v) * fn;
                        SP3(d, 2, w, v) = SP3(d, 2, w, v) + Q(qq, w, l) * FC4(ke, 2, m, l, v) * fn
                                        - Q(qe, w, l) * FC4(fv, 2, m, l, v) * fn + Q(qm, w, l) * FC4(fu, 1, m, l, v) * fn;
                        SP3(t, 1, w, v) = SP3(t, 1, w, v) + Q(qe, w, l) * FC4(vt, 1, m, l, v) * fn
                                        + Q(qc, w, l) * FC4(tn, 1, m, l, v) * fn + Q(qm, w, l) * FC4(ut, 2, m, l, v) * fn;
                        SP3(t, 2, w, v) = SP3(t, 2, w, v) + Q(qe, w, l) * FC4(vt, 2, m, l, v) * fn
                                        + Q(qc, w, l) * FC4(tn, 2, m, l, v) * fn - Q(qm, w, l) * FC4(ut, 1, m, l, v) * fn;
                        SP3(z, 1, w, v) = SP3(z, 1, w, v) + Q(qe, w, l) * FC4(fu, 1, m, l, v) * fn
                                        - Q(qm, w, l) * FC4(fv, 2, m, l, v) * fn;
                        SP3(z, 2, w, v) = SP3(z, 2, w, v) + Q(qe, w, l) * FC4(fu, 2, m, l, v) * fn
                                        + Q(qm, w, l) * FC4(fv, 1, m, l, v) * fn;
                        w = w + 1;
                    }
            }
        } else {
            for (int l = 1; l <= nlat / 2; l++) {
                int k = nlat + 1 - l, w = 1;
                for (int m = 1; m <= ntp1; m++)
                    for (int n = m; n <= ntp1; n++) {
                        double fn = f[n - 1];
                        double s = ((m + n) % 2 == 0) ? 1.0 : -1.0;
                        /* symmetric (s=+1): P-type tables take (N+S), Q-type (N-S);
                         * antisymmetric swaps them -- legmod.f90:557-601 */
                        double keP = s > 0 ? FC4(ke, 1, m, l, v) + FC4(ke, 1, m, k, v) : FC4(ke, 1, m, l, v) - FC4(ke, 1, m, k, v);
                        double keP2 = s > 0 ? FC4(ke, 2, m, l, v) + FC4(ke, 2, m, k, v) : FC4(ke, 2, m, l, v) - FC4(ke, 2, m, k, v);
                        double fvQ1 = s > 0 ? FC4(fv, 1, m, l, v) - FC4(fv, 1, m, k, v) : FC4(fv, 1, m, l, v) + FC4(fv, 1, m, k, v);
                        double fvQ2 = s > 0 ? FC4(fv, 2, m, l, v) - FC4(fv, 2, m, k, v) : FC4(fv, 2, m, l, v) + FC4(fv, 2, m, k, v);
                        double fuP1 = s > 0 ? FC4(fu, 1, m, l, v) + FC4(fu, 1, m, k, v) : FC4(fu, 1, m, l, v) - FC4(fu, 1, m, k, v);
                        double fuP2 = s > 0 ? FC4(fu, 2, m, l, v) + FC4(fu, 2, m, k, v) : FC4(fu, 2, m, l, v) - FC4(fu, 2, m, k, v);
                        double vtQ1 = s > 0 ? FC4(vt, 1, m, l, v) - FC4(vt, 1, m, k, v) : FC4(vt, 1, m, l, v) + FC4(vt, 1, m, k, v);
                        double vtQ2 = s > 0 ? FC4(vt, 2, m, l, v) - FC4(vt, 2, m, k, v) : FC4(vt, 2, m, l, v) + FC4(vt, 2, m, k, v);
                        double tnP1 = s > 0 ? FC4(tn, 1, m, l, v) + FC4(tn, 1, m, k, v) : FC4(tn, 1, m, l, v) - FC4(tn, 1, m, k, v);
                        double tnP2 = s > 0 ? FC4(tn, 2, m, l, v) + FC4(tn, 2, m, k, v) : FC4(tn, 2, m, l, v) - FC4(tn, 2, m, k, v);
                        double utP1 = s > 0 ? FC4(ut, 1, m, l, v) + FC4(ut, 1, m, k, v) : FC4(ut, 1, m, l, v) - FC4(ut, 1, m, k, v);
                        double utP2 = s > 0 ? FC4(ut, 2, m, l, v) + FC4(ut, 2, m, k, v) : FC4(ut, 2, m, l, v) - FC4(ut, 2, m, k, v);
                        double fuQ1 = s > 0 ? FC4(fu, 1, m, l, v) - FC4(fu, 1, m, k, v) : FC4(fu, 1, m, l, v) + FC4(fu, 1, m, k, v);
                        double fuQ2 = s > 0 ? FC4(fu, 2, m, l, v) - FC4(fu, 2, m, k, v) : FC4(fu, 2, m, l, v) + FC4(fu, 2, m, k, v);
                        double fvP1 = s > 0 ? FC4(fv, 1, m, l, v) + FC4(fv, 1, m, k, v) : FC4(fv, 1, m, l, v) - FC4(fv, 1, m, k, v);
                        double fvP2 = s > 0 ? FC4(fv, 2, m, l, v) + FC4(fv, 2, m, k, v) : FC4(fv, 2, m, l, v) - FC4(fv, 2, m, k, v);
                        SP3(d, 1, w, v) = SP3(d, 1, w, v) + Q(qq, w, l) * keP * fn - Q(qe, w, l) * fvQ1 * fn - Q(qm, w, l) * fuP2 * fn;
                        SP3(d, 2, w, v) = SP3(d, 2, w, v) + Q(qq, w, l) * keP2 * fn - Q(qe, w, l) * fvQ2 * fn + Q(qm, w, l) * fuP1 * fn;
                        SP3(t, 1, w, v) = SP3(t, 1, w, v) + Q(qe, w, l) * vtQ1 * fn + Q(qc, w, l) * tnP1 * fn + Q(qm, w, l) * utP2 * fn;
                        SP3(t, 2, w, v) = SP3(t, 2, w, v) + Q(qe, w, l) * vtQ2 * fn + Q(qc, w, l) * tnP2 * fn - Q(qm, w, l) * utP1 * fn;
                        SP3(z, 1, w, v) = SP3(z, 1, w, v) + Q(qe, w, l) * fuQ1 * fn - Q(qm, w, l) * fvP2 * fn;
                        SP3(z, 2, w, v) = SP3(z, 2, w, v) + Q(qe, w, l) * fuQ2 * fn + Q(qm, w, l) * fvP1 * fn;
                        w = w + 1;
                    }
            }
        }
    }
}

/* ===================== fftmod.f90 ===================== */

static const int fft_allowed[13] = {8, 16, 32, 48, 64, 96, 128, 256, 384, 512, 1024, 2048, 4096};

/* SUBROUTINE FFTINI trig table, fftmod.f90:113-118 */
static void fftini(double *trigs, int n) {
    double del = 4.0 * asin(1.0) / n;
    for (int k = 0; k <= n / 2 - 1; k++) {
        double angle = k * del;
        trigs[2 * k] = cos(angle);
        trigs[2 * k + 1] = sin(angle);
    }
}

#define A2(i, l) a[(size_t)((l) - 1) * n + (i) - 1]
#define C2(i, l) c[(size_t)((l) - 1) * n + (i) - 1]
#define TR(i) trigs[(i) - 1]

/* SUBROUTINE DFFT2, fftmod.f90:128-155 (one row) */
static void dfft2(double *a, const double *trigs, int n, double *c) {
    c[0] = a[0] + a[1];
    c[1] = 0.0;
    int ja = 3, jb = n - 1;
#define A1(i) a[(i) - 1]
#define C1(i) c[(i) - 1]
    for (int i = 3; i <= n - 5; i += 4) {
        double c1 = TR(ja), s1 = TR(ja + 1);
        double a1p3 = c1 * A1(i + 1) + s1 * A1(i + 3);
        double a3m1 = c1 * A1(i + 3) - s1 * A1(i + 1);
        C1(ja) = A1(i) + a1p3;
        C1(jb) = A1(i) - a1p3;
        C1(ja + 1) = a3m1 + A1(i + 2);
        C1(jb + 1) = a3m1 - A1(i + 2);
        ja += 2;
        jb -= 2;
    }
    C1(ja) = A1(n - 1);
    C1(ja + 1) = -A1(n);
    memcpy(a, c, sizeof(double) * n);
}

/* SUBROUTINE DFFT3, fftmod.f90:161-206 (one row) */
static void dfft3(double *a, const double *trigs, int n, double *c) {
    const double SIN60 = 0.866025403784438;
    int ja = 1, jb = 2 * (n / 3) + 1, jc = jb;
    C1(ja) = A1(1) + A1(2) + A1(3);
    C1(ja + 1) = 0.0;
    C1(jb) = A1(1) - 0.5 * (A1(2) + A1(3));
    C1(jb + 1) = SIN60 * (A1(3) - A1(2));
    ja = 3; jb = jb + 2; jc = jc - 2;
    for (int i = 4; i <= n - 8; i += 6) {
        double c1 = TR(ja), s1 = TR(ja + 1), c2 = TR(ja + ja - 1), s2 = TR(ja + ja);
        double a1 = (c1 * A1(i + 1) + s1 * A1(i + 4)) + (c2 * A1(i + 2) + s2 * A1(i + 5));
        double b1 = (c1 * A1(i + 4) - s1 * A1(i + 1)) + (c2 * A1(i + 5) - s2 * A1(i + 2));
        double a2 = A1(i) - 0.5 * a1;
        double b2 = A1(i + 3) - 0.5 * b1;
        double a3 = SIN60 * ((c1 * A1(i + 1) + s1 * A1(i + 4)) - (c2 * A1(i + 2) + s2 * A1(i + 5)));
        double b3 = SIN60 * ((c1 * A1(i + 4) - s1 * A1(i + 1)) - (c2 * A1(i + 5) - s2 * A1(i + 2)));
        C1(ja) = A1(i) + a1;
        C1(ja + 1) = A1(i + 3) + b1;
        C1(jb) = a2 + b3;
        C1(jb + 1) = b2 - a3;
        C1(jc) = a2 - b3;
        C1(jc + 1) = -b2 - a3;
        ja += 2; jb += 2; jc -= 2;
    }
    if (ja <= jc) {
        C1(ja) = A1(n - 2) + 0.5 * (A1(n - 1) - A1(n));
        C1(ja + 1) = -SIN60 * (A1(n - 1) + A1(n));
    }
    memcpy(a, c, sizeof(double) * n);
#undef A1
#undef C1
}

/* SUBROUTINE DFFT4, fftmod.f90:212-327 */
static void dfft4(double *a, const double *trigs, int n, int lot, int *la_io, double *c) {
    int la = *la_io / 4;
    int i1 = la, i2 = la + i1, i3 = la + i2, i4 = la + i3, i5 = la + i4, i6 = la + i5, i7 = la + i6;
    int j1 = n / 2 - la, j2 = n - la, j3 = j1, j5 = j1 + la;
    for (int i = 1; i <= la; i++)
        for (int l = 1; l <= lot; l++) {
            double a0p2 = A2(i, l) + A2(i2 + i, l);
            double a1p3 = A2(i1 + i, l) + A2(i3 + i, l);
            C2(i, l) = a0p2 + a1p3;
            C2(j2 + i, l) = a0p2 - a1p3;
            C2(j1 + i, l) = A2(i, l) - A2(i2 + i, l);
            C2(j5 + i, l) = A2(i3 + i, l) - A2(i1 + i, l);
        }
    int jink = 2 * la, j0 = la;
    j1 = j1 + jink; j2 = j2 - jink; j3 = j3 - jink;
    int j4 = j0 + la; j5 = j1 + la; int j6 = j2 + la, j7 = j3 + la;
    int ibase = 4 * la;
    for (int k = la; k <= (n - 4) / 8; k += la) {
        int kb = k + k, kc = kb + kb, kd = kc + kb;
        double c1 = TR(kb + 1), s1 = TR(kb + 2), c2 = TR(kc + 1), s2 = TR(kc + 2), c3 = TR(kd + 1), s3 = TR(kd + 2);
        int i = ibase + 1;
        for (int j = 1; j <= la; j++) {
            for (int l = 1; l <= lot; l++) {
                double a1p5 = c1 * A2(i1 + i, l) + s1 * A2(i5 + i, l);
                double a2p6 = c2 * A2(i2 + i, l) + s2 * A2(i6 + i, l);
                double a3p7 = c3 * A2(i3 + i, l) + s3 * A2(i7 + i, l);
                double a5m1 = c1 * A2(i5 + i, l) - s1 * A2(i1 + i, l);
                double a6m2 = c2 * A2(i6 + i, l) - s2 * A2(i2 + i, l);
                double a7m3 = c3 * A2(i7 + i, l) - s3 * A2(i3 + i, l);
                double a0 = A2(i, l) + a2p6;
                double a2 = A2(i, l) - a2p6;
                double a1 = a1p5 + a3p7;
                double a3 = a3p7 - a1p5;
                double b0 = A2(i4 + i, l) + a6m2;
                double b2 = A2(i4 + i, l) - a6m2;
                double b1 = a5m1 + a7m3;
                double b3 = a5m1 - a7m3;
                C2(j0 + j, l) = a0 + a1;
                C2(j2 + j, l) = a0 - a1;
                C2(j4 + j, l) = b0 + b1;
                C2(j6 + j, l) = b1 - b0;
                C2(j1 + j, l) = a2 + b3;
                C2(j3 + j, l) = a2 - b3;
                C2(j5 + j, l) = a3 + b2;
                C2(j7 + j, l) = a3 - b2;
            }
            i = i + 1;
        }
        ibase = ibase + 8 * la;
        j0 += jink; j1 += jink; j2 -= jink; j3 -= jink;
        j4 = j0 + la; j5 = j1 + la; j6 = j2 + la; j7 = j3 + la;
    }
    if (j1 <= j2) {
        double sin45 = sqrt(0.5);
        int i = ibase + 1;
        for (int j = 1; j <= la; j++) {
            for (int l = 1; l <= lot; l++) {
                double a1p3 = sin45 * (A2(i1 + i, l) + A2(i3 + i, l));
                double a1m3 = sin45 * (A2(i1 + i, l) - A2(i3 + i, l));
                C2(j0 + j, l) = A2(i, l) + a1m3;
                C2(j1 + j, l) = A2(i, l) - a1m3;
                C2(j4 + j, l) = -A2(i2 + i, l) - a1p3;
                C2(j5 + j, l) = A2(i2 + i, l) - a1p3;
            }
            i = i + 1;
        }
    }
    if (la == 1) {
        for (int l = 1; l <= lot; l++) {
            A2(1, l) = C2(1, l);
            A2(2, l) = 0.0;
            for (int i = 3; i <= n; i++) A2(i, l) = C2(i - 1, l);
        }
    } else {
        memcpy(a, c, sizeof(double) * (size_t)n * lot);
    }
    *la_io = la;
}

/* SUBROUTINE DFFT8, fftmod.f90:333-373 (a and c may alias) */
static void dfft8(double *a, double *c, int n, int lot) {
    int la = n / 8;
    double z = 1.0 / n, zsin45 = z * sqrt(0.5);
    for (int i = 0; i <= la * lot - 1; i++) {
        int i0 = (i / la) * n + i % la + 1;
        int i1 = i0 + la, i2 = i1 + la, i3 = i2 + la, i4 = i3 + la, i5 = i4 + la, i6 = i5 + la, i7 = i6 + la;
#define AF(i) a[(i) - 1]
#define CF(i) c[(i) - 1]
        double a0p4 = AF(i0) + AF(i4);
        double a1p5 = AF(i1) + AF(i5);
        double a2p6 = AF(i2) + AF(i6);
        double a3p7 = AF(i3) + AF(i7);
        double a5m1 = AF(i5) - AF(i1);
        double a7m3 = AF(i7) - AF(i3);
        double a0m4 = (AF(i0) - AF(i4)) * z;
        double a6m2 = (AF(i6) - AF(i2)) * z;
        double a0p4p2p6 = a0p4 + a2p6;
        double a1p5p3p7 = a1p5 + a3p7;
        double a7m3p5m1 = (a7m3 + a5m1) * zsin45;
        double a7m3m5m1 = (a7m3 - a5m1) * zsin45;
        CF(i0) = z * (a0p4p2p6 + a1p5p3p7);
        CF(i7) = z * (a0p4p2p6 - a1p5p3p7);
        CF(i3) = z * (a0p4 - a2p6);
        CF(i4) = z * (a3p7 - a1p5);
        CF(i1) = a0m4 + a7m3m5m1;
        CF(i5) = a0m4 - a7m3m5m1;
        CF(i2) = a7m3p5m1 + a6m2;
        CF(i6) = a7m3p5m1 - a6m2;
    }
}

/* SUBROUTINE IFFT4, fftmod.f90:379-486 ("c" is the caller's data) */
static void ifft4(double *c, const double *trigs, int n, int lot, int *la_io, double *a) {
    int la = *la_io;
    if (la == 1) {
        for (int l = 1; l <= lot; l++) {
            A2(1, l) = 0.5 * C2(1, l);
            A2(n, l) = 0.0;
            for (int i = 2; i <= n - 1; i++) A2(i, l) = C2(i + 1, l);
        }
    } else {
        memcpy(a, c, sizeof(double) * (size_t)n * lot);
    }
    int kstop = (n - 4) / 8;
    int i1 = n / 2 - la, i2 = n - la, i5 = i1 + la;
    int j1 = la, j2 = la + j1, j3 = la + j2, j4 = la + j3, j5 = la + j4, j6 = la + j5, j7 = la + j6;
    for (int i = 1; i <= la; i++)
        for (int l = 1; l <= lot; l++) {
            C2(i, l) = A2(i, l) + A2(i2 + i, l) + A2(i1 + i, l);
            C2(j1 + i, l) = A2(i, l) - A2(i2 + i, l) - A2(i5 + i, l);
            C2(j2 + i, l) = A2(i, l) + A2(i2 + i, l) - A2(i1 + i, l);
            C2(j3 + i, l) = A2(i, l) - A2(i2 + i, l) + A2(i5 + i, l);
        }
    int iink = 2 * la, jbase = 4 * la + 1;
    int i0 = la;
    i1 = i0 + n / 2; i2 = n - 3 * la;
    int i3 = i2 - n / 2, i4 = i0 + la;
    i5 = i1 + la;
    int i6 = i2 + la, i7 = i3 + la;
    for (int k = la; k <= kstop; k += la) {
        int kb = k + k, kc = kb + kb, kd = kc + kb;
        double c1 = TR(kb + 1), s1 = TR(kb + 2), c2 = TR(kc + 1), s2 = TR(kc + 2), c3 = TR(kd + 1), s3 = TR(kd + 2);
        for (int i = 1; i <= la; i++) {
            int j = jbase;
            for (int l = 1; l <= lot; l++) {
                double a0p2 = A2(i0 + i, l) + A2(i2 + i, l);
                double a0m2 = A2(i0 + i, l) - A2(i2 + i, l);
                double a1p3 = A2(i1 + i, l) + A2(i3 + i, l);
                double a1m3 = A2(i1 + i, l) - A2(i3 + i, l);
                double a4p6 = A2(i4 + i, l) + A2(i6 + i, l);
                double a4m6 = A2(i4 + i, l) - A2(i6 + i, l);
                double a5p7 = A2(i5 + i, l) + A2(i7 + i, l);
                double a5m7 = A2(i5 + i, l) - A2(i7 + i, l);
                double a0p2m1p3 = a0p2 - a1p3;
                double a4m6m5m7 = a4m6 - a5m7;
                C2(j, l) = a0p2 + a1p3;
                C2(j4 + j, l) = a4m6 + a5m7;
                C2(j2 + j, l) = c2 * a0p2m1p3 - s2 * a4m6m5m7;
                C2(j6 + j, l) = s2 * a0p2m1p3 + c2 * a4m6m5m7;
                C2(j1 + j, l) = c1 * (a0m2 - a5p7) - s1 * (a4p6 + a1m3);
                C2(j5 + j, l) = s1 * (a0m2 - a5p7) + c1 * (a4p6 + a1m3);
                C2(j3 + j, l) = c3 * (a0m2 + a5p7) - s3 * (a4p6 - a1m3);
                C2(j7 + j, l) = s3 * (a0m2 + a5p7) + c3 * (a4p6 - a1m3);
            }
            jbase = jbase + 1;
        }
        i0 += iink; i1 += iink; i2 -= iink; i3 -= iink;
        i4 += iink; i5 += iink; i6 -= iink; i7 -= iink;
        jbase = jbase + 7 * la;
    }
    if (i1 <= i2) {
        double sin45 = sqrt(0.5);
        for (int i = 1; i <= la; i++) {
            int j = jbase;
            for (int l = 1; l <= lot; l++) {
                C2(j, l) = A2(i0 + i, l) + A2(i1 + i, l);
                C2(j1 + j, l) = sin45 * ((A2(i0 + i, l) - A2(i1 + i, l)) - (A2(la + i0 + i, l) + A2(la + i1 + i, l)));
                C2(j2 + j, l) = A2(la + i1 + i, l) - A2(la + i0 + i, l);
                C2(j3 + j, l) = -sin45 * ((A2(i0 + i, l) - A2(i1 + i, l)) + (A2(la + i0 + i, l) + A2(la + i1 + i, l)));
            }
            jbase = jbase + 1;
        }
    }
    *la_io = la * 4;
}

/* SUBROUTINE IFFT2, fftmod.f90:492-529 */
static void ifft2(double *a, const double *trigs, int n, int lot, int *la_io, double *c) {
    for (int l = 1; l <= lot; l++) {
        C2(1, l) = 0.5 * A2(1, l);
        C2(2, l) = C2(1, l);
    }
    int ia = 3, ib = n - 1;
    for (int j = 3; j <= n - 5; j += 4) {
        double c1 = TR(ia), s1 = TR(ia + 1);
        for (int l = 1; l <= lot; l++) {
            double amb = A2(ia, l) - A2(ib, l);
            double apb = A2(ia + 1, l) + A2(ib + 1, l);
            C2(j, l) = A2(ia, l) + A2(ib, l);
            C2(j + 2, l) = A2(ia + 1, l) - A2(ib + 1, l);
            C2(j + 1, l) = c1 * amb - s1 * apb;
            C2(j + 3, l) = s1 * amb + c1 * apb;
        }
        ia += 2; ib -= 2;
    }
    for (int l = 1; l <= lot; l++) {
        C2(n - 1, l) = A2(ia, l);
        C2(n, l) = -A2(ia + 1, l);
    }
    memcpy(a, c, sizeof(double) * (size_t)n * lot);
    *la_io = 2;
}

/* SUBROUTINE IFFT3, fftmod.f90:535-572 */
static void ifft3(double *a, const double *trigs, int n, int lot, int *la_io, double *c) {
    const double SIN60 = 0.866025403784438;
    int ib = 2 * (n / 3) + 1;
    for (int l = 1; l <= lot; l++) {
        C2(1, l) = 0.5 * A2(1, l) + A2(ib, l);
        C2(2, l) = 0.5 * A2(1, l) - 0.5 * A2(ib, l) - SIN60 * A2(ib + 1, l);
        C2(3, l) = 0.5 * A2(1, l) - 0.5 * A2(ib, l) + SIN60 * A2(ib + 1, l);
    }
    int ia = 3, ic = ib - 2;
    ib = ib + 2;
    for (int j = 4; j <= n - 8; j += 6) {
        double c1 = TR(ia), s1 = TR(ia + 1), c2 = TR(ia + ia - 1), s2 = TR(ia + ia);
        for (int l = 1; l <= lot; l++) {
            double hbpc = A2(ia, l) - 0.5 * (A2(ib, l) + A2(ic, l));
            double hbmc = A2(ia + 1, l) - 0.5 * (A2(ib + 1, l) - A2(ic + 1, l));
            double sbmc = SIN60 * (A2(ib, l) - A2(ic, l));
            double sbpc = SIN60 * (A2(ib + 1, l) + A2(ic + 1, l));
            C2(j, l) = A2(ia, l) + A2(ib, l) + A2(ic, l);
            C2(j + 3, l) = A2(ia + 1, l) + A2(ib + 1, l) - A2(ic + 1, l);
            C2(j + 1, l) = c1 * (hbpc - sbpc) - s1 * (hbmc + sbmc);
            C2(j + 4, l) = s1 * (hbpc - sbpc) + c1 * (hbmc + sbmc);
            C2(j + 2, l) = c2 * (hbpc + sbpc) - s2 * (hbmc - sbmc);
            C2(j + 5, l) = s2 * (hbpc + sbpc) + c2 * (hbmc - sbmc);
        }
        ia += 2; ib += 2; ic -= 2;
    }
    for (int l = 1; l <= lot; l++) {
        C2(n - 2, l) = A2(ia, l);
        C2(n - 1, l) = 0.5 * A2(ia, l) - SIN60 * A2(ia + 1, l);
        C2(n, l) = -0.5 * A2(ia, l) - SIN60 * A2(ia + 1, l);
    }
    memcpy(a, c, sizeof(double) * (size_t)n * lot);
    *la_io = 3;
}

/* SUBROUTINE IFFT8, fftmod.f90:578-618 (a and c may alias) */
static void ifft8(double *a, double *c, int n, int lot) {
    const double SQRT2 = 1.414213562373095;
    int la = n / 8;
    for (int i = 0; i <= la * lot - 1; i++) {
        int i0 = (i / la) * n + i % la + 1;
        int i1 = i0 + la, i2 = i1 + la, i3 = i2 + la, i4 = i3 + la, i5 = i4 + la, i6 = i5 + la, i7 = i6 + la;
        double a0p7 = AF(i0) + AF(i7);
        double a0m7 = AF(i0) - AF(i7);
        double a1p5 = AF(i1) + AF(i5);
        double a1m5 = AF(i1) - AF(i5);
        double a2p6 = AF(i2) + AF(i6);
        double a2m6 = AF(i2) - AF(i6);
        double a0p7p3 = a0p7 + AF(i3);
        double a0p7m3 = a0p7 - AF(i3);
        double a0m7p4 = 2.0 * (a0m7 + AF(i4));
        double a0m7m4 = 2.0 * (a0m7 - AF(i4));
        double a1m5p2p6 = SQRT2 * (a1m5 + a2p6);
        double a1m5m2p6 = SQRT2 * (a1m5 - a2p6);
        CF(i0) = 2.0 * (a0p7p3 + a1p5);
        CF(i2) = 2.0 * (a0p7m3 - a2m6);
        CF(i4) = 2.0 * (a0p7p3 - a1p5);
        CF(i6) = 2.0 * (a0p7m3 + a2m6);
        CF(i1) = a0m7m4 + a1m5m2p6;
        CF(i3) = a0m7p4 - a1m5p2p6;
        CF(i5) = a0m7m4 - a1m5m2p6;
        CF(i7) = a0m7p4 + a1m5p2p6;
    }
}
#undef AF
#undef CF

static int fft_ok(int n) {
    for (int j = 0; j < 13; j++) if (n == fft_allowed[j]) return 1;
    return 0;
}

/* SUBROUTINE GP2FC, fftmod.f90:29-58 */
int oracle_gp2fc(double *a, int n, int lot) {
    if (!fft_ok(n)) return -1;
    double *trigs = malloc(sizeof(double) * n);
    double *c = malloc(sizeof(double) * (size_t)n * lot);
    fftini(trigs, n);
    dfft8(a, a, n, lot);
    int la = n / 8;
    while (la >= 4) dfft4(a, trigs, n, lot, &la, c);
    if (la == 3) for (int l = 0; l < lot; l++) dfft3(a + (size_t)l * n, trigs, n, c);
    if (la == 2) for (int l = 0; l < lot; l++) dfft2(a + (size_t)l * n, trigs, n, c);
    free(trigs);
    free(c);
    return 0;
}

/* SUBROUTINE FC2GP, fftmod.f90:64-87 */
int oracle_fc2gp(double *a, int n, int lot) {
    if (!fft_ok(n)) return -1;
    double *trigs = malloc(sizeof(double) * n);
    double *c = malloc(sizeof(double) * (size_t)n * lot);
    fftini(trigs, n);
    int nf = n / 8;
    while (nf >= 4) nf = nf / 4;
    int la = 1;
    if (nf == 2) ifft2(a, trigs, n, lot, &la, c);
    if (nf == 3) ifft3(a, trigs, n, lot, &la, c);
    while (la < n / 8) ifft4(a, trigs, n, lot, &la, c);
    ifft8(a, a, n, lot);
    free(trigs);
    free(c);
    return 0;
}

/* ===================== fft991mod.f90 contract ===================== */
/* fft991mod.f90 supports n in {4,64,96,128,192,256,320,384} (:12).  Its
 * transform is defined at fft991mod.f90:147-155; gp2fc/fc2gp (:32-80) pad to
 * n+2 with zeros and copy back the first n values, so the Nyquist term is
 * dropped and the m=0 imaginary slot is zero (forward) / ignored (inverse).
 * The restatement evaluates that definition directly in extended precision
 * (the Temperton passes rpassm/qpassm compute the same sums). */
static const int fft991_allowed[8] = {4, 64, 96, 128, 192, 256, 320, 384};
static int fft991_ok(int n) {
    for (int j = 0; j < 8; j++) if (n == fft991_allowed[j]) return 1;
    return 0;
}

int oracle_gp2fc_991(double *a, int n, int lot) {
    if (!fft991_ok(n)) return -1;
    long double *x = malloc(sizeof(long double) * n);
    const long double TWOPI_L = 6.283185307179586476925286766559L;
    for (int l = 0; l < lot; l++) {
        double *row = a + (size_t)l * n;
        for (int j = 0; j < n; j++) x[j] = row[j];
        for (int k = 0; k < n / 2; k++) {
            long double sa = 0.0L, sb = 0.0L;
            for (int j = 0; j < n; j++) {
                long jk = ((long)j * k) % n;
                long double ang = TWOPI_L * (long double)jk / (long double)n;
                sa += x[j] * cosl(ang);
                sb += x[j] * sinl(ang);
            }
            row[2 * k] = (double)(sa / n);
            row[2 * k + 1] = (double)(-sb / n);
        }
        row[1] = 0.0;
    }
    free(x);
    return 0;
}

int oracle_fc2gp_991(double *a, int n, int lot) {
    if (!fft991_ok(n)) return -1;
    long double *cr = malloc(sizeof(long double) * n);
    const long double TWOPI_L = 6.283185307179586476925286766559L;
    for (int l = 0; l < lot; l++) {
        double *row = a + (size_t)l * n;
        for (int j = 0; j < n; j++) cr[j] = row[j];
        for (int j = 0; j < n; j++) {
            long double s = cr[0];
            for (int k = 1; k < n / 2; k++) {
                long jk = ((long)j * k) % n;
                long double ang = TWOPI_L * (long double)jk / (long double)n;
                s += 2.0L * (cr[2 * k] * cosl(ang) - cr[2 * k + 1] * sinl(ang));
            }
            row[j] = (double)s;
        }
    }
    free(cr);
    return 0;
}
