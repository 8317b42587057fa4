/*
 * Oracle (test infrastructure): FP64 restatement of the grid-point part of
 * PlaSim's gridpointa between the inverse and the forward transforms
 * (plasim.f90:2441-2455): gp = exp(gp), calcgp (:2587-2755) and the flux
 * products gut, gvt, gke (+ gphi), guq, gvq; and of the constants of the
 * semi-implicit scheme calcgp reads (initsi, :1709-1768; rdsig :1564).
 * Loop and operation order follow the Fortran.  Only tests use it.
 *
 * Arrays are the reference's (NHOR fastest, then level), columns h < nhor:
 *   gin  [6L+3][nhor]  gu[L], gv[L], gt[L], gd[L], gz[L], gq[L], gpj, gpmt, gp  (gp = ln ps)
 *   gout [9L+1][nhor]  gtn[L], gqn[L], gut[L], gvt[L], guz[L], gvz[L], gke[L], gvpp, guq[L], gvq[L]
 *   dw   [L][nhor]     vertical velocity diagnostic (may be NULL)
 *   rcsq [nhor / nlon] 1/cos^2 of each latitude row
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "exo_oracle.h"

/* initsi (plasim.f90:1709-1745) and rdsig (:1564): g, c (NLEV x NLEV, column
 * major: g[i + L*j] = g(i+1, j+1)), tkp, t01s2, rdsig from sigmah, dsigma, t0, akap */
void oracle_initsi(int nlev, const double *sigmah, const double *dsigma, const double *t0, double akap,
                   double *g, double *c, double *tkp, double *t01s2, double *rdsig) {
    int L = nlev;
    double *zalp = calloc(L, sizeof(double));
    for (int j = 0; j < L; j++) tkp[j] = akap * t0[j];
    for (int j = 0; j < L - 1; j++) t01s2[j] = t0[j + 1] - t0[j];
    t01s2[L - 1] = 0.0;
    for (int j = 1; j < L; j++) zalp[j] = log(sigmah[j]) - log(sigmah[j - 1]);
    for (int i = 0; i < L * L; i++) g[i] = 0.0;
    g[0] = 1.0;
    for (int jl = 1; jl < L; jl++) {
        g[jl + L * jl] = 1.0 - zalp[jl] * sigmah[jl - 1] / dsigma[jl];
        for (int k = 0; k < jl; k++) g[jl + L * k] = zalp[jl];
    }
    for (int jl = 0; jl < L; jl++)
        for (int k = 0; k < L; k++) c[jl + L * k] = g[k + L * jl] * (dsigma[jl] / dsigma[k]);
    for (int j = 0; j < L; j++) rdsig[j] = 0.5 / dsigma[j];
    free(zalp);
}

#define G(i, j) P->g[(i) + L * (j)]
#define CC(i, j) P->c[(i) + L * (j)]

void oracle_gridpoint(const oracle_gppar *P, const double *gin, double *gout, double *dw, const double *rcsq) {
    const int L = P->nlev, nhor = P->nhor, nlon = P->nlon;
    const size_t n = (size_t)nhor;
    const double *gu = gin, *gv = gin + L * n, *gt = gin + 2 * L * n, *gd = gin + 3 * L * n, *gz = gin + 4 * L * n,
                 *gq = gin + 5 * L * n, *gpj = gin + 6 * L * n, *gpm = gpj + n, *glnp = gpm + n;
    double *gtn = gout, *gqn = gout + L * n, *gut = gout + 2 * L * n, *gvt = gout + 3 * L * n,
           *guz = gout + 4 * L * n, *gvz = gout + 5 * L * n, *gke = gout + 6 * L * n, *gvp = gout + 7 * L * n,
           *guq = gvp + n, *gvq = gvp + n + L * n;
    double *zvgpg = malloc(sizeof(double) * L), *ztv1 = malloc(sizeof(double) * L),
           *ztv2 = malloc(sizeof(double) * L), *zsdotp = malloc(sizeof(double) * L),
           *gtd = malloc(sizeof(double) * L), *gqm = malloc(sizeof(double) * L),
           *gud = malloc(sizeof(double) * L), *gvd = malloc(sizeof(double) * L);
    for (int h = 0; h < nhor; h++) {
#define A(x, k) (x)[(size_t)(k) * n + h]
        const double rc = rcsq[h / nlon];
        const double gp = exp(glnp[h]);                      /* gp = exp(gp), plasim.f90:2441 */
        for (int k = 0; k < L; k++) {
            zvgpg[k] = rc * (A(gu, k) * gpm[h] + A(gv, k) * gpj[h]);
            double zq = P->nqspec == 1 ? fmax(A(gq, k) / gp, 0.0) : fmax(P->dq ? A(P->dq, k) : 0.0, 0.0);
            ztv1[k] = (A(gt, k) + P->t0[k]) * (1. + (1. / P->rdbrv - 1.) * zq) - P->t0[k];
            ztv2[k] = (A(gt, k) + P->t0[k]) * (1. + (1. / P->rdbrv - 1.) * zq) / (1. + P->adv * zq) - P->t0[k];
        }
        double zsumd = P->dsigma[0] * A(gd, 0);
        double gvpv = P->dsigma[0] * zvgpg[0];
        zsdotp[0] = zsumd + gvpv;
        for (int k = 1; k < L - 1; k++) {
            zsumd = zsumd + P->dsigma[k] * A(gd, k);
            gvpv = gvpv + P->dsigma[k] * zvgpg[k];
            zsdotp[k] = zsumd + gvpv;
        }
        zsumd = zsumd + P->dsigma[L - 1] * A(gd, L - 1);
        gvpv = gvpv + P->dsigma[L - 1] * zvgpg[L - 1];
        for (int k = 0; k < L - 1; k++) {
            zsdotp[k] = (P->sigmah[k] * (zsumd + gvpv) - zsdotp[k]);
            gtd[k] = zsdotp[k] * (A(gt, k + 1) - A(gt, k));
            gqm[k] = zsdotp[k] * (A(gq, k + 1) + A(gq, k));
            gud[k] = zsdotp[k] * (A(gu, k + 1) - A(gu, k));
            gvd[k] = zsdotp[k] * (A(gv, k + 1) - A(gv, k));
        }
        /* top level */
        zsumd = zvgpg[0] * P->dsigma[0];
        A(gtn, 0) = A(gt, 0) * A(gd, 0) - P->akap * ztv2[0] * A(gd, 0) -
                    P->rdsig[0] * (gtd[0] + P->t01s2[0] * (P->sigmah[0] * gvpv - zsumd));
        A(gqn, 0) = -P->rdsig[0] * gqm[0];
        A(guz, 0) = -A(gu, 0) * A(gz, 0) - gpj[h] * ztv1[0] - P->rdsig[0] * gvd[0];
        A(gvz, 0) = A(gv, 0) * A(gz, 0) - gpm[h] * ztv1[0] - P->rdsig[0] * gud[0];
        if (dw) A(dw, 0) = A(gd, 0) * gp * P->psurf * P->ww;
        /* inner levels */
        for (int k = 1; k < L - 1; k++) {
            double ztpta = CC(0, k) * zvgpg[0];
            double ztptb = CC(0, k) * (zvgpg[0] + A(gd, 0));
            for (int j = 1; j <= k; j++) {
                ztpta = ztpta + CC(j, k) * zvgpg[j];
                ztptb = ztptb + CC(j, k) * (zvgpg[j] + A(gd, j));
            }
            zsumd = zsumd + zvgpg[k] * P->dsigma[k];
            A(gtn, k) = A(gt, k) * A(gd, k) + P->akap * ztv2[k] * (zvgpg[k] - ztptb) +
                        P->tkp[k] * (zvgpg[k] - ztpta) -
                        P->rdsig[k] * (gtd[k] + gtd[k - 1] +
                                       gvpv * (P->t01s2[k] * P->sigmah[k] + P->t01s2[k - 1] * P->sigmah[k - 1]) -
                                       zsumd * (P->t01s2[k - 1] + P->t01s2[k]) +
                                       zvgpg[k] * P->dsigma[k] * P->t01s2[k - 1]);
            A(gqn, k) = -P->rdsig[k] * (gqm[k] - gqm[k - 1]);
            A(guz, k) = -A(gu, k) * A(gz, k) - gpj[h] * ztv1[k] - P->rdsig[k] * (gvd[k] + gvd[k - 1]);
            A(gvz, k) = A(gv, k) * A(gz, k) - gpm[h] * ztv1[k] - P->rdsig[k] * (gud[k] + gud[k - 1]);
            if (dw) A(dw, k) = (zvgpg[k] - ztptb) * gp * P->psurf * P->ww;
        }
        /* bottom level */
        {
            const int k = L - 1;
            double ztpta = CC(0, k) * zvgpg[0];
            double ztptb = CC(0, k) * (zvgpg[0] + A(gd, 0));
            for (int j = 1; j <= k; j++) {
                ztpta = ztpta + CC(j, k) * zvgpg[j];
                ztptb = ztptb + CC(j, k) * (zvgpg[j] + A(gd, j));
            }
            A(gtn, k) = A(gt, k) * A(gd, k) + P->akap * ztv2[k] * (zvgpg[k] - ztptb) +
                        P->tkp[k] * (zvgpg[k] - ztpta) -
                        P->rdsig[k] * (gtd[k - 1] + P->t01s2[k - 1] * (P->sigmah[k - 1] * gvpv - zsumd));
            A(gqn, k) = P->rdsig[k] * gqm[k - 1];
            A(guz, k) = -A(gu, k) * A(gz, k) - gpj[h] * ztv1[k] - P->rdsig[k] * gvd[k - 1];
            A(gvz, k) = A(gv, k) * A(gz, k) - gpm[h] * ztv1[k] - P->rdsig[k] * gud[k - 1];
            if (dw) A(dw, k) = (zvgpg[k] - ztptb) * gp * P->psurf * P->ww;
        }
        gvp[h] = gvpv;
        /* non-linear geopotential and the flux products (plasim.f90:2445-2455) */
        for (int k = 0; k < L; k++) {
            double dot = 0.0;
            for (int i = 0; i < L; i++) dot += G(i, k) * (ztv1[i] - A(gt, i));
            double gphi = dot * 2. / rc;
            A(gut, k) = A(gu, k) * A(gt, k);
            A(gvt, k) = A(gv, k) * A(gt, k);
            A(gke, k) = A(gu, k) * A(gu, k) + A(gv, k) * A(gv, k);
            A(gke, k) = A(gke, k) + gphi;
            A(guq, k) = A(gu, k) * A(gq, k);
            A(gvq, k) = A(gv, k) * A(gq, k);
        }
#undef A
    }
    free(zvgpg); free(ztv1); free(ztv2); free(zsdotp); free(gtd); free(gqm); free(gud); free(gvd);
}
