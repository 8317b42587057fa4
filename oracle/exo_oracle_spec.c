/*
 * Oracle (test infrastructure): FP64 restatement of PlaSim's semi-implicit
 * spectral time step -- the adiabatic part spectrala (plasim.f90:2757-2918,
 * single process, nadv > 0, without the diagnostic branches) and the
 * diabatic part spectrald (:3645-3999, nkits = 0, ndheat = 0, ndivdamp = 0,
 * without diagnostics) -- with the matrices they use: tau of initsi
 * (:1709-1760), bm1 of makebm (:1683-1704, inverted with the reference's own
 * ludcmp/lubksb, :1785-1838) and the diffusion coefficients sak (:1617-1633).
 * Loop and operation order follow the Fortran.  Only tests use it.
 *
 * Spectral arrays are [level][NRSP] (Fortran (NESP, NLEV)); matrices are
 * column major with leading dimension nlev: m[i + L*j] = m(i+1, j+1).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "exo_oracle.h"

/* tau of initsi (plasim.f90:1729-1752) from t0, sigmah, dsigma, rdsig, tkp, t01s2, c */
void oracle_tau(int L, const double *sigmah, const double *dsigma, const double *rdsig, const double *tkp,
                const double *t01s2, const double *c, double *tau) {
#define TAU(i, j) tau[(i) + L * (j)]
#define CM(i, j) c[(i) + L * (j)]
    double zt01s2 = t01s2[0], zsig = sigmah[0];
    TAU(0, 0) = 0.5 * zt01s2 * (zsig - 1.0) + tkp[0];
    for (int j = 1; j < L; j++) TAU(j, 0) = 0.5 * zt01s2 * dsigma[j];
    for (int jl = 1; jl < L; jl++) {          /* Fortran jlev = jl + 1 */
        double zttm = zt01s2, zsigm = zsig;
        zt01s2 = t01s2[jl];
        zsig = sigmah[jl];
        for (int j2 = 0; j2 < L; j2++) {
            double ztm = 0., ztmm = 0.;
            if (j2 <= jl) ztm = 1;
            if (j2 < jl) ztmm = 1;
            double ztau = zttm * (zsigm - ztmm);
            if (jl < L - 1) ztau = ztau + zt01s2 * (zsig - ztm);
            ztau = ztau * rdsig[jl] * dsigma[j2];
            if (j2 <= jl) ztau = ztau + tkp[jl] * CM(j2, jl);
            TAU(j2, jl) = ztau;
        }
    }
#undef TAU
#undef CM
}

/* ludcmp (plasim.f90:1785-1819), a column major n x n */
static void ludcmp(double *a, int n, int *indx) {
#define A_(i, j) a[(i) + n * (j)]
    double *vv = malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) {
        double mx = 0.0;
        for (int j = 0; j < n; j++) mx = fmax(mx, fabs(A_(i, j)));
        vv[i] = 1.0 / mx;
    }
    for (int j = 0; j < n; j++) {
        for (int i = 1; i < j; i++) {
            double dot = 0.0;
            for (int k = 0; k < i; k++) dot += A_(i, k) * A_(k, j);
            A_(i, j) = A_(i, j) - dot;
        }
        double aamax = 0.0;
        int imax = j;
        for (int i = j; i < n; i++) {
            if (j > 0) {
                double dot = 0.0;
                for (int k = 0; k < j; k++) dot += A_(i, k) * A_(k, j);
                A_(i, j) = A_(i, j) - dot;
            }
            double dum = vv[i] * fabs(A_(i, j));
            if (dum >= aamax) { imax = i; aamax = dum; }
        }
        if (j != imax) {
            for (int k = 0; k < n; k++) {
                double dum = A_(imax, k);
                A_(imax, k) = A_(j, k);
                A_(j, k) = dum;
            }
            vv[imax] = vv[j];
        }
        indx[j] = imax;
        if (A_(j, j) == 0.0) A_(j, j) = 2.2250738585072014e-308;
        if (j < n - 1)
            for (int i = j + 1; i < n; i++) A_(i, j) = A_(i, j) / A_(j, j);
    }
    free(vv);
}

/* lubksb (plasim.f90:1823-1845) */
static void lubksb(const double *a, int n, const int *indx, double *b) {
    int k = -1;
    for (int i = 0; i < n; i++) {
        int l = indx[i];
        double sum = b[l];
        b[l] = b[i];
        if (k >= 0) {
            for (int j = k; j < i; j++) sum = sum - A_(i, j) * b[j];
        } else if (sum != 0.0) {
            k = i;
        }
        b[i] = sum;
    }
    for (int i = n - 1; i >= 0; i--) {
        double sum = b[i];
        for (int j = i + 1; j < n; j++) sum = sum - A_(i, j) * b[j];
        b[i] = sum / A_(i, i);
    }
#undef A_
}

/* makebm (plasim.f90:1683-1704): bm1[jn] (jn = 1..ntru), each L x L column major,
 * bm1 sized (ntru+1) L^2 with jn = 0 left zero */
void oracle_makebm(int L, int ntru, double delt, const double *t0, const double *dsigma, const double *g,
                   const double *tau, double *bm1) {
    double zdeltsq = delt * delt;
    double *base = malloc(sizeof(double) * L * L), *b = malloc(sizeof(double) * L * L);
    double *col = malloc(sizeof(double) * L);
    int *indx = malloc(sizeof(int) * L);
    for (int j1 = 0; j1 < L; j1++)
        for (int j2 = 0; j2 < L; j2++) {
            double dot = 0.0;
            for (int i = 0; i < L; i++) dot += g[i + L * j1] * tau[j2 + L * i];
            base[j2 + L * j1] = zdeltsq * (t0[j1] * dsigma[j2] + dot);
        }
    memset(bm1, 0, sizeof(double) * L * L);
    for (int jn = 1; jn <= ntru; jn++) {
        memcpy(b, base, sizeof(double) * L * L);
        for (int j = 0; j < L; j++) b[j + L * j] = b[j + L * j] + 1.0 / (jn * (jn + 1));
        ludcmp(b, L, indx);
        double *out = bm1 + (size_t)jn * L * L;
        for (int j = 0; j < L; j++) {
            for (int i = 0; i < L; i++) col[i] = i == j ? 1.0 : 0.0;
            lubksb(b, L, indx, col);
            for (int i = 0; i < L; i++) out[i + L * j] = col[i];
        }
    }
    free(base); free(b); free(col); free(indx);
}

/* sak (plasim.f90:1617-1633), [L][NRSP] */
void oracle_sak(int L, int ntru, const int *ndel, int nhdiff, double *sak) {
    int nrsp = (ntru + 1) * (ntru + 2);
    for (int jl = 0; jl < L; jl++) {
        int jdel = ndel[jl];
        double zakk = 1. / pow((double)(ntru - nhdiff), jdel);
        int jr = 0;
        for (int jm = 0; jm <= ntru; jm++)
            for (int jn = jm; jn <= ntru; jn++) {
                double zsq = (double)(jn - nhdiff);
                double v = jn >= nhdiff ? zakk * pow(zsq, jdel) : 0.;
                sak[(size_t)jl * nrsp + jr] = v;
                sak[(size_t)jl * nrsp + jr + 1] = v;
                jr += 2;
            }
    }
}

static int nindex(int jsp, int ntru) {   /* total wavenumber n of spectral real jsp */
    int w = jsp / 2, m = 0, left = ntru + 1;
    while (w >= left) { w -= left; m++; left--; }
    return m + w;
}

/* spectrala, plasim.f90:2757-2918 (nadv > 0, nkits = 0, single process) */
void oracle_spectrala(const oracle_specpar *P, oracle_specstate *S) {
    const int L = P->nlev, ntru = P->ntru, nrsp = (ntru + 1) * (ntru + 2);
    const size_t n = (size_t)nrsp;
    double *apm = malloc(sizeof(double) * n), *adm = malloc(sizeof(double) * n * L),
           *azm = malloc(sizeof(double) * n * L), *atm = malloc(sizeof(double) * n * L),
           *adt = malloc(sizeof(double) * n * L), *aqm = malloc(sizeof(double) * n * L),
           *zgt = malloc(sizeof(double) * n * L), *zgm = malloc(sizeof(double) * n * L);
    memcpy(apm, S->spm, sizeof(double) * n);
    memcpy(adm, S->sdm, sizeof(double) * n * L);
    memcpy(azm, S->szm, sizeof(double) * n * L);
    memcpy(atm, S->stm, sizeof(double) * n * L);
    memcpy(adt, S->sdt, sizeof(double) * n * L);
    if (P->nqspec == 1) memcpy(aqm, S->sqm, sizeof(double) * n * L);
#define X(a, j, l) (a)[(size_t)(l) * n + (j)]
    /* 1.a */
    for (int jl = 0; jl < L; jl++)
        for (int j = 0; j < nrsp; j++) {
            double d1 = 0.0, d2 = 0.0;
            for (int i = 0; i < L; i++) {
                d1 += P->g[i + L * jl] * X(S->stt, j, i);
                d2 += P->g[i + L * jl] * X(atm, j, i);
            }
            X(zgt, j, jl) = d1;
            X(zgm, j, jl) = d2;
        }
    /* 1.b */
    for (int jl = 0; jl < L; jl++)
        for (int j = 0; j < nrsp; j++) {
            int jn = nindex(j, ntru);
            double zsum = 0.0;
            if (jn > 0) {
                double zq = 1.0 / (jn * (jn + 1));
                const double *bm = P->bm1 + (size_t)jn * L * L;
                for (int j2 = 0; j2 < L; j2++) {
                    double z0 = P->t0[j2];
                    double zt = X(zgt, j, j2) - z0 * S->spt[j];
                    double zm = X(zgm, j, j2) + z0 * S->spm[j];
                    double za = X(adt, j, j2) * zq + S->sop[j];
                    double zb = X(adm, j, j2) * zq;
                    double zz = zb + P->delt * (zm + za + P->delt * zt);
                    zsum = zsum + zz * bm[j2 + L * jl];
                }
            }
            X(S->sdt, j, jl) = zsum;
        }
    for (int jl = 0; jl < L; jl++) { X(S->sdt, 0, jl) = 0.0; X(S->sdt, 1, jl) = 0.0; }
    /* 2. */
    for (int jl = 0; jl < L; jl++)
        for (int j = 0; j < nrsp; j++) S->spt[j] = S->spt[j] + P->dsigma[jl] * X(S->sdt, j, jl);
    /* 3. */
    for (int jl = 0; jl < L; jl++)
        for (int j = 0; j < nrsp; j++) {
            double dot = 0.0;
            for (int i = 0; i < L; i++) dot += P->tau[i + L * jl] * X(S->sdt, j, i);
            X(S->stt, j, jl) = X(S->stt, j, jl) - dot;
        }
    /* 4.a */
    for (int j = 0; j < nrsp; j++) S->spm[j] = P->pnu21 * S->spp[j] + P->pnu * apm[j];
    for (size_t i = 0; i < n * L; i++) {
        S->sdm[i] = P->pnu21 * S->sdp[i] + P->pnu * adm[i];
        S->szm[i] = P->pnu21 * S->szp[i] + P->pnu * azm[i];
        S->stm[i] = P->pnu21 * S->stp[i] + P->pnu * atm[i];
        if (P->nqspec == 1) S->sqm[i] = P->pnu21 * S->sqp[i] + P->pnu * aqm[i];
    }
    /* 4.b */
    for (int j = 0; j < nrsp; j++) S->spp[j] = apm[j] - P->delt2 * S->spt[j];
    for (size_t i = 0; i < n * L; i++) {
        S->sdp[i] = 2.0 * S->sdt[i] - adm[i];
        S->stp[i] = P->delt2 * S->stt[i] + atm[i];
        S->szp[i] = P->delt2 * S->szt[i] + azm[i];
        if (P->nqspec == 1) S->sqp[i] = P->delt2 * S->sqt[i] + aqm[i];
    }
    S->spp[0] = 0.0;
    S->spp[1] = 0.0;
    free(apm); free(adm); free(azm); free(atm); free(adt); free(aqm); free(zgt); free(zgm);
}

/* spectrald, plasim.f90:3645-3999 (nkits = 0, ndheat = 0, ndivdamp = 0) */
void oracle_spectrald(const oracle_specpar *P, oracle_specstate *S) {
    const int L = P->nlev, ntru = P->ntru, nrsp = (ntru + 1) * (ntru + 2);
    const size_t n = (size_t)nrsp;
    const double d2 = P->delt2;
    for (size_t i = 0; i < n * L; i++) {
        S->szp[i] = S->szp[i] + d2 * S->szt[i];
        S->stp[i] = S->stp[i] + d2 * S->stt[i];
        S->sdp[i] = S->sdp[i] + d2 * S->sdt[i];
        if (P->nqspec == 1) S->sqp[i] = S->sqp[i] + d2 * S->sqt[i];
    }
    double *zszt1 = malloc(sizeof(double) * n * L), *zszt2 = malloc(sizeof(double) * n * L);
    for (int jl = 0; jl < L; jl++) {
        const double dm = P->damp[jl], tt = P->tdisst[jl], tq = P->tdissq[jl], td = P->tdissd[jl],
                     tz = P->tdissz[jl], tf = P->tfrc[jl];
        for (int j = 0; j < nrsp; j++) {
            double sk = X(P->sak, j, jl);
            X(S->stt, j, jl) = ((-dm - tt * sk) * X(S->stp, j, jl) + dm * X(S->srp, j, jl)) /
                               (1. + d2 * (dm + tt * sk));
            if (P->nqspec == 1) X(S->sqt, j, jl) = -tq * sk * X(S->sqp, j, jl) / (1. + d2 * tq * sk);
            double s1 = -tf * X(S->sdp, j, jl) / (1. + d2 * tf);
            double s2 = -td * sk * X(S->sdp, j, jl) / (1. + d2 * td * sk);
            X(S->sdt, j, jl) = s1 + s2;
            X(zszt1, j, jl) = -tf * X(S->szp, j, jl) / (1. + d2 * tf);
            X(zszt2, j, jl) = -tz * sk * X(S->szp, j, jl) / (1. + d2 * tz * sk);
            X(S->szt, j, jl) = X(zszt1, j, jl) + X(zszt2, j, jl);
        }
    }
    S->spp[0] = 0.0;
    S->spp[1] = 0.0;
    for (int jl = 0; jl < L; jl++) {
        const double tf = P->tfrc[jl], tz = P->tdissz[jl], sk = X(P->sak, 2, jl);
        X(S->szt, 2, jl) = X(S->szt, 2, jl) + P->plavor * (tf / (1. + d2 * tf) + tz * sk / (1. + d2 * tz * sk));
    }
    if (P->nsponge > 0)
        for (int j = 0; j < nrsp; j++)
            X(S->stt, j, 0) = P->dampsp * (X(S->stp, j, 1) - X(S->stp, j, 0)) + X(S->stt, j, 0);
    for (size_t i = 0; i < n * L; i++) {
        S->szp[i] = S->szp[i] + d2 * S->szt[i];
        S->stp[i] = S->stp[i] + d2 * S->stt[i];
        S->sdp[i] = S->sdp[i] + d2 * S->sdt[i];
        if (P->nqspec == 1) S->sqp[i] = S->sqp[i] + d2 * S->sqt[i];
    }
    for (size_t i = 0; i < n * L; i++) {
        S->szm[i] = S->szm[i] + P->pnu * S->szp[i];
        S->stm[i] = S->stm[i] + P->pnu * S->stp[i];
        S->sdm[i] = S->sdm[i] + P->pnu * S->sdp[i];
        if (P->nqspec == 1) S->sqm[i] = S->sqm[i] + P->pnu * S->sqp[i];
    }
    for (int j = 0; j < nrsp; j++) S->spm[j] = S->spm[j] + P->pnu * S->spp[j];
#undef X
    free(zszt1); free(zszt2);
}
