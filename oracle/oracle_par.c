/*
 * Oracle (test infrastructure): OpenMP drivers over the FP64 restatement,
 * used only as the timed CPU baseline.  They run the reference's own
 * per-timestep transform set (plasim.f90 gridpointa, :2396-2486) and the
 * radiation column pass over all host cores: levels and Fourier rows in
 * parallel for the transforms, column blocks for radmod -- the same work
 * split the reference gets from MPI ranks, without message passing.
 *
 * Field order (nlev = L):
 *   spin   [4L+1][2*NCSP]  sd[L], st[L], sz[L], sq[L], sp
 *   gpout  [6L+3][NLAT*NLON] gu[L], gv[L], gt[L], gd[L], gz[L], gq[L], gpj, gpmt, gp
 *   gpin   [9L+1][NLAT*NLON] gtn[L], gqn[L], gut[L], gvt[L], guz[L], gvz[L], gke[L], gvpp, guq[L], gvq[L]
 *   spout  [4L+1][2*NCSP]  sdf[L], stf[L], szf[L], sqf[L], spf
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>
#include "exo_oracle.h"

int oracle_num_threads(void) { return omp_get_max_threads(); }

/* inverse half of gridpointa: invlega (legmod.f90:635-654), Fourier-space
 * d/dlambda of ln ps (plasim.f90:2425-2430) and the fc2gp calls (:2432-2440) */
void oracle_inverse_set(const oracle_leg *L, int nlev, const double *spin, double *gpout,
                        double plavor, int use991) {
    int nlat = L->nlat, nlon = L->nlon, nrsp = 2 * L->ncsp;
    size_t nhor = (size_t)nlat * nlon;
    const double *sd = spin, *st = spin + (size_t)nlev * nrsp, *sz = spin + (size_t)2 * nlev * nrsp,
                 *sq = spin + (size_t)3 * nlev * nrsp, *sp = spin + (size_t)4 * nlev * nrsp;
    double *gu = gpout, *gv = gpout + nlev * nhor, *gt = gpout + 2 * nlev * nhor,
           *gd = gpout + 3 * nlev * nhor, *gz = gpout + 4 * nlev * nhor, *gq = gpout + 5 * nlev * nhor,
           *gpj = gpout + 6 * nlev * nhor, *gpmt = gpj + nhor, *gp = gpmt + nhor;
#pragma omp parallel for schedule(dynamic)
    for (int v = 0; v < nlev; v++) {
        double *pz = malloc(sizeof(double) * nrsp);
        memcpy(pz, sz + (size_t)v * nrsp, sizeof(double) * nrsp);
        oracle_dv2uv(L, sd + (size_t)v * nrsp, pz, gu + v * nhor, gv + v * nhor, 1, plavor);
        free(pz);
        oracle_sp2fc(L, sd + (size_t)v * nrsp, gd + v * nhor);
        oracle_sp2fc(L, st + (size_t)v * nrsp, gt + v * nhor);
        oracle_sp2fc(L, sz + (size_t)v * nrsp, gz + v * nhor);
        oracle_sp2fc(L, sq + (size_t)v * nrsp, gq + v * nhor);
    }
    oracle_sp2fc(L, sp, gp);
    oracle_sp2fcdmu(L, sp, gpj);
    for (int jlat = 0; jlat < nlat; jlat++)
        for (int jlon = 1; jlon <= nlon; jlon += 2) {
            size_t o = (size_t)jlat * nlon;
            gpmt[o + jlon - 1] = -gp[o + jlon] * ((jlon - 1) / 2);
            gpmt[o + jlon] = gp[o + jlon - 1] * ((jlon - 1) / 2);
        }
    int nrows = (int)((6 * nlev + 3) * (size_t)nlat);
    int chunk = nlat;
#pragma omp parallel for schedule(dynamic)
    for (int r = 0; r < nrows; r += chunk) {
        if (use991) oracle_fc2gp_991(gpout + (size_t)r * nlon, nlon, chunk);
        else oracle_fc2gp(gpout + (size_t)r * nlon, nlon, chunk);
    }
}

/* forward half of gridpointa: gp2fc calls (plasim.f90:2461-2473), then
 * fc2sp(gvpp), mktend and qtend (:2477-2486); gpin is transformed in place */
void oracle_forward_set(const oracle_leg *L, int nlev, double *gpin, double *spout, int use991) {
    int nlat = L->nlat, nlon = L->nlon, nrsp = 2 * L->ncsp;
    size_t nhor = (size_t)nlat * nlon;
    int nrows = (int)((9 * nlev + 1) * (size_t)nlat);
    int chunk = nlat;
#pragma omp parallel for schedule(dynamic)
    for (int r = 0; r < nrows; r += chunk) {
        if (use991) oracle_gp2fc_991(gpin + (size_t)r * nlon, nlon, chunk);
        else oracle_gp2fc(gpin + (size_t)r * nlon, nlon, chunk);
    }
    double *gtn = gpin, *gqn = gpin + nlev * nhor, *gut = gpin + 2 * nlev * nhor,
           *gvt = gpin + 3 * nlev * nhor, *guz = gpin + 4 * nlev * nhor, *gvz = gpin + 5 * nlev * nhor,
           *gke = gpin + 6 * nlev * nhor, *gvpp = gpin + 7 * nlev * nhor,
           *guq = gvpp + nhor, *gvq = gvpp + nhor + nlev * nhor;
    double *sdf = spout, *stf = spout + (size_t)nlev * nrsp, *szf = spout + (size_t)2 * nlev * nrsp,
           *sqf = spout + (size_t)3 * nlev * nrsp, *spf = spout + (size_t)4 * nlev * nrsp;
    oracle_fc2sp(L, gvpp, spf, 1);
#pragma omp parallel for schedule(dynamic)
    for (int v = 0; v < nlev; v++) {
        oracle_mktend(L, sdf + (size_t)v * nrsp, stf + (size_t)v * nrsp, szf + (size_t)v * nrsp,
                      gtn + v * nhor, gvz + v * nhor, guz + v * nhor, gke + v * nhor,
                      gut + v * nhor, gvt + v * nhor, 1, 1);
        oracle_qtend(L, sqf + (size_t)v * nrsp, gqn + v * nhor, guq + v * nhor, gvq + v * nhor, 1, 1);
    }
}

/* inverse half of gridpointd: invlegd (legmod.f90:661-677) and the fc2gp
 * calls (plasim.f90:3142-3149).  spin as above;
 * gpout [4L+1][NLAT*NLON] gu[L], gv[L], gt[L], gq[L], gp */
void oracle_inverse_set_d(const oracle_leg *L, int nlev, const double *spin, double *gpout,
                          double plavor, int use991) {
    int nlat = L->nlat, nlon = L->nlon, nrsp = 2 * L->ncsp;
    size_t nhor = (size_t)nlat * nlon;
    const double *sd = spin, *st = spin + (size_t)nlev * nrsp, *sz = spin + (size_t)2 * nlev * nrsp,
                 *sq = spin + (size_t)3 * nlev * nrsp, *sp = spin + (size_t)4 * nlev * nrsp;
    double *gu = gpout, *gv = gpout + nlev * nhor, *gt = gpout + 2 * nlev * nhor, *gq = gpout + 3 * nlev * nhor,
           *gp = gpout + 4 * nlev * nhor;
#pragma omp parallel for schedule(dynamic)
    for (int v = 0; v < nlev; v++) {
        double *pz = malloc(sizeof(double) * nrsp);
        memcpy(pz, sz + (size_t)v * nrsp, sizeof(double) * nrsp);
        oracle_dv2uv(L, sd + (size_t)v * nrsp, pz, gu + v * nhor, gv + v * nhor, 1, plavor);
        free(pz);
        oracle_sp2fc(L, sq + (size_t)v * nrsp, gq + v * nhor);
        oracle_sp2fc(L, st + (size_t)v * nrsp, gt + v * nhor);
    }
    oracle_sp2fc(L, sp, gp);
    int nrows = (int)((4 * nlev + 1) * (size_t)nlat);
    int chunk = nlat;
#pragma omp parallel for schedule(dynamic)
    for (int r = 0; r < nrows; r += chunk) {
        if (use991) oracle_fc2gp_991(gpout + (size_t)r * nlon, nlon, chunk);
        else oracle_fc2gp(gpout + (size_t)r * nlon, nlon, chunk);
    }
}

/* forward half of gridpointd: the gp2fc calls (plasim.f90:3415-3418), fc2sp
 * of the temperature and humidity tendencies and uv2dv (:3423-3428); gpin
 * [4L][NLAT*NLON] gtdt[L], gudt[L], gvdt[L], gqdt[L] is transformed in place;
 * spout [4L][2*NCSP] sdf[L], stf[L], szf[L], sqf[L] */
void oracle_forward_set_d(const oracle_leg *L, int nlev, double *gpin, double *spout, int use991) {
    int nlat = L->nlat, nlon = L->nlon, nrsp = 2 * L->ncsp;
    size_t nhor = (size_t)nlat * nlon;
    int nrows = (int)((4 * nlev) * (size_t)nlat);
    int chunk = nlat;
#pragma omp parallel for schedule(dynamic)
    for (int r = 0; r < nrows; r += chunk) {
        if (use991) oracle_gp2fc_991(gpin + (size_t)r * nlon, nlon, chunk);
        else oracle_gp2fc(gpin + (size_t)r * nlon, nlon, chunk);
    }
    double *gtdt = gpin, *gudt = gpin + nlev * nhor, *gvdt = gpin + 2 * nlev * nhor, *gqdt = gpin + 3 * nlev * nhor;
    double *sdf = spout, *stf = spout + (size_t)nlev * nrsp, *szf = spout + (size_t)2 * nlev * nrsp,
           *sqf = spout + (size_t)3 * nlev * nrsp;
#pragma omp parallel for schedule(dynamic)
    for (int v = 0; v < nlev; v++) {
        oracle_fc2sp(L, gtdt + v * nhor, stf + (size_t)v * nrsp, 1);
        oracle_fc2sp(L, gqdt + v * nhor, sqf + (size_t)v * nrsp, 1);
        oracle_uv2dv(L, gudt + v * nhor, gvdt + v * nhor, sdf + (size_t)v * nrsp, szf + (size_t)v * nrsp, 1, 1);
    }
}

/* radstep over all columns in blocks of whole latitude rows */
void oracle_radstep_par(const oracle_radpar *p, oracle_radio *io) {
    int nlat = p->nhor / p->nlon;
#pragma omp parallel for schedule(dynamic)
    for (int jl = 0; jl < nlat; jl++)
        oracle_radstep_range(p, io, jl * p->nlon, (jl + 1) * p->nlon);
}
