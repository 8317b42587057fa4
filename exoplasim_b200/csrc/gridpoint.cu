// The grid-point step of gridpointa between the inverse and the forward
// transforms (plasim.f90:2441-2455): gp = exp(gp); calcgp (:2587-2755) -- the
// vertical sigma-dot velocity, adiabatic temperature tendency, humidity flux
// divergence, the vorticity/divergence flux terms and the non-linear
// geopotential; then the flux products gut, gvt, gke (+ gphi), guq, gvq.
//
// Everything here is per grid column, so one thread owns one column of one
// instance: it reads the inverse set's 6L+3 fields of that column and writes
// the forward set's 9L+1 fields, with consecutive threads on consecutive
// columns (every access is a coalesced row of the NHOR-fastest layout).  The
// O(L^2) sums (the c(j,k) and g(i,k) matrices of the semi-implicit scheme)
// need the whole column's zvgpg, zvgpg + gd and ztv1 - gt: those three
// profiles live in shared memory, laid out level-major so that a warp's
// accesses fall in distinct banks.  The matrices and per-level constants are
// one small block, staged in shared memory in the step's precision once per
// block where it fits (every thread of a warp then reads it word for word
// alike).  The kernel is HBM-bound: (15L+4) values move per column.
#include <cmath>
#include <cstring>
#include <vector>
#include "gridpoint_kernel.cuh"

struct exotx_gpconst_s {
    exotx_gp_params h;  // host copy
    double *d = nullptr;  // device: dsigma sigmah rdsig t0 t01s2 tkp [L each], g, c [L*L each]
    int g_lower = 0;      // g(i, k) = 0 for every i < k (initsi's g is)
};

namespace exotx {

exotx_status launch_gridpoint_fp64(const GpArgs<double> &A, cudaStream_t s);

static exotx_status launch_gridpoint_fp32(const GpArgs<float> &A, cudaStream_t s) { return gp_launch<float>(A, s); }

}  // namespace exotx

using namespace exotx;

// initsi (plasim.f90:1709-1745) and rdsig (:1564) from the levels, t0 and akap
static void gp_derive(exotx_gp_params *p) {
    const int L = p->nlev;
    double zalp[64] = {0};
    for (int j = 0; j < L; j++) p->tkp[j] = p->akap * p->t0[j];
    for (int j = 0; j < L - 1; j++) p->t01s2[j] = p->t0[j + 1] - p->t0[j];
    p->t01s2[L - 1] = 0.0;
    for (int j = 1; j < L; j++) zalp[j] = log(p->sigmah[j]) - log(p->sigmah[j - 1]);
    for (int i = 0; i < L * L; i++) p->g[i] = 0.0;
    p->g[0] = 1.0;
    for (int jl = 1; jl < L; jl++) {
        p->g[jl + L * jl] = 1.0 - zalp[jl] * p->sigmah[jl - 1] / p->dsigma[jl];
        for (int k = 0; k < jl; k++) p->g[jl + L * k] = zalp[jl];
    }
    for (int jl = 0; jl < L; jl++)
        for (int k = 0; k < L; k++) p->c[jl + L * k] = p->g[k + L * jl] * (p->dsigma[jl] / p->dsigma[k]);
    for (int j = 0; j < L; j++) p->rdsig[j] = 0.5 / p->dsigma[j];
}

EXOTX_API exotx_status exotx_gp_params_default(int nlev, exotx_gp_params *p) {
    if (!p || nlev < 2 || nlev > 64) return EXOTX_BAD_ARG;
    memset(p, 0, sizeof(*p));
    p->nlev = nlev;
    p->nqspec = 1;
    // Earth defaults (plasimmod.f90, p_earth.f90; scalings plasim.f90:1316-1322)
    const double gascon = 287.0, akap = 0.286, rv = 461.51, acpv = 1870.0, plarad = 6371220.0,
                 sidereal_day = 86164.0, twopi = 2.0 * 3.14159265359;
    p->akap = akap;
    p->rdbrv = gascon / rv;
    p->adv = acpv / (gascon / akap) - 1.0;
    p->psurf = 101100.0;
    p->ww = twopi / sidereal_day;
    const double cv = plarad * p->ww, ct = cv * cv / gascon;
    for (int j = 0; j < nlev; j++) {
        const double z = (double)(j + 1) / nlev;
        p->sigmah[j] = 0.75 * z + 1.75 * z * z * z - 1.5 * z * z * z * z;   // plasim.f90:1554-1564
    }
    p->dsigma[0] = p->sigmah[0];
    for (int j = 1; j < nlev; j++) p->dsigma[j] = p->sigmah[j] - p->sigmah[j - 1];
    // a reference profile: 288 K at the surface, 6.5 K/km up to 216.65 K (dimensionless by ct)
    for (int j = 0; j < nlev; j++) {
        const double sig = j == 0 ? 0.5 * p->sigmah[0] : 0.5 * (p->sigmah[j - 1] + p->sigmah[j]);
        double t = 288.0 * pow(sig, 0.0065 * gascon / 9.80665);
        p->t0[j] = (t < 216.65 ? 216.65 : t) / ct;
    }
    gp_derive(p);
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_gp_params_derive(exotx_gp_params *p) {
    if (!p || p->nlev < 2 || p->nlev > 64) return EXOTX_BAD_ARG;
    gp_derive(p);
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_gpconst_create(const exotx_gp_params *p, exotx_gpconst *out) {
    if (!p || !out || p->nlev < 2 || p->nlev > 64) return EXOTX_BAD_ARG;
    const int L = p->nlev;
    std::vector<double> k((size_t)6 * L + 2 * (size_t)L * L);
    for (int j = 0; j < L; j++) {
        k[j] = p->dsigma[j]; k[L + j] = p->sigmah[j]; k[2 * L + j] = p->rdsig[j];
        k[3 * L + j] = p->t0[j]; k[4 * L + j] = p->t01s2[j]; k[5 * L + j] = p->tkp[j];
    }
    for (int i = 0; i < L * L; i++) { k[6 * L + i] = p->g[i]; k[6 * L + L * L + i] = p->c[i]; }
    exotx_gpconst c = new exotx_gpconst_s();
    c->h = *p;
    c->g_lower = 1;
    for (int k = 0; k < L; k++)
        for (int i = 0; i < k; i++)
            if (p->g[i + L * k] != 0.0) c->g_lower = 0;
    if (cudaMalloc(&c->d, sizeof(double) * k.size()) != cudaSuccess) { delete c; return EXOTX_NO_MEM; }
    if (cudaMemcpy(c->d, k.data(), sizeof(double) * k.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(c->d);
        delete c;
        return EXOTX_CUDA_ERR;
    }
    *out = c;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_gpconst_destroy(exotx_gpconst c) {
    if (!c) return EXOTX_BAD_ARG;
    cudaFree(c->d);
    delete c;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_gridpoint(exotx_plan p, exotx_gpconst c, int prec, const void *gin, void *gout,
                                       void *dw, const void *dq, int ninst, exotx_stream s) {
    if (!p || !c || (prec != EXOTX_FP64 && prec != EXOTX_FP32 && prec != EXOTX_MIXED)) return EXOTX_BAD_ARG;
    if (ninst == 0) return EXOTX_OK;
    if (!gin || !gout || ninst < 0) return EXOTX_BAD_ARG;
    if (c->h.nqspec == 0 && !dq) return EXOTX_BAD_ARG;
    const int L = c->h.nlev;
    const size_t smem = 3 * (size_t)L * GP_THREADS * (prec == EXOTX_FP64 ? 8 : 4);
    if (smem > 227 * 1024) return EXOTX_BAD_DIM;
    const long long nhor = (long long)p->nlat * p->nlon;
    if (prec == EXOTX_FP64) {
        GpArgs<double> A;
        A.gin = (const double *)gin; A.gout = (double *)gout; A.dw = (double *)dw; A.dq = (const double *)dq;
        A.sid = p->d_sid; A.k = c->d; A.ncol = nhor * ninst;
        A.L = L; A.nhor = (int)nhor; A.nlon = p->nlon; A.nqspec = c->h.nqspec; A.g_lower = c->g_lower;
        A.akap = c->h.akap; A.rdbrv = c->h.rdbrv; A.adv = c->h.adv; A.psurf = c->h.psurf; A.ww = c->h.ww;
        return launch_gridpoint_fp64(A, (cudaStream_t)s);
    }
    GpArgs<float> A;
    A.gin = (const float *)gin; A.gout = (float *)gout; A.dw = (float *)dw; A.dq = (const float *)dq;
    A.sid = p->d_sid; A.k = c->d; A.ncol = nhor * ninst;
    A.L = L; A.nhor = (int)nhor; A.nlon = p->nlon; A.nqspec = c->h.nqspec; A.g_lower = c->g_lower;
    A.akap = c->h.akap; A.rdbrv = c->h.rdbrv; A.adv = c->h.adv; A.psurf = c->h.psurf; A.ww = c->h.ww;
    return launch_gridpoint_fp32(A, (cudaStream_t)s);
}
