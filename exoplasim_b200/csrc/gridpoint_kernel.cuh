// The grid-point step of gridpointa (plasim.f90:2441-2455): the kernel,
// shared by gridpoint.cu (FP32) and gridpoint_fp64.cu (FP64, compiled
// without FMA contraction so that every product and sum is rounded as the
// reference's 8-byte build rounds it).
#pragma once
#include "exotx_internal.cuh"

namespace exotx {

constexpr int GP_THREADS = 128;

template <typename T>
struct GpArgs {
    const T *gin;
    T *gout, *dw;
    const double *sid;      // per latitude (rcsq = 1/(1 - sid^2))
    const double *k;        // constants block
    const T *dq;            // nqspec == 0: grid humidity [inst][L][nhor]
    long long ncol;         // instances x nhor
    int L, nhor, nlon, nqspec;
    double akap, rdbrv, adv, psurf, ww;
};

template <typename T>
__global__ void __launch_bounds__(GP_THREADS) k_gridpoint(const GpArgs<T> A) {
    extern __shared__ __align__(16) unsigned char gsm[];
    T *sv = reinterpret_cast<T *>(gsm);                 // zvgpg      [L][GP_THREADS]
    T *sb = sv + (size_t)A.L * GP_THREADS;              // zvgpg + gd [L][GP_THREADS]
    T *s1 = sb + (size_t)A.L * GP_THREADS;              // ztv1 - gt  [L][GP_THREADS]
    const long long col = blockIdx.x * (long long)GP_THREADS + threadIdx.x;
    if (col >= A.ncol) return;
    const int L = A.L, tx = threadIdx.x;
    const long long inst = col / A.nhor;
    const int h = (int)(col - inst * A.nhor);
    const size_t n = (size_t)A.nhor;
    const T *gin = A.gin + (size_t)inst * (6 * L + 3) * n;
    T *gout = A.gout + (size_t)inst * (9 * L + 1) * n;
    const double *dsigma = A.k, *sigmah = A.k + L, *rdsig = A.k + 2 * L, *t0 = A.k + 3 * L, *t01s2 = A.k + 4 * L,
                 *tkp = A.k + 5 * L, *gm = A.k + 6 * L, *cm = A.k + 6 * L + L * L;
#define IN(f, k) gin[((size_t)(f) * L + (k)) * n + h]
#define OUT(f, k) gout[((size_t)(f) * L + (k)) * n + h]
#define SH(a, k) a[(size_t)(k) * GP_THREADS + tx]
    const T gpj = gin[(size_t)6 * L * n + h], gpm = gin[((size_t)6 * L + 1) * n + h];
    const T gp = exp(gin[((size_t)6 * L + 2) * n + h]);   // gp = exp(gp), plasim.f90:2441
    const double s = A.sid[h / A.nlon];
    const T rc = (T)(1.0 / (1.0 - s * s));
    const T rdbrv1 = (T)1. / (T)A.rdbrv - (T)1.;
    // pass 1: profiles and the column totals of the divergence and of zvgpg
    T zsumd = 0, gvp = 0;
    for (int k = 0; k < L; k++) {
        const T gu = IN(0, k), gv = IN(1, k), gt = IN(2, k), gd = IN(3, k), gq = IN(5, k);
        const T zv = rc * (gu * gpm + gv * gpj);
        T zq;
        if (A.nqspec == 1) zq = fmax(gq / gp, (T)0.);
        else zq = A.dq ? fmax(A.dq[((size_t)inst * L + k) * n + h], (T)0.) : (T)0.;
        const T tv1 = (gt + (T)t0[k]) * ((T)1. + rdbrv1 * zq) - (T)t0[k];
        SH(sv, k) = zv;
        SH(sb, k) = zv + gd;
        SH(s1, k) = tv1 - gt;
        if (k == 0) { zsumd = (T)dsigma[0] * gd; gvp = (T)dsigma[0] * zv; }
        else { zsumd = zsumd + (T)dsigma[k] * gd; gvp = gvp + (T)dsigma[k] * zv; }
    }
    const T tot = zsumd + gvp;
    // pass 2, level by level: sigma-dot, vertical advection terms and tendencies
    T psd = 0, psv = 0;                 // running sums of dsigma * gd and of dsigma * zvgpg
    T gtd_m = 0, gqm_m = 0, gud_m = 0, gvd_m = 0;   // the level above's products
    T zs = 0;                           // zsumd of the tendency loop (plasim.f90:2661, :2692)
    for (int k = 0; k < L; k++) {
        const T gu = IN(0, k), gv = IN(1, k), gt = IN(2, k), gd = IN(3, k), gz = IN(4, k), gq = IN(5, k);
        const T zv = SH(sv, k);
        T zq;
        if (A.nqspec == 1) zq = fmax(gq / gp, (T)0.);
        else zq = A.dq ? fmax(A.dq[((size_t)inst * L + k) * n + h], (T)0.) : (T)0.;
        const T tv1 = (gt + (T)t0[k]) * ((T)1. + rdbrv1 * zq) - (T)t0[k];
        const T tv2 = (gt + (T)t0[k]) * ((T)1. + rdbrv1 * zq) / ((T)1. + (T)A.adv * zq) - (T)t0[k];
        // this level's products of the sigma-dot flux with the layer differences
        T gtd = 0, gqm = 0, gud = 0, gvd = 0;
        if (k < L - 1) {
            if (k == 0) { psd = (T)dsigma[0] * gd; psv = (T)dsigma[0] * zv; }
            else { psd = psd + (T)dsigma[k] * gd; psv = psv + (T)dsigma[k] * zv; }
            const T zsdotp = ((T)sigmah[k] * tot - (psd + psv));
            gtd = zsdotp * (IN(2, k + 1) - gt);
            gqm = zsdotp * (IN(5, k + 1) + gq);
            gud = zsdotp * (IN(0, k + 1) - gu);
            gvd = zsdotp * (IN(1, k + 1) - gv);
        }
        T gtn, gqn, guz, gvz, dwv;
        if (k == 0) {
            zs = zv * (T)dsigma[0];
            gtn = gt * gd - (T)A.akap * tv2 * gd - (T)rdsig[0] * (gtd + (T)t01s2[0] * ((T)sigmah[0] * gvp - zs));
            gqn = -(T)rdsig[0] * gqm;
            guz = -gu * gz - gpj * tv1 - (T)rdsig[0] * gvd;
            gvz = gv * gz - gpm * tv1 - (T)rdsig[0] * gud;
            dwv = gd * gp * (T)A.psurf * (T)A.ww;
        } else {
            T ztpta = (T)cm[0 + L * k] * SH(sv, 0);
            T ztptb = (T)cm[0 + L * k] * SH(sb, 0);
            for (int j = 1; j <= k; j++) {
                ztpta = ztpta + (T)cm[j + L * k] * SH(sv, j);
                ztptb = ztptb + (T)cm[j + L * k] * SH(sb, j);
            }
            if (k < L - 1) {
                zs = zs + zv * (T)dsigma[k];
                gtn = gt * gd + (T)A.akap * tv2 * (zv - ztptb) + (T)tkp[k] * (zv - ztpta) -
                      (T)rdsig[k] * (gtd + gtd_m + gvp * ((T)t01s2[k] * (T)sigmah[k] + (T)t01s2[k - 1] * (T)sigmah[k - 1]) -
                                     zs * ((T)t01s2[k - 1] + (T)t01s2[k]) + zv * (T)dsigma[k] * (T)t01s2[k - 1]);
                gqn = -(T)rdsig[k] * (gqm - gqm_m);
                guz = -gu * gz - gpj * tv1 - (T)rdsig[k] * (gvd + gvd_m);
                gvz = gv * gz - gpm * tv1 - (T)rdsig[k] * (gud + gud_m);
            } else {
                gtn = gt * gd + (T)A.akap * tv2 * (zv - ztptb) + (T)tkp[k] * (zv - ztpta) -
                      (T)rdsig[k] * (gtd_m + (T)t01s2[k - 1] * ((T)sigmah[k - 1] * gvp - zs));
                gqn = (T)rdsig[k] * gqm_m;
                guz = -gu * gz - gpj * tv1 - (T)rdsig[k] * gvd_m;
                gvz = gv * gz - gpm * tv1 - (T)rdsig[k] * gud_m;
            }
            dwv = (zv - ztptb) * gp * (T)A.psurf * (T)A.ww;
        }
        // non-linear geopotential, summed over every level as dot_product does
        T dot = 0;
        for (int i = 0; i < L; i++) dot = dot + (T)gm[i + L * k] * SH(s1, i);
        const T gphi = dot * (T)2. / rc;
        T ke = gu * gu + gv * gv;
        ke = ke + gphi;
        OUT(0, k) = gtn;                 // gtn
        OUT(1, k) = gqn;                 // gqn
        OUT(2, k) = gu * gt;             // gut
        OUT(3, k) = gv * gt;             // gvt
        OUT(4, k) = guz;                 // guz
        OUT(5, k) = gvz;                 // gvz
        OUT(6, k) = ke;                  // gke
        gout[((size_t)7 * L + 1 + k) * n + h] = gu * gq;       // guq
        gout[((size_t)8 * L + 1 + k) * n + h] = gv * gq;       // gvq
        if (A.dw) A.dw[((size_t)inst * L + k) * n + h] = dwv;
        gtd_m = gtd; gqm_m = gqm; gud_m = gud; gvd_m = gvd;
    }
    gout[(size_t)7 * L * n + h] = gvp;   // gvpp
#undef IN
#undef OUT
#undef SH
}

}  // namespace exotx
