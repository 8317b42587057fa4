// The semi-implicit spectral time step (plasim.f90 spectrala :2757-2918,
// spectrald :3645-3999): kernels shared by spectral.cu (FP32) and
// spectral_fp64.cu (FP64, compiled without FMA contraction so that every
// product and sum is rounded in the reference's order).
//
// spectrala works on one spectral real (a mode's re or im part) per thread,
// through all levels: the level profiles it needs more than once (stt, stm,
// the right-hand side zz of the implicit divergence equation and the new
// divergence) sit in shared memory as [level][thread] rows, so a warp's
// accesses fall in distinct banks; the level matrices g, tau and the inverse
// bm1(n) of the semi-implicit operator are read from global memory (L2).
// spectrald is element-wise over (level, real).
#pragma once
#include "exotx_internal.cuh"

namespace exotx {

template <typename T>
struct SpecArgs {
    T *sdp, *szp, *stp, *sqp, *spp, *sdm, *szm, *stm, *sqm, *spm, *sdt, *szt, *stt, *sqt, *spt;
    const T *sop, *srp;
    const double *k;        // t0 dsigma damp tdisst tdissq tdissd tdissz tfrc [L each], g tau [L*L], bm1 [(ntru+1) L*L]
    const double *sak;      // [L][NRSP]
    const int *nidx;        // total wavenumber of each spectral real
    int L, nrsp, ntru, nqspec, nsponge;
    double delt, delt2, pnu, pnu21, plavor, dampsp;
};

template <typename T>
__global__ void k_spectrala(const SpecArgs<T> A) {
    extern __shared__ __align__(16) unsigned char ssm[];
    const int nt = blockDim.x, tx = threadIdx.x, L = A.L;
    T *s_stt = reinterpret_cast<T *>(ssm), *s_atm = s_stt + (size_t)L * nt, *s_zz = s_atm + (size_t)L * nt,
      *s_sd = s_zz + (size_t)L * nt;
    const int j = blockIdx.x * nt + tx;
    if (j >= A.nrsp) return;
    const size_t n = (size_t)A.nrsp;
    const double *t0 = A.k, *dsigma = A.k + L, *gm = A.k + 8 * L, *taum = gm + L * L, *bm1 = taum + L * L;
#define V(a, l) (a)[(size_t)(l) * n + j]
#define SH(a, l) a[(size_t)(l) * nt + tx]
    // 0. the values at t-dt and the non-linear divergence tendency, saved
    const T apm = A.spm[j];
    for (int l = 0; l < L; l++) { SH(s_stt, l) = V(A.stt, l); SH(s_atm, l) = V(A.stm, l); }
    // 1.a/b the right-hand side of the implicit divergence equation (HS75 eq. 17)
    const int jn = A.nidx[j];
    const T spt0 = A.spt[j], sopj = A.sop[j];
    const T zq = jn > 0 ? (T)(1.0 / (jn * (jn + 1))) : (T)0;
    for (int l2 = 0; l2 < L; l2++) {
        T zgt = 0, zgm = 0;
        for (int i = 0; i < L; i++) {
            zgt = zgt + (T)gm[i + L * l2] * SH(s_stt, i);
            zgm = zgm + (T)gm[i + L * l2] * SH(s_atm, i);
        }
        const T z0 = (T)t0[l2];
        const T zt = zgt - z0 * spt0;
        const T zm = zgm + z0 * apm;
        const T za = V(A.sdt, l2) * zq + sopj;
        const T zb = V(A.sdm, l2) * zq;
        SH(s_zz, l2) = zb + (T)A.delt * (zm + za + (T)A.delt * zt);
    }
    // the new divergence: bm1(n) applied to the right-hand side; modes n = 0
    // (and the first, mass-carrying real pair) carry none
    const double *bm = bm1 + (size_t)jn * L * L;
    for (int l = 0; l < L; l++) {
        T zsum = 0;
        if (jn > 0 && j > 1)
            for (int l2 = 0; l2 < L; l2++) zsum = zsum + SH(s_zz, l2) * (T)bm[l2 + L * l];
        SH(s_sd, l) = zsum;
    }
    // 2. (-log) surface-pressure tendency (HS75 eq. 15), 3. temperature (eq. 14)
    T spt = spt0;
    for (int l = 0; l < L; l++) spt = spt + (T)dsigma[l] * SH(s_sd, l);
    A.spt[j] = spt;
    // 4.a time filter, first part; 4.b the tendencies added
    const T pnu = (T)A.pnu, pnu21 = (T)A.pnu21, d2 = (T)A.delt2;
    A.spm[j] = pnu21 * A.spp[j] + pnu * apm;
    A.spp[j] = j > 1 ? apm - d2 * spt : (T)0;          // conserve p (spp(1:2) = 0)
    for (int l = 0; l < L; l++) {
        T dot = 0;
        for (int i = 0; i < L; i++) dot = dot + (T)taum[i + L * l] * SH(s_sd, i);
        const T stt = SH(s_stt, l) - dot;
        const T sd = SH(s_sd, l);
        const T adm = V(A.sdm, l), azm = V(A.szm, l), atm = SH(s_atm, l);
        V(A.stt, l) = stt;
        V(A.sdt, l) = sd;
        V(A.sdm, l) = pnu21 * V(A.sdp, l) + pnu * adm;
        V(A.szm, l) = pnu21 * V(A.szp, l) + pnu * azm;
        V(A.stm, l) = pnu21 * V(A.stp, l) + pnu * atm;
        V(A.sdp, l) = (T)2.0 * sd - adm;
        V(A.stp, l) = d2 * stt + atm;
        V(A.szp, l) = d2 * V(A.szt, l) + azm;
        if (A.nqspec == 1) {
            const T aqm = V(A.sqm, l);
            V(A.sqm, l) = pnu21 * V(A.sqp, l) + pnu * aqm;
            V(A.sqp, l) = d2 * V(A.sqt, l) + aqm;
        }
    }
#undef V
#undef SH
}

// spectrald: one thread per spectral real, through the levels
template <typename T>
__global__ void k_spectrald(const SpecArgs<T> A) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= A.nrsp) return;
    const int L = A.L;
    const size_t n = (size_t)A.nrsp;
    const double *damp = A.k + 2 * L, *tdisst = A.k + 3 * L, *tdissq = A.k + 4 * L, *tdissd = A.k + 5 * L,
                 *tdissz = A.k + 6 * L, *tfrc = A.k + 7 * L;
    const T d2 = (T)A.delt2, pnu = (T)A.pnu;
#define V(a, l) (a)[(size_t)(l) * n + j]
    // the diabatic tendencies added, then the implicit restoration, drag and
    // diffusion tendencies of the new values (spectrald :3690-3760)
    T stp1 = 0, stp0 = 0;
    for (int l = 0; l < L; l++) {
        const T szp = V(A.szp, l) + d2 * V(A.szt, l);
        const T stp = V(A.stp, l) + d2 * V(A.stt, l);
        const T sdp = V(A.sdp, l) + d2 * V(A.sdt, l);
        const T dm = (T)damp[l], tt = (T)tdisst[l], td = (T)tdissd[l], tz = (T)tdissz[l], tf = (T)tfrc[l];
        const T sk = (T)A.sak[(size_t)l * n + j];
        T stt = ((-dm - tt * sk) * stp + dm * V(A.srp, l)) / ((T)1. + d2 * (dm + tt * sk));
        const T s1 = -tf * sdp / ((T)1. + d2 * tf);
        const T s2 = -td * sk * sdp / ((T)1. + d2 * td * sk);
        const T sdt = s1 + s2;
        const T z1 = -tf * szp / ((T)1. + d2 * tf);
        const T z2 = -tz * sk * szp / ((T)1. + d2 * tz * sk);
        T szt = z1 + z2;
        if (j == 2) szt = szt + (T)A.plavor * (tf / ((T)1. + d2 * tf) + tz * sk / ((T)1. + d2 * tz * sk));
        if (l == 0) stp0 = stp;
        if (l == 1) stp1 = stp;
        if (A.nqspec == 1) {
            const T tq = (T)tdissq[l];
            const T sqp = V(A.sqp, l) + d2 * V(A.sqt, l);
            const T sqt = -tq * sk * sqp / ((T)1. + d2 * tq * sk);
            V(A.sqt, l) = sqt;
            const T sqp2 = sqp + d2 * sqt;
            V(A.sqp, l) = sqp2;
            V(A.sqm, l) = V(A.sqm, l) + pnu * sqp2;
        }
        // the sponge relaxes the top level's temperature to the second's,
        // applied below once that level's value is known
        V(A.stt, l) = stt;
        V(A.sdt, l) = sdt;
        V(A.szt, l) = szt;
        const T szp2 = szp + d2 * szt, sdp2 = sdp + d2 * sdt;
        V(A.szp, l) = szp2;
        V(A.sdp, l) = sdp2;
        V(A.stp, l) = stp;   // the diabatic step only; the restoration step follows
        V(A.szm, l) = V(A.szm, l) + pnu * szp2;
        V(A.sdm, l) = V(A.sdm, l) + pnu * sdp2;
    }
    for (int l = 0; l < L; l++) {
        T stt = V(A.stt, l);
        if (l == 0 && A.nsponge > 0) {
            stt = (T)A.dampsp * (stp1 - stp0) + stt;
            V(A.stt, 0) = stt;
        }
        const T stp2 = V(A.stp, l) + d2 * stt;
        V(A.stp, l) = stp2;
        V(A.stm, l) = V(A.stm, l) + pnu * stp2;
    }
    const T spp = j > 1 ? A.spp[j] : (T)0;           // conserve p
    A.spp[j] = spp;
    A.spm[j] = A.spm[j] + pnu * spp;
#undef V
}

}  // namespace exotx
