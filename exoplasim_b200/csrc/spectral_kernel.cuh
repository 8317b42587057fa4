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
    // the constants in the step's precision (the FP32 step's values are the
    // FP64 ones rounded once): t0 dsigma damp tdisst tdissq tdissd tdissz tfrc
    // [L each], g tau [L*L], bm1 [(ntru+1) L*L]
    const T *k;
    const T *sak;           // [L][NRSP]
    const int *nidx;        // total wavenumber of each spectral real
    int L, nrsp, ntru, nqspec, nsponge;
    double delt, delt2, pnu, pnu21, plavor, dampsp;
};

// up to SPEC_MAXB model states in one launch (blockIdx.y: the state)
constexpr int SPEC_MAXB = 12;
template <typename T>
struct SpecBatch {
    SpecArgs<T> s[SPEC_MAXB];
};

// Both steps work on a block of R spectral reals (threadIdx.x) by L levels
// (threadIdx.y): each thread owns one (real, level) value of every array, and
// the level profiles a real needs across levels sit in shared memory as
// [level][real] rows.  Every dot product over levels is still summed by one
// thread in the reference's order, so the FP64 instance rounds as before.
constexpr int SPEC_MAXTHREADS = 512;
__host__ __device__ inline int spec_reals(int L) { return L <= 16 ? 32 : (L <= 32 ? 16 : 8); }
template <typename T>
__host__ __device__ inline size_t spec_smem_a(int L) {
    const int R = spec_reals(L);
    return sizeof(T) * ((size_t)2 * L * L + 2 * (size_t)L + 4 * (size_t)L * R + 4 * (size_t)R);
}

template <typename T>
__global__ void __launch_bounds__(SPEC_MAXTHREADS) k_spectrala(const __grid_constant__ SpecBatch<T> P) {
    const SpecArgs<T> &A = P.s[blockIdx.y];
    extern __shared__ __align__(16) unsigned char ssm[];
    const int L = A.L, R = blockDim.x, r = threadIdx.x, l = threadIdx.y;
    T *c_g = reinterpret_cast<T *>(ssm), *c_tau = c_g + (size_t)L * L, *c_t0 = c_tau + (size_t)L * L,
      *c_ds = c_t0 + L;
    T *s_stt = c_ds + L, *s_atm = s_stt + (size_t)L * R, *s_zz = s_atm + (size_t)L * R, *s_sd = s_zz + (size_t)L * R;
    T *s_r = s_sd + (size_t)L * R;   // per real: spt0, apm, sop, zq
    const int tid = l * R + r, nthr = L * R;
    for (int i = tid; i < L * L; i += nthr) { c_g[i] = A.k[8 * L + i]; c_tau[i] = A.k[8 * L + L * L + i]; }
    for (int i = tid; i < L; i += nthr) { c_t0[i] = A.k[i]; c_ds[i] = A.k[L + i]; }
    const int j = blockIdx.x * R + r;
    const bool live = j < A.nrsp;
    const size_t n = (size_t)A.nrsp;
#define V(a, lv) (a)[(size_t)(lv) * n + j]
#define SH(a, lv, rr) a[(size_t)(lv) * R + (rr)]
    // every value of this (real, level) the step reads, loaded at once
    T v_sdt = 0, v_sdm = 0, v_szm = 0, v_sdp = 0, v_szp = 0, v_stp = 0, v_szt = 0, v_sqm = 0, v_sqp = 0, v_sqt = 0;
    // 0. the values at t-dt and the non-linear divergence tendency, saved
    int jn = 0;
    if (live) {
        jn = A.nidx[j];
        SH(s_stt, l, r) = V(A.stt, l);
        SH(s_atm, l, r) = V(A.stm, l);
        v_sdt = V(A.sdt, l); v_sdm = V(A.sdm, l); v_szm = V(A.szm, l); v_sdp = V(A.sdp, l);
        v_szp = V(A.szp, l); v_stp = V(A.stp, l); v_szt = V(A.szt, l);
        if (A.nqspec == 1) { v_sqm = V(A.sqm, l); v_sqp = V(A.sqp, l); v_sqt = V(A.sqt, l); }
        if (l == 0) {
            s_r[4 * r + 0] = A.spt[j];
            s_r[4 * r + 1] = A.spm[j];
            s_r[4 * r + 2] = A.sop[j];
            s_r[4 * r + 3] = jn > 0 ? (T)(1.0 / (jn * (jn + 1))) : (T)0;
        }
    }
    __syncthreads();
    // 1.a/b level l of the right-hand side of the implicit divergence equation (HS75 eq. 17)
    if (live) {
        const T spt0 = s_r[4 * r + 0], apm = s_r[4 * r + 1], sopj = s_r[4 * r + 2], zq = s_r[4 * r + 3];
        const int l2 = l;
        T zgt = 0, zgm = 0;
        for (int i = 0; i < L; i++) {
            zgt = zgt + c_g[i + L * l2] * SH(s_stt, i, r);
            zgm = zgm + c_g[i + L * l2] * SH(s_atm, i, r);
        }
        const T z0 = c_t0[l2];
        const T zt = zgt - z0 * spt0;
        const T zm = zgm + z0 * apm;
        const T za = v_sdt * zq + sopj;
        const T zb = v_sdm * zq;
        SH(s_zz, l2, r) = zb + (T)A.delt * (zm + za + (T)A.delt * zt);
    }
    __syncthreads();
    // the new divergence at level l: bm1(n) applied to the right-hand side;
    // modes n = 0 (and the first, mass-carrying real pair) carry none
    if (live) {
        const T *bm = A.k + 8 * L + 2 * L * L + (size_t)jn * L * L;
        T zsum = 0;
        if (jn > 0 && j > 1)
            for (int l2 = 0; l2 < L; l2++) zsum = zsum + SH(s_zz, l2, r) * bm[l2 + L * l];
        SH(s_sd, l, r) = zsum;
    }
    __syncthreads();
    if (live) {
        const T pnu = (T)A.pnu, pnu21 = (T)A.pnu21, d2 = (T)A.delt2;
        if (l == 0) {
            // 2. (-log) surface-pressure tendency (HS75 eq. 15); 4.a the filter's first part
            const T apm = s_r[4 * r + 1];
            T spt = s_r[4 * r + 0];
            for (int i = 0; i < L; i++) spt = spt + c_ds[i] * SH(s_sd, i, r);
            A.spt[j] = spt;
            A.spm[j] = pnu21 * A.spp[j] + pnu * apm;
            A.spp[j] = j > 1 ? apm - d2 * spt : (T)0;      // conserve p (spp(1:2) = 0)
        }
        // 3. temperature (eq. 14) and 4.b the tendencies added, level l
        T dot = 0;
        for (int i = 0; i < L; i++) dot = dot + c_tau[i + L * l] * SH(s_sd, i, r);
        const T stt = SH(s_stt, l, r) - dot;
        const T sd = SH(s_sd, l, r);
        const T adm = v_sdm, azm = v_szm, atm = SH(s_atm, l, r);
        V(A.stt, l) = stt;
        V(A.sdt, l) = sd;
        V(A.sdm, l) = pnu21 * v_sdp + pnu * adm;
        V(A.szm, l) = pnu21 * v_szp + pnu * azm;
        V(A.stm, l) = pnu21 * v_stp + pnu * atm;
        V(A.sdp, l) = (T)2.0 * sd - adm;
        V(A.stp, l) = d2 * stt + atm;
        V(A.szp, l) = d2 * v_szt + azm;
        if (A.nqspec == 1) {
            const T aqm = v_sqm;
            V(A.sqm, l) = pnu21 * v_sqp + pnu * aqm;
            V(A.sqp, l) = d2 * v_sqt + aqm;
        }
    }
#undef V
#undef SH
}

// spectrald: one thread per (real, level); the sponge's coupling of the top
// level to the second goes through shared memory
template <typename T>
__global__ void __launch_bounds__(SPEC_MAXTHREADS) k_spectrald(const __grid_constant__ SpecBatch<T> P) {
    const SpecArgs<T> &A = P.s[blockIdx.y];
    __shared__ T s_stp[2][32];
    const int L = A.L, r = threadIdx.x, l = threadIdx.y;
    const int j = blockIdx.x * blockDim.x + r;
    const bool live = j < A.nrsp;
    const size_t n = (size_t)A.nrsp;
    const T *damp = A.k + 2 * L, *tdisst = A.k + 3 * L, *tdissq = A.k + 4 * L, *tdissd = A.k + 5 * L,
            *tdissz = A.k + 6 * L, *tfrc = A.k + 7 * L;
    const T d2 = (T)A.delt2, pnu = (T)A.pnu;
#define V(a, lv) (a)[(size_t)(lv) * n + j]
    // the diabatic tendencies added, then the implicit restoration, drag and
    // diffusion tendencies of the new values (spectrald :3690-3760), level l
    if (live) {
        const T szp = V(A.szp, l) + d2 * V(A.szt, l);
        const T stp = V(A.stp, l) + d2 * V(A.stt, l);
        const T sdp = V(A.sdp, l) + d2 * V(A.sdt, l);
        const T dm = damp[l], tt = tdisst[l], td = tdissd[l], tz = tdissz[l], tf = tfrc[l];
        const T sk = A.sak[(size_t)l * n + j];
        T stt = ((-dm - tt * sk) * stp + dm * V(A.srp, l)) / ((T)1. + d2 * (dm + tt * sk));
        const T s1 = -tf * sdp / ((T)1. + d2 * tf);
        const T s2 = -td * sk * sdp / ((T)1. + d2 * td * sk);
        const T sdt = s1 + s2;
        const T z1 = -tf * szp / ((T)1. + d2 * tf);
        const T z2 = -tz * sk * szp / ((T)1. + d2 * tz * sk);
        T szt = z1 + z2;
        if (j == 2) szt = szt + (T)A.plavor * (tf / ((T)1. + d2 * tf) + tz * sk / ((T)1. + d2 * tz * sk));
        if (l < 2) s_stp[l][r] = stp;
        if (A.nqspec == 1) {
            const T tq = tdissq[l];
            const T sqp = V(A.sqp, l) + d2 * V(A.sqt, l);
            const T sqt = -tq * sk * sqp / ((T)1. + d2 * tq * sk);
            V(A.sqt, l) = sqt;
            const T sqp2 = sqp + d2 * sqt;
            V(A.sqp, l) = sqp2;
            V(A.sqm, l) = V(A.sqm, l) + pnu * sqp2;
        }
        V(A.sdt, l) = sdt;
        V(A.szt, l) = szt;
        const T szp2 = szp + d2 * szt, sdp2 = sdp + d2 * sdt;
        V(A.szp, l) = szp2;
        V(A.sdp, l) = sdp2;
        V(A.szm, l) = V(A.szm, l) + pnu * szp2;
        V(A.sdm, l) = V(A.sdm, l) + pnu * sdp2;
        // the sponge relaxes the top level's temperature to the second's
        // (applied once that level's value is known, below)
        if (l > 0 || A.nsponge <= 0) {
            V(A.stt, l) = stt;
            const T stp2 = stp + d2 * stt;
            V(A.stp, l) = stp2;
            V(A.stm, l) = V(A.stm, l) + pnu * stp2;
        } else {
            V(A.stt, 0) = stt;   // finished below
        }
    }
    __syncthreads();
    if (live && l == 0) {
        if (A.nsponge > 0) {
            T stt = V(A.stt, 0);
            stt = (T)A.dampsp * (s_stp[1][r] - s_stp[0][r]) + stt;
            V(A.stt, 0) = stt;
            const T stp2 = s_stp[0][r] + d2 * stt;
            V(A.stp, 0) = stp2;
            V(A.stm, 0) = V(A.stm, 0) + pnu * stp2;
        }
        const T spp = j > 1 ? A.spp[j] : (T)0;           // conserve p
        A.spp[j] = spp;
        A.spm[j] = A.spm[j] + pnu * spp;
    }
#undef V
}

// launch shapes: blocks of spec_reals(L) reals by L levels, states along y
// (every state of a batch has the plan's NRSP and the constants' L)
template <typename T>
inline exotx_status spec_launch(const SpecBatch<T> &P, int n, bool d_part, cudaStream_t s) {
    const SpecArgs<T> &A = P.s[0];
    const int R = spec_reals(A.L);
    const dim3 block((unsigned)R, (unsigned)A.L), grid((unsigned)((A.nrsp + R - 1) / R), (unsigned)n);
    if (d_part) {
        k_spectrald<T><<<grid, block, 0, s>>>(P);
    } else {
        const size_t smem = spec_smem_a<T>(A.L);
        if (smem > 48 * 1024)
            EXOTX_CUDA(cudaFuncSetAttribute(k_spectrala<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_spectrala<T><<<grid, block, smem, s>>>(P);
    }
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}

}  // namespace exotx
