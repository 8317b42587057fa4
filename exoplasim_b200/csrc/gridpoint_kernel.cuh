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
    int g_lower;            // g(i, k) = 0 for every i < k
    double akap, rdbrv, adv, psurf, ww;
};

// the constants block in the step's precision: in shared memory (SK, staged
// once per block) or read from global memory and rounded at each use
template <typename T, bool SK>
struct GpConsts {
    const T *s;
    const double *g;
    __device__ __forceinline__ T operator()(int i) const {
        if constexpr (SK) return s[i];
        else return (T)g[i];
    }
};
template <typename T>
__host__ __device__ inline size_t gp_smem(int L, bool sk) {
    return sizeof(T) * (3 * (size_t)L * GP_THREADS + (sk ? 6 * (size_t)L + 2 * (size_t)L * L : 0));
}

// LC > 0: the level count fixed at compile time, so the index arithmetic of
// the profiles and constants folds (the arithmetic, and its order, is the same)
template <typename T, bool SK, int LC>
__global__ void __launch_bounds__(GP_THREADS) k_gridpoint(const GpArgs<T> A) {
    extern __shared__ __align__(16) unsigned char gsm[];
    T *sv = reinterpret_cast<T *>(gsm);                 // zvgpg      [L][GP_THREADS]
    T *sb = sv + (size_t)A.L * GP_THREADS;              // zvgpg + gd [L][GP_THREADS]
    T *s1 = sb + (size_t)A.L * GP_THREADS;              // ztv1 - gt  [L][GP_THREADS]
    T *sk = s1 + (size_t)A.L * GP_THREADS;              // constants (SK)
    if constexpr (SK) {
        for (int i = threadIdx.x; i < 6 * A.L + 2 * A.L * A.L; i += GP_THREADS) sk[i] = (T)A.k[i];
        __syncthreads();
    }
    const GpConsts<T, SK> K{sk, A.k};
    const long long col = blockIdx.x * (long long)GP_THREADS + threadIdx.x;
    if (col >= A.ncol) return;
    const int L = LC > 0 ? LC : A.L, tx = threadIdx.x;
    const long long inst = col / A.nhor;
    const int h = (int)(col - inst * A.nhor);
    const size_t n = (size_t)A.nhor;
    const T *gin = A.gin + (size_t)inst * (6 * L + 3) * n;
    T *gout = A.gout + (size_t)inst * (9 * L + 1) * n;
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
        const T tv1 = (gt + K(3 * L + k)) * ((T)1. + rdbrv1 * zq) - K(3 * L + k);
        SH(sv, k) = zv;
        SH(sb, k) = zv + gd;
        SH(s1, k) = tv1 - gt;
        if (k == 0) { zsumd = K(0) * gd; gvp = K(0) * zv; }
        else { zsumd = zsumd + K(k) * gd; gvp = gvp + K(k) * zv; }
    }
    const T tot = zsumd + gvp;
    // pass 2, level by level: sigma-dot, vertical advection terms and tendencies
    T psd = 0, psv = 0;                 // running sums of dsigma * gd and of dsigma * zvgpg
    T gtd_m = 0, gqm_m = 0, gud_m = 0, gvd_m = 0;   // the level above's products
    T zs = 0;                           // zsumd of the tendency loop (plasim.f90:2661, :2692)
    // the next level's fields are loaded one iteration ahead (n* = level k + 1)
    T nu = IN(0, 0), nv = IN(1, 0), nt = IN(2, 0), nd = IN(3, 0), nz = IN(4, 0), nq = IN(5, 0);
    for (int k = 0; k < L; k++) {
        const T gu = nu, gv = nv, gt = nt, gd = nd, gz = nz, gq = nq;
        if (k + 1 < L) {
            nu = IN(0, k + 1); nv = IN(1, k + 1); nt = IN(2, k + 1);
            nd = IN(3, k + 1); nz = IN(4, k + 1); nq = IN(5, k + 1);
        }
        const T zv = SH(sv, k);
        T zq;
        if (A.nqspec == 1) zq = fmax(gq / gp, (T)0.);
        else zq = A.dq ? fmax(A.dq[((size_t)inst * L + k) * n + h], (T)0.) : (T)0.;
        const T tv1 = (gt + K(3 * L + k)) * ((T)1. + rdbrv1 * zq) - K(3 * L + k);
        const T tv2 = (gt + K(3 * L + k)) * ((T)1. + rdbrv1 * zq) / ((T)1. + (T)A.adv * zq) - K(3 * L + k);
        // this level's products of the sigma-dot flux with the layer differences
        T gtd = 0, gqm = 0, gud = 0, gvd = 0;
        if (k < L - 1) {
            if (k == 0) { psd = K(0) * gd; psv = K(0) * zv; }
            else { psd = psd + K(k) * gd; psv = psv + K(k) * zv; }
            const T zsdotp = (K(L + k) * tot - (psd + psv));
            gtd = zsdotp * (nt - gt);
            gqm = zsdotp * (nq + gq);
            gud = zsdotp * (nu - gu);
            gvd = zsdotp * (nv - gv);
        }
        T gtn, gqn, guz, gvz, dwv;
        if (k == 0) {
            zs = zv * K(0);
            gtn = gt * gd - (T)A.akap * tv2 * gd - K(2 * L + 0) * (gtd + K(4 * L + 0) * (K(L + 0) * gvp - zs));
            gqn = -K(2 * L + 0) * gqm;
            guz = -gu * gz - gpj * tv1 - K(2 * L + 0) * gvd;
            gvz = gv * gz - gpm * tv1 - K(2 * L + 0) * gud;
            dwv = gd * gp * (T)A.psurf * (T)A.ww;
        } else {
            T ztpta = K(6 * L + L * L + 0 + L * k) * SH(sv, 0);
            T ztptb = K(6 * L + L * L + 0 + L * k) * SH(sb, 0);
#pragma unroll 4
            for (int j = 1; j <= k; j++) {
                ztpta = ztpta + K(6 * L + L * L + j + L * k) * SH(sv, j);
                ztptb = ztptb + K(6 * L + L * L + j + L * k) * SH(sb, j);
            }
            if (k < L - 1) {
                zs = zs + zv * K(k);
                gtn = gt * gd + (T)A.akap * tv2 * (zv - ztptb) + K(5 * L + k) * (zv - ztpta) -
                      K(2 * L + k) * (gtd + gtd_m + gvp * (K(4 * L + k) * K(L + k) + K(4 * L + k - 1) * K(L + k - 1)) -
                                     zs * (K(4 * L + k - 1) + K(4 * L + k)) + zv * K(k) * K(4 * L + k - 1));
                gqn = -K(2 * L + k) * (gqm - gqm_m);
                guz = -gu * gz - gpj * tv1 - K(2 * L + k) * (gvd + gvd_m);
                gvz = gv * gz - gpm * tv1 - K(2 * L + k) * (gud + gud_m);
            } else {
                gtn = gt * gd + (T)A.akap * tv2 * (zv - ztptb) + K(5 * L + k) * (zv - ztpta) -
                      K(2 * L + k) * (gtd_m + K(4 * L + k - 1) * (K(L + k - 1) * gvp - zs));
                gqn = K(2 * L + k) * gqm_m;
                guz = -gu * gz - gpj * tv1 - K(2 * L + k) * gvd_m;
                gvz = gv * gz - gpm * tv1 - K(2 * L + k) * gud_m;
            }
            dwv = (zv - ztptb) * gp * (T)A.psurf * (T)A.ww;
        }
        // non-linear geopotential, summed over every level as dot_product does;
        // initsi's g is lower triangular (g(i, k) = 0 for i < k), and those
        // exact zero terms leave the partial sum at +0, so they are skipped
        T dot = 0;
        if (A.g_lower) {
#pragma unroll 4
            for (int i = k; i < L; i++) dot = dot + K(6 * L + i + L * k) * SH(s1, i);
        } else {
#pragma unroll 4
            for (int i = 0; i < L; i++) dot = dot + K(6 * L + i + L * k) * SH(s1, i);
        }
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

// the launch: the constants in shared memory where they fit beside the profiles
template <typename T, bool SK, int LC>
inline exotx_status gp_launch_k(const GpArgs<T> &A, size_t smem, cudaStream_t s) {
    const long long nb = (A.ncol + GP_THREADS - 1) / GP_THREADS;
    if (smem > 48 * 1024)
        EXOTX_CUDA(cudaFuncSetAttribute(k_gridpoint<T, SK, LC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gridpoint<T, SK, LC><<<(unsigned)nb, GP_THREADS, smem, s>>>(A);
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}
template <typename T>
inline exotx_status gp_launch(const GpArgs<T> &A, cudaStream_t s) {
    const bool sk = gp_smem<T>(A.L, true) <= 227 * 1024;
    const size_t smem = gp_smem<T>(A.L, sk);
    if (!sk) return gp_launch_k<T, false, 0>(A, smem, s);
    switch (A.L) {   // the level counts of the standard configurations
        case 10: return gp_launch_k<T, true, 10>(A, smem, s);
        case 20: return gp_launch_k<T, true, 20>(A, smem, s);
        case 25: return gp_launch_k<T, true, 25>(A, smem, s);
        default: return gp_launch_k<T, true, 0>(A, smem, s);
    }
}

}  // namespace exotx
