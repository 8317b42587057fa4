// Folded SIMT Legendre transforms (FP64 parity path and FP32 path).
//
// Every spectral->Fourier operation of legmod.f90 is, per zonal wavenumber m,
//     F(lat, m) = sum_n c * T(m,n,lat) * X(m,n)      c in {1,-1,i,-i}
// and every Fourier->spectral operation is
//     X(m,n)    = sum_lat c * T(m,n,lat) * F(lat, m).
// The tables are exactly symmetric (P-type: qi,qc,qm,qq,qu) or antisymmetric
// (Q-type: qj,qe,qv) under lat -> -lat when n-m is even, and the reverse when
// n-m is odd, so both directions run over northern latitudes only:
//   inverse:  north = sym + anti, south = sym - anti
//   forward:  P-type terms see N+S for n-m even and N-S for odd; Q-type the reverse.
// The forward direction is the reference's own single-CPU branch
// (legmod.f90:191-220, :391-424, :466-497, :555-602); the inverse direction
// halves the work of the reference's unfolded loops (:240-254).
//
// Fourier-side addressing is general: complex element (field f, latitude l,
// wavenumber m) lives at base + f*fs + l*ls + m*ms (complex units), so the
// same kernels read and write both the reference layout fc(2,NLON/2,NLAT)
// and the m-major intermediate used inside the transform sets.
#include "exotx_internal.cuh"

namespace exotx {

template <typename T> struct C2 { T x, y; };
template <typename T> __device__ __forceinline__ C2<T> ld2(const T *p) { return C2<T>{p[0], p[1]}; }

template <typename T>
struct InvArgs {
    const T *tab;        // 4 inverse tables [t][w][j]
    const int *woff;
    const T *filt;       // skspgp(n)
    const T *a, *b;      // spectral inputs (re,im) pairs; field stride in reals
    long long a_fs, b_fs;
    T *oa, *ob;          // Fourier outputs
    long long fs, ls, ms;
    int nlev, nlat, nlath, ntp1, ncsp, mz;  // mz: m < mz are written (zeros for m > NTRU)
    T plavor;
};

// items: (j, level group of LT levels); one block per (m, level chunk)
template <typename T, int OP, int LT>
__global__ void __launch_bounds__(128) k_leg_inv(InvArgs<T> A, int lv) {
    extern __shared__ __align__(16) unsigned char smraw[];
    C2<T> *xa = reinterpret_cast<C2<T> *>(smraw);
    const int m = blockIdx.x;
    const int lev0 = blockIdx.y * lv;
    const int nl = min(lv, A.nlev - lev0);
    if (nl <= 0) return;
    const int nlat = A.nlat, nlath = A.nlath;
    if (m > A.ntp1 - 1) {  // zero tail of the Fourier row
        for (int idx = threadIdx.x; idx < nl * nlat; idx += blockDim.x) {
            int l = idx / nlat, lat = idx % nlat;
            size_t o = 2 * ((lev0 + l) * A.fs + lat * A.ls + (long long)m * A.ms);
            A.oa[o] = 0; A.oa[o + 1] = 0;
            if (OP == OP_DV2UV || OP == OP_SP2FC_GPMT) { A.ob[o] = 0; A.ob[o + 1] = 0; }
        }
        return;
    }
    const int K = A.ntp1 - m, w0 = A.woff[m];
    C2<T> *xb = xa + K * lv;
    // stage spectral coefficients (filtered) as [k][l]
    for (int idx = threadIdx.x; idx < K * nl; idx += blockDim.x) {
        int k = idx / nl, l = idx % nl;
        T f = A.filt[m + k];
        C2<T> va = ld2(A.a + (lev0 + l) * A.a_fs + 2 * (w0 + k));
        if (OP == OP_DV2UV) {
            // dv2uv: a = divergence, b = vorticity; plavor leaves mode (0,1) (legmod.f90:332)
            C2<T> vb = ld2(A.b + (lev0 + l) * A.b_fs + 2 * (w0 + k));
            if (m == 0 && k == 1) vb.x -= A.plavor;
            xb[k * lv + l] = C2<T>{vb.x * f, vb.y * f};
        }
        xa[k * lv + l] = C2<T>{va.x * f, va.y * f};
    }
    __syncthreads();
    const int ngroups = (nl + LT - 1) / LT;
    const T *tabP;
    if (OP == OP_SP2FCDMU) tabP = A.tab + (size_t)INV_QJ * A.ncsp * nlath;
    else tabP = A.tab + (size_t)INV_QI * A.ncsp * nlath;
    const T *tabU = A.tab + (size_t)INV_QU * A.ncsp * nlath;
    const T *tabV = A.tab + (size_t)INV_QV * A.ncsp * nlath;
    for (int item = threadIdx.x; item < nlath * ngroups; item += blockDim.x) {
        const int j = item % nlath, g = item / nlath;
        const int l0 = g * LT;
        C2<T> s1[LT], a1[LT], s2[LT], a2[LT];
#pragma unroll
        for (int q = 0; q < LT; q++) s1[q] = a1[q] = s2[q] = a2[q] = C2<T>{0, 0};
        for (int k = 0; k < K; k++) {
            const bool even = !(k & 1);
            if (OP == OP_DV2UV) {
                // u = sum qv*Z - i*qu*D ; v = sum -i*qu*Z - qv*D  (legmod.f90:338-341)
                T tu = tabU[(size_t)(w0 + k) * nlath + j];
                T tv = tabV[(size_t)(w0 + k) * nlath + j];
#pragma unroll
                for (int q = 0; q < LT; q++) {
                    if (l0 + q >= nl) break;
                    C2<T> D = xa[k * lv + l0 + q], Z = xb[k * lv + l0 + q];
                    // P-type (qu) terms
                    C2<T> uP{tu * D.y, -tu * D.x};      // -i*qu*D
                    C2<T> vP{tu * Z.y, -tu * Z.x};      // -i*qu*Z
                    // Q-type (qv) terms
                    C2<T> uQ{tv * Z.x, tv * Z.y};
                    C2<T> vQ{-tv * D.x, -tv * D.y};
                    if (even) {
                        s1[q].x += uP.x; s1[q].y += uP.y; a1[q].x += uQ.x; a1[q].y += uQ.y;
                        s2[q].x += vP.x; s2[q].y += vP.y; a2[q].x += vQ.x; a2[q].y += vQ.y;
                    } else {
                        a1[q].x += uP.x; a1[q].y += uP.y; s1[q].x += uQ.x; s1[q].y += uQ.y;
                        a2[q].x += vP.x; a2[q].y += vP.y; s2[q].x += vQ.x; s2[q].y += vQ.y;
                    }
                }
            } else {
                T t = tabP[(size_t)(w0 + k) * nlath + j];
                // qi is P-type (sym on even n-m); qj is Q-type (sym on odd n-m)
                const bool sym = (OP == OP_SP2FCDMU) ? !even : even;
#pragma unroll
                for (int q = 0; q < LT; q++) {
                    if (l0 + q >= nl) break;
                    C2<T> X = xa[k * lv + l0 + q];
                    if (sym) { s1[q].x += t * X.x; s1[q].y += t * X.y; }
                    else     { a1[q].x += t * X.x; a1[q].y += t * X.y; }
                }
            }
        }
        const int latN = j, latS = nlat - 1 - j;
#pragma unroll
        for (int q = 0; q < LT; q++) {
            if (l0 + q >= nl) break;
            const long long f = lev0 + l0 + q;
            size_t oN = 2 * (f * A.fs + latN * A.ls + (long long)m * A.ms);
            size_t oS = 2 * (f * A.fs + latS * A.ls + (long long)m * A.ms);
            C2<T> n1{s1[q].x + a1[q].x, s1[q].y + a1[q].y}, d1{s1[q].x - a1[q].x, s1[q].y - a1[q].y};
            A.oa[oN] = n1.x; A.oa[oN + 1] = n1.y;
            A.oa[oS] = d1.x; A.oa[oS + 1] = d1.y;
            if (OP == OP_DV2UV) {
                C2<T> n2{s2[q].x + a2[q].x, s2[q].y + a2[q].y}, d2{s2[q].x - a2[q].x, s2[q].y - a2[q].y};
                A.ob[oN] = n2.x; A.ob[oN + 1] = n2.y;
                A.ob[oS] = d2.x; A.ob[oS + 1] = d2.y;
            }
            if (OP == OP_SP2FC_GPMT) {
                // gpmt = i*m*gp  (plasim.f90:2425-2430)
                T mm = (T)m;
                A.ob[oN] = -n1.y * mm; A.ob[oN + 1] = n1.x * mm;
                A.ob[oS] = -d1.y * mm; A.ob[oS + 1] = d1.x * mm;
            }
        }
    }
}

template <typename T>
struct FwdArgs {
    const T *tab;        // 4 forward tables, per-m blocks [t][woff*nlath + j*K + k]
    const int *woff;
    const T *filt;       // skgpsp(n)
    const T *in[6];
    long long fs, ls, ms;  // Fourier addressing of the inputs
    T *out[3];
    long long o_fs;        // spectral field stride (reals)
    int nlev, nlat, nlath, ntp1, ncsp;
};

template <int OP> struct FwdNin { static constexpr int v = 1; };
template <> struct FwdNin<OP_UV2DV> { static constexpr int v = 2; };
template <> struct FwdNin<OP_QTEND> { static constexpr int v = 3; };
template <> struct FwdNin<OP_MKTEND> { static constexpr int v = 6; };

// one block per (m, level chunk); items (k, level)
template <typename T, int OP>
__global__ void __launch_bounds__(128) k_leg_fwd(FwdArgs<T> A, int lv) {
    extern __shared__ __align__(16) unsigned char smraw[];
    constexpr int NIN = FwdNin<OP>::v;
    const int m = blockIdx.x;
    const int lev0 = blockIdx.y * lv;
    const int nl = min(lv, A.nlev - lev0);
    if (nl <= 0) return;
    const int nlath = A.nlath, nlat = A.nlat;
    const int K = A.ntp1 - m, w0 = A.woff[m];
    // staged sums and differences: sd[((i*lv + l)*nlath + j)*2 + {0:sum,1:diff}]
    C2<T> *sd = reinterpret_cast<C2<T> *>(smraw);
    for (int idx = threadIdx.x; idx < NIN * nl * nlath; idx += blockDim.x) {
        int j = idx % nlath, r = idx / nlath, l = r % nl, i = r / nl;
        const long long f = lev0 + l;
        C2<T> vn = ld2(A.in[i] + 2 * (f * A.fs + j * A.ls + (long long)m * A.ms));
        C2<T> vs = ld2(A.in[i] + 2 * (f * A.fs + (nlat - 1 - j) * A.ls + (long long)m * A.ms));
        C2<T> *dst = sd + ((size_t)(i * lv + l) * nlath + j) * 2;
        dst[0] = C2<T>{vn.x + vs.x, vn.y + vs.y};
        dst[1] = C2<T>{vn.x - vs.x, vn.y - vs.y};
    }
    __syncthreads();
    const size_t tsz = (size_t)A.ncsp * nlath;
    const T *qc = A.tab + FWD_QC * tsz + (size_t)w0 * nlath;
    const T *qe = A.tab + FWD_QE * tsz + (size_t)w0 * nlath;
    const T *qm = A.tab + FWD_QM * tsz + (size_t)w0 * nlath;
    const T *qq = A.tab + FWD_QQ * tsz + (size_t)w0 * nlath;
    for (int item = threadIdx.x; item < K * nl; item += blockDim.x) {
        const int k = item % K, l = item / K;
        const bool even = !(k & 1);
        const int P = even ? 0 : 1, Q = even ? 1 : 0;   // sum/diff selectors
        auto F = [&](int i, int j, int sel) -> C2<T> {
            return sd[((size_t)(i * lv + l) * nlath + j) * 2 + sel];
        };
        C2<T> o0{0, 0}, o1{0, 0}, o2{0, 0};
        for (int j = 0; j < nlath; j++) {
            const size_t ti = (size_t)j * K + k;
            if (OP == OP_FC2SP) {
                // sp = sum qc*(N +- S)  (legmod.f90:203-220)
                T c = qc[ti];
                C2<T> x = F(0, j, P);
                o0.x += c * x.x; o0.y += c * x.y;
            } else if (OP == OP_UV2DV) {
                // pz = sum qe*u(Q) + i*qm*v(P); pd = sum -qe*v(Q) + i*qm*u(P)  (legmod.f90:391-424)
                T e = qe[ti], mm = qm[ti];
                C2<T> uQ = F(0, j, Q), vP = F(1, j, P), vQ = F(1, j, Q), uP = F(0, j, P);
                o1.x += e * uQ.x - mm * vP.y; o1.y += e * uQ.y + mm * vP.x;      // vorticity
                o0.x += -e * vQ.x - mm * uP.y; o0.y += -e * vQ.y + mm * uP.x;    // divergence
            } else if (OP == OP_QTEND) {
                // q = sum qe*vq(Q) + qc*qn(P) - i*qm*uq(P)  (legmod.f90:466-497); in = qn,uq,vq
                T e = qe[ti], c = qc[ti], mm = qm[ti];
                C2<T> qn = F(0, j, P), uq = F(1, j, P), vq = F(2, j, Q);
                o0.x += e * vq.x + c * qn.x + mm * uq.y;
                o0.y += e * vq.y + c * qn.y - mm * uq.x;
            } else {  // OP_MKTEND, in = tn,fu,fv,ke,ut,vt (legmod.f90:555-602)
                T e = qe[ti], c = qc[ti], mm = qm[ti], qv = qq[ti];
                C2<T> tn = F(0, j, P), fuP = F(1, j, P), fuQ = F(1, j, Q), fvP = F(2, j, P),
                      fvQ = F(2, j, Q), ke = F(3, j, P), ut = F(4, j, P), vt = F(5, j, Q);
                // d = qq*ke - qe*fv + i*qm*fu
                o0.x += qv * ke.x - e * fvQ.x - mm * fuP.y;
                o0.y += qv * ke.y - e * fvQ.y + mm * fuP.x;
                // t = qe*vt + qc*tn - i*qm*ut
                o1.x += e * vt.x + c * tn.x + mm * ut.y;
                o1.y += e * vt.y + c * tn.y - mm * ut.x;
                // z = qe*fu + i*qm*fv
                o2.x += e * fuQ.x - mm * fvP.y;
                o2.y += e * fuQ.y + mm * fvP.x;
            }
        }
        const T f = A.filt[m + k];
        const long long fld = lev0 + l;
        const size_t o = (size_t)fld * A.o_fs + 2 * (w0 + k);
        A.out[0][o] = o0.x * f; A.out[0][o + 1] = o0.y * f;
        if (OP == OP_UV2DV || OP == OP_MKTEND) { A.out[1][o] = o1.x * f; A.out[1][o + 1] = o1.y * f; }
        if (OP == OP_MKTEND) { A.out[2][o] = o2.x * f; A.out[2][o + 1] = o2.y * f; }
    }
}

static int pick_lv(size_t per_level_bytes, int nlev, size_t budget = 40 * 1024) {
    int lv = (int)(budget / (per_level_bytes ? per_level_bytes : 1));
    lv = lv < 1 ? 1 : lv;
    lv = lv > 16 ? 16 : lv;
    return lv > nlev ? nlev : lv;
}

template <typename T> static const T *inv_tab(exotx_plan p);
template <> const double *inv_tab<double>(exotx_plan p) { return p->d_inv64; }
template <> const float *inv_tab<float>(exotx_plan p) { return p->d_inv32; }
template <typename T> static const T *fwd_tab(exotx_plan p);
template <> const double *fwd_tab<double>(exotx_plan p) { return p->d_fwd64; }
template <> const float *fwd_tab<float>(exotx_plan p) { return p->d_fwd32; }
template <typename T> static const T *filt_s(exotx_plan p);
template <> const double *filt_s<double>(exotx_plan p) { return p->d_fs64; }
template <> const float *filt_s<float>(exotx_plan p) { return p->d_fs32; }
template <typename T> static const T *filt_g(exotx_plan p);
template <> const double *filt_g<double>(exotx_plan p) { return p->d_fg64; }
template <> const float *filt_g<float>(exotx_plan p) { return p->d_fg32; }

template <typename T>
exotx_status leg_inverse_l(exotx_plan p, int op, const T *a, const T *b, T *oa, T *ob, int nlev,
                           long long a_fs, long long b_fs, FourierLayout L, cudaStream_t s) {
    if (nlev <= 0) return EXOTX_OK;
    InvArgs<T> A;
    A.tab = inv_tab<T>(p); A.woff = p->d_woff; A.filt = filt_s<T>(p);
    A.a = a; A.b = b; A.a_fs = a_fs; A.b_fs = b_fs;
    A.oa = oa; A.ob = ob; A.fs = L.fs; A.ls = L.ls; A.ms = L.ms;
    A.nlev = nlev; A.nlat = p->nlat; A.nlath = p->nlath; A.ntp1 = p->ntp1; A.ncsp = p->ncsp;
    A.mz = L.mz; A.plavor = (T)p->desc.plavor;
    int nin = (op == OP_DV2UV) ? 2 : 1;
    size_t per_level = (size_t)nin * p->ntp1 * sizeof(T) * 2;
    int lv = pick_lv(per_level, nlev);
    size_t smem = per_level * lv;
    dim3 grid(L.mz, (nlev + lv - 1) / lv);
    constexpr int LT = 4;
    cudaEvent_t ev = ktimer_start(EXOTX_K_LEG_INVERSE, s);
    switch (op) {
        case OP_SP2FC: k_leg_inv<T, OP_SP2FC, LT><<<grid, 128, smem, s>>>(A, lv); break;
        case OP_SP2FCDMU: k_leg_inv<T, OP_SP2FCDMU, LT><<<grid, 128, smem, s>>>(A, lv); break;
        case OP_DV2UV: k_leg_inv<T, OP_DV2UV, LT><<<grid, 128, smem, s>>>(A, lv); break;
        case OP_SP2FC_GPMT: k_leg_inv<T, OP_SP2FC_GPMT, LT><<<grid, 128, smem, s>>>(A, lv); break;
        default: return EXOTX_BAD_ARG;
    }
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_LEG_INVERSE, s, ev);
    return EXOTX_OK;
}

template <typename T>
exotx_status leg_forward_l(exotx_plan p, int op, const T *const *in, T *const *out, int nlev,
                           FourierLayout L, long long o_fs, cudaStream_t s) {
    if (nlev <= 0) return EXOTX_OK;
    FwdArgs<T> A;
    A.tab = fwd_tab<T>(p); A.woff = p->d_woff; A.filt = filt_g<T>(p);
    int nin = op == OP_FC2SP ? 1 : op == OP_UV2DV ? 2 : op == OP_QTEND ? 3 : 6;
    int nout = op == OP_MKTEND ? 3 : op == OP_UV2DV ? 2 : 1;
    for (int i = 0; i < 6; i++) A.in[i] = i < nin ? in[i] : nullptr;
    for (int i = 0; i < 3; i++) A.out[i] = i < nout ? out[i] : nullptr;
    A.fs = L.fs; A.ls = L.ls; A.ms = L.ms; A.o_fs = o_fs;
    A.nlev = nlev; A.nlat = p->nlat; A.nlath = p->nlath; A.ntp1 = p->ntp1; A.ncsp = p->ncsp;
    size_t per_level = (size_t)nin * p->nlath * 2 * 2 * sizeof(T);
    int lv = pick_lv(per_level, nlev);
    size_t smem = per_level * lv;
    if (smem > 48 * 1024) return EXOTX_BAD_DIM;
    dim3 grid(p->ntp1, (nlev + lv - 1) / lv);
    cudaEvent_t ev = ktimer_start(EXOTX_K_LEG_FORWARD, s);
    switch (op) {
        case OP_FC2SP: k_leg_fwd<T, OP_FC2SP><<<grid, 128, smem, s>>>(A, lv); break;
        case OP_UV2DV: k_leg_fwd<T, OP_UV2DV><<<grid, 128, smem, s>>>(A, lv); break;
        case OP_QTEND: k_leg_fwd<T, OP_QTEND><<<grid, 128, smem, s>>>(A, lv); break;
        case OP_MKTEND: k_leg_fwd<T, OP_MKTEND><<<grid, 128, smem, s>>>(A, lv); break;
        default: return EXOTX_BAD_ARG;
    }
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_LEG_FORWARD, s, ev);
    return EXOTX_OK;
}

template exotx_status leg_inverse_l<double>(exotx_plan, int, const double *, const double *, double *, double *,
                                            int, long long, long long, FourierLayout, cudaStream_t);
template exotx_status leg_inverse_l<float>(exotx_plan, int, const float *, const float *, float *, float *, int,
                                           long long, long long, FourierLayout, cudaStream_t);
template exotx_status leg_forward_l<double>(exotx_plan, int, const double *const *, double *const *, int,
                                            FourierLayout, long long, cudaStream_t);
template exotx_status leg_forward_l<float>(exotx_plan, int, const float *const *, float *const *, int,
                                           FourierLayout, long long, cudaStream_t);

}  // namespace exotx
