// radmod.f90 radiation column pass on the GPU: one warp per column (device code).
//
// The reference evaluates radstep (:927-1110) with array statements over all
// NHOR columns.  Here a warp owns a column; its 32 lanes share the
// transcendental work (per-level cloud optics, ozone/water-vapour
// transmissivities, and the O(NLEV^2) longwave absorptivities of lwr, which
// are spread over all lanes as a flat list of (jlev, jlev2) pairs), while
// the adding-method recurrences of swr and the running sums/products of lwr
// keep the reference's summation order on one lane.  Columns are read and
// written in the reference layout x(NHOR,NLEV).
#pragma once
#include <cmath>
#include "exotx_internal.cuh"

namespace exotx {

constexpr int RAD_MAXLEV = 64;
constexpr int RAD_WARPS = 4;

struct RadDev {
    exotx_rad_params p;
    const void *sid, *cola, *dt, *dq, *dcc, *dql, *dqco2, *dp, *dls, *dicec;
    void *dqo3, *gmu0, *dalb, *dsalb;
    void *dfu, *dfd, *dftu, *dftd, *dswfl, *dlwfl, *dflux, *dtdt, *dtdtswr, *dtdtlwr, *dconv;
    const void *zsol;       // optional (NHOR,3): per-column zsolar1, zsolar2, rcoeff
    const int *cols;        // optional list of the columns to compute ...
    const int *ncols;       // ... and its length (device memory)
};

template <typename T> __device__ __forceinline__ T P_(T x, T y);
template <> __device__ __forceinline__ double P_(double x, double y) { return pow(x, y); }
template <> __device__ __forceinline__ float P_(float x, float y) { return powf(x, y); }

// ozone and water-vapour broadband absorption fits (radmod.f90:1907-1913, :1992-1993)
template <typename T> __device__ T ao3_(T x) {
    return (T)0.02118 * x / ((T)1 + (T)0.042 * x + (T)0.000323 * (x * x)) +
           (T)1.082 * x / P_((T)1 + (T)138.6 * x, (T)0.805) +
           (T)0.0658 * x / ((T)1 + ((T)103.6 * x) * ((T)103.6 * x) * ((T)103.6 * x));
}
template <typename T> __device__ T awv_(T x) {
    return (T)2.9 * x / (P_((T)1 + (T)141.5 * x, (T)0.635) + (T)5.925 * x);
}

// shared scratch per warp (sizes for nlev levels)
template <typename T> struct ColScratch {
    T *dt, *dq, *dcc, *dql, *o3, *co2;              // inputs
    T *rcl1, *rcl2, *rcl1s, *rcl2s, *tcl2, *tcl2s, *csabove;
    T *o3l, *xo3l, *wvl, *ywvl, *ao3d, *ao3u, *awvd, *awvu, *zwv, *zo3;
    T *tb1, *tb1u, *tb2, *tb2u, *rb1, *rb1s, *rb2, *rb2s;
    T *t1, *t2, *r1s, *r2s, *rl1, *rl2, *rl1s, *rl2s;
    T *st4, *st4h, *q, *qo3, *qco2, *taucc0, *bu, *bd, *tau, *row1;
    T *fu, *fd, *sw, *ftu, *ftd, *lw;
    T *sc;  // scalars
};
template <typename T> __device__ size_t scratch_elems(int L) {
    int E = L + 1;
    return (size_t)6 * E + 7 * L + 11 * L + 8 * L + 8 * E + 2 * E + 4 * L + 2 * (E + 1) + (size_t)L * L + L +
           6 * E + 32;
}
template <typename T> __device__ ColScratch<T> carve(T *b, int L) {
    int E = L + 1;
    ColScratch<T> s;
    T *p = b;
    auto take = [&](int n) { T *r = p; p += n; return r; };
    s.dt = take(E); s.dq = take(E); s.dcc = take(E); s.dql = take(E); s.o3 = take(E); s.co2 = take(E);
    s.rcl1 = take(L); s.rcl2 = take(L); s.rcl1s = take(L); s.rcl2s = take(L); s.tcl2 = take(L); s.tcl2s = take(L);
    s.csabove = take(L);
    s.o3l = take(L); s.xo3l = take(L); s.wvl = take(L); s.ywvl = take(L); s.ao3d = take(L); s.ao3u = take(L);
    s.awvd = take(L); s.awvu = take(L); s.zwv = take(L); s.zo3 = take(L); take(L);
    s.tb1 = take(L); s.tb1u = take(L); s.tb2 = take(L); s.tb2u = take(L); s.rb1 = take(L); s.rb1s = take(L);
    s.rb2 = take(L); s.rb2s = take(L);
    s.t1 = take(E); s.t2 = take(E); s.r1s = take(E); s.r2s = take(E); s.rl1 = take(E); s.rl2 = take(E);
    s.rl1s = take(E); s.rl2s = take(E);
    s.st4 = take(E); s.st4h = take(E);
    s.q = take(L); s.qo3 = take(L); s.qco2 = take(L); s.taucc0 = take(L);
    s.bu = take(E + 1); s.bd = take(E + 1);
    s.tau = take(L * L); s.row1 = take(L);
    s.fu = take(E); s.fd = take(E); s.sw = take(E); s.ftu = take(E); s.ftd = take(E); s.lw = take(E);
    s.sc = take(32);
    return s;
}

template <typename T>
__device__ void swr_warp(const exotx_rad_params &P, ColScratch<T> &s, int L, T zmu0, T zmu1, T dp, T &dalb,
                         T *dsalb, T dls, T dicec, T csol1, T csol2, T crco, int lane) {
    const T zero = (T)1e-6, zbetta = (T)1.66, zmbar = (T)1.9, zro3 = (T)2.14, zfo3 = (T)100. / zro3;
    const T aa = (T)0.2542857142857143, bb = (T)0.8229693877551021, c0 = (T)0.14997959183673468;
    const T ga = (T)P.ga;
    const int E = L + 1;
    const int nclouds = P.nclouds;
    for (int k = lane; k < E; k += 32) { s.fu[k] = 0; s.fd[k] = 0; s.sw[k] = 0; }
    T zftop1 = csol1 * (T)P.gsol0 * (T)P.gdist2 * zmu1;
    T zftop2 = csol2 * (T)P.gsol0 * (T)P.gdist2 * zmu1;
    bool losun = (zftop1 + zftop2 > zero);
    const T zmu00 = (T)0.5;
    if (!losun) { __syncwarp(); return; }
    // clear-sky fraction above each level (cloud block, :1681-1768): serial product
    if (lane == 0) {
        T zcs = 1;
        for (int jl = 0; jl < L; jl++) { s.csabove[jl] = zcs; zcs = zcs * ((T)1 - s.dcc[jl]); }
    }
    __syncwarp();
    T zb3 = (T)P.tswr1 * sqrt(zmu00) / zmu00;
    T zb4 = (T)P.tswr2 * sqrt(zmu00);
    T zb5 = (T)P.tswr3 * zmu00 * zmu00;
    for (int jl = lane; jl < L; jl += 32) {
        T dcc = s.dcc[jl], zcs = s.csabove[jl];
        T rcl1 = 0, rcl2 = 0, tcl2 = 1, rcl1s = 0, rcl2s = 0, tcl2s = 1;
        if (nclouds == 1) {
            if (P.nswrcl == 0) {
                T sg = (T)P.sigma[jl];
                int r = (sg <= (T)(1. / 3.)) ? 0 : ((sg > (T)(1. / 3.) && sg <= (T)(2. / 3.)) ? 1 : 2);
                T c1 = (T)P.rcl1[r], c2 = (T)P.rcl2[r], a2 = (T)P.acl2[r];
                rcl1s = c1 / (c1 + zmu00);
                rcl1 = zcs * c1 / (c1 + zmu0) + ((T)1 - zcs) * rcl1s;
                rcl2s = fmin((T)1 - a2, c2 / (c2 + zmu00));
                rcl2 = fmin((T)1 - a2, zcs * c2 / (c2 + zmu0) + ((T)1 - zcs) * rcl2s);
                tcl2s = (T)1 - rcl2s - a2;
                tcl2 = (T)1 - rcl2 - a2;
            } else if (dcc > (T)0) {
                T zlwp = fmin((T)1000.0, (T)1000. * s.dql[jl] * dp / ga * (T)P.dsigma[jl]);
                T ztau = (T)2.0 * P_(log10(zlwp + (T)1.5), (T)3.9);
                T zlog = log((T)1000.0 / ztau);
                T zb2 = zb4 / log((T)3. + (T)0.1 * ztau);
                T zom0 = fmin((T)0.9999, (T)1.0 - zb5 * zlog);
                T zun = (T)1.0 - zom0;
                T zuz = zun + (T)2.0 * zb2 * zom0;
                T zu = sqrt(zuz / zun);
                T zexp = exp(fmin((T)25.0, ztau * sqrt(zuz * zun) / zmu00));
                T zr = (zu + (T)1.) * (zu + (T)1.) * zexp - (zu - (T)1.) * (zu - (T)1.) / zexp;
                rcl1s = (T)1. - (T)1. / ((T)1. + zb3 * ztau);
                tcl2s = (T)4. * zu / zr;
                rcl2s = (zu * zu - (T)1.) / zr * (zexp - (T)1. / zexp);
                T zb1 = (T)P.tswr1 * sqrt(zmu0);
                zb2 = (T)P.tswr2 * sqrt(zmu0) / log((T)3. + (T)0.1 * ztau);
                zom0 = fmin((T)0.9999, (T)1. - (T)P.tswr3 * zmu0 * zmu0 * zlog);
                zun = (T)1.0 - zom0;
                zuz = zun + (T)2.0 * zb2 * zom0;
                zu = sqrt(zuz / zun);
                zexp = exp(fmin((T)25.0, ztau * sqrt(zuz * zun) / zmu0));
                zr = (zu + (T)1.) * (zu + (T)1.) * zexp - (zu - (T)1.) * (zu - (T)1.) / zexp;
                rcl1 = (T)1. - (T)1. / ((T)1. + zb1 * ztau / zmu0);
                tcl2 = (T)4. * zu / zr;
                rcl2 = (zu * zu - (T)1.) / zr * (zexp - (T)1. / zexp);
                rcl1 = zcs * rcl1 + ((T)1. - zcs) * rcl1s;
                tcl2 = zcs * tcl2 + ((T)1. - zcs) * tcl2s;
                rcl2 = zcs * rcl2 + ((T)1. - zcs) * rcl2s;
            }
        }
        s.rcl1[jl] = rcl1; s.rcl2[jl] = rcl2; s.tcl2[jl] = tcl2;
        s.rcl1s[jl] = rcl1s; s.rcl2s[jl] = rcl2s; s.tcl2s[jl] = tcl2s;
        // absorber amounts of this layer (:1785-1789)
        s.zo3[jl] = zfo3 * (T)P.dsigma[jl] * dp * s.o3[jl] / ga;
        s.zwv[jl] = (T)0.1 * (T)P.dsigma[jl] * s.dq[jl] * dp / ga * sqrt((T)273. / s.dt[jl]) * (T)P.sigma[jl] *
                    dp / (T)100000.;
    }
    __syncwarp();
    // accumulated absorber paths with the clear-sky mixing (:1779-1802): serial
    T zm = (T)35. / sqrt((T)1. + (T)1224. * zmu0 * zmu0);
    if (lane == 0) {
        T zcs = 1, zo3t = 0, zxo3t = 0, zwvt = 0, zywvt = 0;
        for (int jl = 0; jl < L; jl++) {
            T zo3 = s.zo3[jl];
            zo3t = zo3t + zo3;
            zxo3t = zcs * (zxo3t + zm * zo3) + ((T)1. - zcs) * (zxo3t + zmbar * zo3);
            s.o3l[jl] = zo3t;
            s.xo3l[jl] = zxo3t;
            T zwv = s.zwv[jl];
            zwvt = zwvt + zwv;
            zywvt = zcs * (zywvt + zm * zwv) + ((T)1. - zcs) * (zywvt + zbetta * zwv);
            s.wvl[jl] = zwvt;
            s.ywvl[jl] = zywvt;
            zcs = zcs * ((T)1. - s.dcc[jl] * nclouds);
        }
        s.sc[0] = zcs; s.sc[1] = zo3t; s.sc[2] = zxo3t; s.sc[3] = zwvt; s.sc[4] = zywvt;
    }
    __syncwarp();
    const T zcsf = s.sc[0], zo3t = s.sc[1], zxo3t = s.sc[2], zwvt = s.sc[3], zywvt = s.sc[4];
    // transmissivity fits per level, lane-parallel
    for (int jl = lane; jl < L; jl += 32) {
        s.ao3d[jl] = ao3_<T>(s.xo3l[jl]);
        s.ao3u[jl] = ao3_<T>(zxo3t + zmbar * (zo3t - s.o3l[jl]));
        s.awvd[jl] = awv_<T>(s.ywvl[jl]);
        s.awvu[jl] = awv_<T>(zywvt + zbetta * (zwvt - s.wvl[jl]));
    }
    __syncwarp();
    if (lane == 0) {
        const int newrsc = P.newrsc, nrscat = P.nrscat;
        const T zs1 = csol1, zs2 = csol2;
        const T dccL = s.dcc[L - 1];
        T zta1 = 1, zta1s = 1, zra1 = 0, zra1s = 0, zta2 = 1, zta2s = 1, zra2 = 0, zra2s = 0;
        T zto3t = 1;
        T zto3tu = (T)1. - ao3_<T>(zxo3t + zmbar * zo3t) / zs1;
        T ztwvt = 1;
        T ztwvtu = (T)1. - awv_<T>(zywvt + zbetta * zwvt) / zs2;
        // Rayleigh scattering in the lowest layer only (newrsc = 0 default, :1928-1939)
        T zcs_run = 1;
        T zscf = crco * dp / (T)101100.0 * (T)9.80665 / ga;
        for (int jl = 0; jl < L; jl++) {
            zcs_run = zcs_run * ((T)1. - s.dcc[jl] * nclouds);
            T zrcs = (aa / ((T)1. + bb * zmu0) * zcs_run + c0 * ((T)1. - zcs_run - dccL * nclouds)) *
                     (T)P.dsigma[jl] * (dp / (T)101100.0) * ((T)9.80665 / ga) * nrscat * newrsc;
            T zrcsu = c0 * ((T)1. - dccL) * (T)P.dsigma[jl] * (dp / (T)101100.0) * ((T)9.80665 / ga) * nrscat *
                      newrsc;
            if (jl == L - 1) {
                zrcs = zrcs * newrsc;
                zrcsu = zrcsu * newrsc;
                zrcsu = zrcsu + ((T)1.0 - exp(zscf * log((T)1.0 - (T)0.144))) * (1 - newrsc) * nrscat *
                                    ((T)1 - dccL * nclouds);
                zrcs = zrcs + ((T)1.0 - exp(zscf * log((T)1.0 - ((T)0.219 / ((T)1. + (T)0.816 * zmu0))))) * zcsf *
                                  (1 - newrsc) * nrscat +
                       ((T)1.0 - exp(zscf * log((T)1.0 - (T)0.144))) * ((T)1. - zcsf - dccL) * nrscat *
                           (1 - newrsc);
            }
            T dcc = s.dcc[jl];
            s.t1[jl] = zta1; s.t2[jl] = zta2; s.r1s[jl] = zra1s; s.r2s[jl] = zra2s;
            T rb1 = zrcs + s.rcl1[jl] * dcc * nclouds;
            T rb1s = zrcsu + s.rcl1s[jl] * dcc * nclouds;
            T zto3 = ((T)1. - s.ao3d[jl] / zs1) / zto3t;
            zto3t = zto3t * zto3;
            T zto3u = zto3tu / ((T)1. - s.ao3u[jl] / zs1);
            zto3tu = zto3tu / zto3u;
            T tb1 = (T)1. - ((T)1. - zto3) * ((T)1. - dcc) - rb1;
            T tb1u = (T)1. - ((T)1. - zto3u) * ((T)1. - dcc) - rb1s;
            T z1mrabr = (T)1. / ((T)1. - zra1s * rb1s);
            zra1 = zra1 + zta1 * rb1 * zta1s * z1mrabr;
            zta1 = zta1 * tb1 * z1mrabr;
            zra1s = rb1s + tb1u * zra1s * tb1 * z1mrabr;
            zta1s = tb1u * zta1s * z1mrabr;
            T rb2 = s.rcl2[jl] * dcc * nclouds;
            T rb2s = s.rcl2s[jl] * dcc * nclouds;
            T ztwv = ((T)1. - s.awvd[jl] / zs2) / ztwvt;
            ztwvt = ztwvt * ztwv;
            T ztwvu = ztwvtu / ((T)1. - s.awvu[jl] / zs2);
            ztwvtu = ztwvtu / ztwvu;
            T tb2 = (T)1. - ((T)1. - ztwv) * ((T)1. - dcc * nclouds) - ((T)1. - s.tcl2[jl]) * dcc * nclouds;
            T tb2u = (T)1. - ((T)1. - ztwvu) * ((T)1. - dcc * nclouds) - ((T)1. - s.tcl2s[jl]) * dcc * nclouds;
            z1mrabr = (T)1. / ((T)1. - zra2s * rb2s);
            zra2 = zra2 + zta2 * rb2 * zta2s * z1mrabr;
            zta2 = zta2 * tb2 * z1mrabr;
            zra2s = rb2s + tb2u * zra2s * tb2 * z1mrabr;
            zta2s = tb2u * zta2s * z1mrabr;
            s.rb1[jl] = rb1; s.rb1s[jl] = rb1s; s.tb1[jl] = tb1; s.tb1u[jl] = tb1u;
            s.rb2[jl] = rb2; s.rb2s[jl] = rb2s; s.tb2[jl] = tb2; s.tb2u[jl] = tb2u;
        }
        s.t1[L] = zta1; s.t2[L] = zta2; s.r1s[L] = zra1s; s.r2s[L] = zra2s;
        // surface albedo for the direct beam (:2046-2071)
        const int nst = P.nstartemp, ne = P.necham, ne6 = P.necham6;
        zra1s = dalb * (1 - nst) + dsalb[0] * nst;
        zra2s = dalb * (1 - nst) + dsalb[1] * nst;
        T ocean3 = fmin((T)0.05 / (zmu0 + (T)0.15), (T)0.15);
        T ocean6 = ((T)0.026 / (P_(zmu0, (T)1.7) + (T)0.065) +
                    (T)0.15 * (zmu0 - (T)1) * (zmu0 - (T)0.5) * (zmu0 - (T)0.1) + (T)0.0082);
        for (int b = 0; b < 2; b++) {
            dsalb[b] = dls * dsalb[b] + ((T)1. - dls) * dicec * dsalb[b] +
                       ((T)1. - dls) * ((T)1. - dicec) * ocean3 * ne * (1 - ne6) +
                       ((T)1. - dls) * ((T)1. - dicec) * (1 - ne) * ne6 * ocean6 +
                       ((T)1. - dls) * ((T)1. - dicec) * ((T)1. - ne) * (1 - ne6) * dsalb[b];
        }
        dalb = (csol1 * dsalb[0] + csol2 * dsalb[1]) * nst +
               (dls * dalb + ((T)1. - dls) * dicec * dalb + ((T)1. - dls) * ((T)1. - dicec) * ocean3 * ne * (1 - ne6) +
                ((T)1. - dls) * ((T)1. - dicec) * (1 - ne) * ne6 * ocean6 +
                ((T)1. - dls) * ((T)1. - dicec) * ((T)1. - ne) * (1 - ne6) * dalb) *
                   (1 - nst);
        zra1 = dsalb[0] * nst + dalb * (1 - nst);
        zra2 = dsalb[1] * nst + dalb * (1 - nst);
        for (int jl = L - 1; jl >= 0; jl--) {
            s.rl1[jl + 1] = zra1; s.rl2[jl + 1] = zra2; s.rl1s[jl + 1] = zra1s; s.rl2s[jl + 1] = zra2s;
            zra1 = s.rb1[jl] + s.tb1[jl] * zra1 * s.tb1u[jl] / ((T)1. - zra1s * s.rb1s[jl]);
            zra1s = s.rb1s[jl] + s.tb1u[jl] * zra1s * s.tb1u[jl] / ((T)1. - zra1s * s.rb1s[jl]);
            zra2 = s.rb2[jl] + s.tb2[jl] * zra2 * s.tb2u[jl] / ((T)1. - zra2s * s.rb2s[jl]);
            zra2s = s.rb2s[jl] + s.tb2u[jl] * zra2s * s.tb2u[jl] / ((T)1. - zra2s * s.rb2s[jl]);
        }
        s.rl1[0] = zra1; s.rl2[0] = zra2; s.rl1s[0] = zra1s; s.rl2s[0] = zra2s;
    }
    __syncwarp();
    for (int jl = lane; jl < E; jl += 32) {
        T z1mrabr = (T)1. / ((T)1. - s.r1s[jl] * s.rl1s[jl]);
        T zfd1 = s.t1[jl] * z1mrabr;
        T zfu1 = -s.t1[jl] * s.rl1[jl] * z1mrabr;
        z1mrabr = (T)1. / ((T)1. - s.r2s[jl] * s.rl2s[jl]);
        T zfd2 = s.t2[jl] * z1mrabr;
        T zfu2 = -s.t2[jl] * s.rl2[jl] * z1mrabr;
        s.fu[jl] = zfu1 * zftop1 + zfu2 * zftop2;
        s.fd[jl] = zfd1 * zftop1 + zfd2 * zftop2;
        s.sw[jl] = s.fu[jl] + s.fd[jl];
    }
    __syncwarp();
}

template <typename T>
__device__ void lwr_warp(const exotx_rad_params &P, ColScratch<T> &s, int L, T dp, T dls, int lane) {
    const T SBK = (T)5.67e-8;
    const T zmmair = (T)0.0289644, zmmco2 = (T)0.0440098, zpv2pm = zmmco2 / zmmair;
    const T zrco2 = (T)1.9635, zro3 = (T)2.14;
    const T zfh2o = (T)0.1, zfco2 = (T)100. / zrco2, zfo3 = (T)100. / zro3;
    const T zero = (T)1.e-6;
    const T ga = (T)P.ga;
    const int E = L + 1;
    const T zao30 = (T)0.209 * P_((T)7.e-5, (T)0.436);
    const T zco20 = (T)0.0676 * P_((T)0.01022, (T)0.421);
    const T zh2o0a = (T)0.846 * P_((T)3.59e-5, (T)0.243);
    const T zh2o0 = (T)0.832 * P_((T)0.0286, (T)0.26);
    const T zao3c = (T)0.209 * P_((T)0.01 + (T)7.e-5, (T)0.436) - zao30 - (T)0.0212 * log10((T)0.01);
    const T zaco2c = (T)0.0676 * P_((T)1.01022, (T)0.421) - zco20;
    const T zah2oc = (T)0.846 * P_((T)0.01 + (T)3.59e-5, (T)0.243) - zh2o0a - (T)0.24 * log10((T)0.02);
    const T zth2oc = (T)1. - ((T)0.832 * P_((T)2. + (T)0.0286, (T)0.26) - zh2o0) + (T)0.1196 * log((T)2. - (T)0.6931);
    const T zps2 = (P.npbroaden > 0.5) ? dp * dp : (T)101100.0 * (T)101100.0;
    const T th2oc = (T)P.th2oc;
    // sigma T^4 on full levels and the surface
    for (int k = lane; k < E; k += 32) { T t2 = s.dt[k] * s.dt[k]; s.st4[k] = SBK * (t2 * t2); }
    for (int jl = lane; jl < L; jl += 32) {
        T zzf1 = (T)P.sigma[jl] * (T)P.dsigma[jl] / ga / (T)100000.;
        T zzf2 = zpv2pm * (T)1.e-6;
        T zzf3 = (T)-1.66 * (T)P.acllwr * (T)1000. * (T)P.dsigma[jl] / ga;
        T zsfac = zzf1 * zps2;
        s.q[jl] = zfh2o * zsfac * s.dq[jl];
        s.qo3[jl] = zfo3 * zsfac * s.o3[jl];
        s.qco2[jl] = zfco2 * zzf2 * zsfac * s.co2[jl];
        if (P.clgray > 0) s.taucc0[jl] = (T)1. - s.dcc[jl] * (T)P.clgray;
        else s.taucc0[jl] = (T)1. - s.dcc[jl] * ((T)1. - exp(zzf3 * s.dql[jl] * dp));
    }
    __syncwarp();
    // half levels (:2230-2249)
    for (int k = lane; k < E; k += 32) {
        T v;
        if (k == 0) {
            v = s.st4[0] - (s.st4[0] - s.st4[1]) * (T)P.sigma[0] / ((T)P.sigma[0] - (T)P.sigma[1]);
        } else if (k < L) {
            v = (s.st4[k] * ((T)P.sigma[k - 1] - (T)P.sigmah[k - 1]) + s.st4[k - 1] * ((T)P.sigmah[k - 1] - (T)P.sigma[k])) /
                ((T)P.sigma[k - 1] - (T)P.sigma[k]);
        } else {
            v = s.st4[L];
            T h_L = (s.st4[L - 1] * ((T)P.sigma[L - 2] - (T)P.sigmah[L - 2]) +
                     s.st4[L - 2] * ((T)P.sigmah[L - 2] - (T)P.sigma[L - 1])) /
                    ((T)P.sigma[L - 2] - (T)P.sigma[L - 1]);
            if (!((s.st4[L - 1] - h_L) * (s.st4[L - 1] - s.st4[L]) > (T)0.))
                v = s.st4[L - 1] + (s.st4[L - 1] - s.st4[L - 2]) * ((T)1. - (T)P.sigma[L - 1]) /
                                       ((T)P.sigma[L - 1] - (T)P.sigma[L - 2]);
        }
        s.st4h[k] = v;
    }
    __syncwarp();
    // clear-sky transmissivities for every (jlev, jlev2 >= jlev) pair, lanes over pairs.
    // Each pair sums its absorbers from jlev upward in the reference order (:2297-2301).
    const int npair = L * (L + 1) / 2;
    for (int pi = lane; pi < npair; pi += 32) {
        // decode pair index -> (jl, jl2): rows jl have L-jl entries
        int jl = 0, rem = pi;
        while (rem >= L - jl) { rem -= L - jl; jl++; }
        int jl2 = jl + rem;
        T zsumwv = 0, zsumo3 = 0, zsumco2 = 0;
        for (int k = jl; k <= jl2; k++) { zsumwv = zsumwv + s.q[k]; zsumo3 = zsumo3 + s.qo3[k]; zsumco2 = zsumco2 + s.qco2[k]; }
        T zah2o, zaco2, zth2o, zao3;
        if (zsumwv <= (T)0.01) zah2o = (T)0.846 * P_(zsumwv + (T)3.59e-5, (T)0.243) - zh2o0a;
        else zah2o = (T)0.24 * log10(zsumwv + (T)0.01) + zah2oc;
        if (th2oc > (T)0.) zah2o = fmin(zah2o + ((T)1. - exp(-th2oc * zsumwv)), (T)1.);
        if (zsumco2 <= (T)1.0) zaco2 = (T)0.0676 * P_(zsumco2 + (T)0.01022, (T)0.421) - zco20;
        else zaco2 = (T)0.0546 * log10(zsumco2) + zaco2c;
        if (zsumwv <= (T)2.) zth2o = (T)1. - ((T)0.832 * P_(zsumwv + (T)0.0286, (T)0.26) - zh2o0);
        else zth2o = fmax((T)0., zth2oc - (T)0.1196 * log(zsumwv - (T)0.6931));
        if (zsumo3 <= (T)0.01) zao3 = (T)0.209 * P_(zsumo3 + (T)7.e-5, (T)0.436) - zao30;
        else zao3 = (T)0.0212 * log10(zsumo3) + zao3c;
        T tcs = (T)1. - zah2o - zao3 - zaco2 * zth2o;
        tcs = fmin((T)1. - zero, fmax(zero, tcs));
        s.tau[jl * L + jl2] = tcs;
    }
    __syncwarp();
    // effective emission of each layer from the jlev = 1 transmissivities (:2376-2400)
    for (int jl2 = lane; jl2 < L; jl2 += 32) {
        T prev = (jl2 == 0) ? (T)1. - zero : s.tau[jl2 - 1];
        T ztau0 = s.tau[jl2] / prev * s.taucc0[jl2] * (T)P.tpofmt;
        ztau0 = fmin((T)1. - zero, fmax(zero, ztau0));
        T a = s.st4[jl2], h0 = s.st4h[jl2], h1 = s.st4h[jl2 + 1];
        T bd, bu;
        if ((a - h0) * (a - h1) > (T)0.) {
            bd = (T)0.5 * a + (T)0.25 * (h0 + h1);
            bu = bd;
        } else {
            bd = (h1 - ztau0 * h0) / ((T)1. - ztau0) - (h0 - h1) / log(ztau0);
            bu = h0 + h1 - bd;
        }
        s.bd[jl2 + 1] = bd;
        s.bu[jl2 + 1] = bu;
    }
    if (lane == 0) {
        s.bd[0] = 0;   // SBK * zttop**4 with zttop = 0
        s.bu[E] = (dls + (T)0.98 * ((T)1. - dls)) * s.st4[L];
    }
    __syncwarp();
    // cloud transmissivity with random overlap: running product along each row
    for (int jl = lane; jl < L; jl += 32) {
        T ztaucc = 1;
        for (int jl2 = jl; jl2 < L; jl2++) {
            ztaucc = ztaucc * s.taucc0[jl2];
            s.tau[jl * L + jl2] = s.tau[jl * L + jl2] * ztaucc;
        }
    }
    __syncwarp();
    // fluxes (:2401-2415), each sum in the reference's order.
    // upward dftu(jlev): -zbu(jlev) then the terms of jlev2 = jlev..NLEV;
    // downward dftd(k): rows jlev < k contribute zbdl(jlev)*ztau(jlev,k-1) in
    // order, then iteration jlev = k (or the surface step) adds zbd(k-1).
    for (int k = lane; k < E; k += 32) {
        if (k < L) {
            T u = (T)0 - s.bu[k + 1];
            for (int jl2 = k; jl2 < L; jl2++) u = u - (s.bu[jl2 + 2] - s.bu[jl2 + 1]) * s.tau[k * L + jl2];
            s.ftu[k] = u;
        }
        T d = 0;
        for (int jl = 0; jl < k; jl++) d = d + (s.bd[jl] - s.bd[jl + 1]) * s.tau[jl * L + (k - 1)];
        s.ftd[k] = d + s.bd[k];
    }
    __syncwarp();
    if (lane == 0) {
        s.ftu[L] = (T)0 - s.bu[E];
        T zeps = dls + (T)0.98 * ((T)1. - dls);
        s.sc[8] = ((T)1. - zeps) * s.ftd[L];
    }
    __syncwarp();
    T zeps = s.sc[8];
    for (int k = lane; k < E; k += 32) {
        if (k < L) s.ftu[k] = s.ftu[k] - s.tau[k * L + (L - 1)] * zeps;
        s.lw[k] = s.ftu[k] + s.ftd[k];
    }
    __syncwarp();
}

// cos zenith of column (jlat, jlon) clipped at dawn (solang, radmod.f90:1380-1436)
template <typename T>
__device__ __forceinline__ T solang_mu(const exotx_rad_params &P, const T *sid, const T *cola, int jlat, int jlon,
                                       int nlon) {
    const T PI = (T)3.14159265359, TWOPI = PI + PI;
    T zdawn = sin((T)P.dawn * PI / (T)180.0), zmuz;
    if (P.ncstsol == 0) {
        T zrlon = TWOPI / nlon;
        T zhangle = (T)P.zmins * (T)P.zrtim + jlon * zrlon - PI;
        if (P.ngenkeplerian == 1) zhangle = zhangle - (T)P.rasc;
        if (zhangle < -PI) zhangle = zhangle + TWOPI;
        if (zhangle > PI) zhangle = zhangle - TWOPI;
        if (P.nfixed == 1) zhangle = zhangle + PI;
        zmuz = sin((T)P.zdecl) * sid[jlat] + cola[jlat] * cos((T)P.zdecl) * cos(zhangle);
    } else {
        T solclatcdec = (T)P.solclat * (T)P.solcdec;
        T solslat = sqrt((T)1 - (T)P.solclat * (T)P.solclat);
        T solsdec = sqrt((T)1 - (T)P.solcdec * (T)P.solcdec);
        if (P.ndcycle == 1) zmuz = solslat * solsdec + solclatcdec * cos((T)P.zmins * (T)P.zrtim - PI);
        else zmuz = solslat * solsdec + solclatcdec / PI;
    }
    return (zmuz > zdawn) ? zmuz : (T)0.0;
}

template <typename T>
__global__ void __launch_bounds__(RAD_WARPS * 32) k_radstep(RadDev D) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const exotx_rad_params &P = D.p;
    const int L = P.nlev, E = L + 1, nhor = P.nhor, nlon = P.nlon;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t per_warp = scratch_elems<T>(L);
    T *base = reinterpret_cast<T *>(smraw) + per_warp * warp;
    ColScratch<T> s = carve<T>(base, L);
    const T *dt = (const T *)D.dt, *dq = (const T *)D.dq, *dcc = (const T *)D.dcc, *dql = (const T *)D.dql;
    const T *dqco2 = (const T *)D.dqco2, *dpv = (const T *)D.dp, *dlsv = (const T *)D.dls,
            *dicv = (const T *)D.dicec, *sid = (const T *)D.sid, *cola = (const T *)D.cola;
    T *dqo3 = (T *)D.dqo3, *gmu0 = (T *)D.gmu0, *dalbv = (T *)D.dalb, *dsalbv = (T *)D.dsalb;
    const T PI = (T)3.14159265359, TWOPI = PI + PI;
    const T ga = (T)P.ga, gascon = (T)P.gascon;
    const int nwarps = blockDim.x >> 5;
    const int count = D.cols ? *D.ncols : nhor;
    for (int w = blockIdx.x * nwarps + warp; w < count; w += gridDim.x * nwarps) {
        const int col = D.cols ? D.cols[w] : w;
        const int jlat = col / nlon, jlon = col - jlat * nlon;
        T csol1 = (T)P.zsolar1, csol2 = (T)P.zsolar2, crco = (T)P.rcoeff;
        if (D.zsol) {
            const T *z = (const T *)D.zsol;
            csol1 = z[col];
            csol2 = z[(size_t)nhor + col];
            crco = z[2 * (size_t)nhor + col];
        }
        for (int k = lane; k < E; k += 32) {
            s.dt[k] = dt[(size_t)k * nhor + col];
            s.dq[k] = dq[(size_t)k * nhor + col];
            s.dcc[k] = dcc[(size_t)k * nhor + col];
            s.dql[k] = dql[(size_t)k * nhor + col];
            if (k < L) s.co2[k] = dqco2[(size_t)k * nhor + col];
            if (k < L && P.no3 != 1) s.o3[k] = dqo3[(size_t)k * nhor + col];
        }
        const T dp = dpv[col], dls = dlsv[col], dicec = dicv[col];
        __syncwarp();
        // solang (radmod.f90:1380-1436)
        T mu0;
        if (P.nsol == 1) {
            mu0 = solang_mu<T>(P, sid, cola, jlat, jlon, nlon);
            if (lane == 0) gmu0[col] = mu0;
        } else {
            mu0 = gmu0[col];
        }
        // insolation and cloud zenith factors (radmod.f90:1650-1669): the
        // column's own cos zenith, or with ndcycle = 0 the means over its
        // latitude row -- over the sunlit columns (clouds) and over all
        // (insolation).  Every warp of the row forms the same sums, reading the
        // row's gmu0 or, when this launch computes gmu0, evaluating solang for
        // each column of the row itself.
        T mu1 = mu0;
        if (P.ndcycle == 0) {
            T zsum = 0;
            int icnt = 0;
            for (int j = lane; j < nlon; j += 32) {
                T g = P.nsol == 1 ? solang_mu<T>(P, sid, cola, jlat, j, nlon) : gmu0[(size_t)jlat * nlon + j];
                zsum += g;
                icnt += g > (T)0.0 ? 1 : 0;
            }
            for (int o = 16; o > 0; o >>= 1) {
                zsum += __shfl_xor_sync(0xffffffffu, zsum, o);
                icnt += __shfl_xor_sync(0xffffffffu, icnt, o);
            }
            mu0 = icnt > 0 ? zsum / (T)icnt : (T)0.0;
            mu1 = icnt > 0 ? zsum / (T)nlon : (T)0.0;
        }
        // mko3 (radmod.f90:1489-1522): serial in height on lane 0
        if (P.no3 == 1) {
            if (lane == 0) {
                const T zfo3 = (T)100.0 / (T)2.14;
                T sd = sid[jlat];
                T za = (T)P.a0o3 + (T)P.a1o3 * fabs(sd) + (T)P.aco3 * sd * cos(TWOPI * ((T)P.zcday - (T)P.toffo3));
                T zconst = exp(-(T)P.bo3 / (T)P.co3);
                T zo3t = za, zh = 0;
                for (int jl = L - 1; jl >= 1; jl--) {
                    zh = zh - s.dt[jl] * gascon / ga * log((T)P.sigmah[jl - 1] / (T)P.sigmah[jl]);
                    T zo3 = -(za + za * zconst) / ((T)1. + exp((zh - (T)P.bo3) / (T)P.co3)) + zo3t;
                    s.o3[jl] = zo3 * ga / (zfo3 * (T)P.dsigma[jl] * dp);
                    zo3t = zo3t - zo3;
                }
                s.o3[0] = zo3t * ga / (zfo3 * (T)P.dsigma[0] * dp);
                if (P.o3scale != 1.0)
                    for (int jl = 0; jl < L; jl++) s.o3[jl] = s.o3[jl] * (T)P.o3scale;
            }
            __syncwarp();
            for (int k = lane; k < L; k += 32) dqo3[(size_t)k * nhor + col] = s.o3[k];
        }
        __syncwarp();
        T dalb = dalbv[col];
        T dsalb[2] = {dsalbv[2 * col], dsalbv[2 * col + 1]};
        if (P.nswr == 1) {
            swr_warp<T>(P, s, L, mu0, mu1, dp, dalb, dsalb, dls, dicec, csol1, csol2, crco, lane);
        } else {
            for (int k = lane; k < E; k += 32) { s.fu[k] = 0; s.fd[k] = 0; s.sw[k] = 0; }
        }
        if (lane == 0) {
            dalbv[col] = dalb;
            dsalbv[2 * col] = dsalb[0];
            dsalbv[2 * col + 1] = dsalb[1];
        }
        if (P.nlwr == 1) {
            lwr_warp<T>(P, s, L, dp, dls, lane);
        } else {
            for (int k = lane; k < E; k += 32) { s.ftu[k] = 0; s.ftd[k] = 0; s.lw[k] = 0; }
            __syncwarp();
        }
        // outputs and heating rates (radstep :1084-1110)
        for (int k = lane; k < E; k += 32) {
            size_t o = (size_t)k * nhor + col;
            ((T *)D.dfu)[o] = s.fu[k];
            ((T *)D.dfd)[o] = s.fd[k];
            ((T *)D.dswfl)[o] = s.sw[k];
            ((T *)D.dftu)[o] = s.ftu[k];
            ((T *)D.dftd)[o] = s.ftd[k];
            ((T *)D.dlwfl)[o] = s.lw[k];
            ((T *)D.dflux)[o] = s.lw[k] + s.sw[k];
        }
        for (int jl = lane; jl < L; jl += 32) {
            size_t o = (size_t)jl * nhor + col;
            T fl0 = s.lw[jl] + s.sw[jl], fl1 = s.lw[jl + 1] + s.sw[jl + 1];
            T zdh;
            if (jl >= 1) zdh = -s.dt[jl] * gascon / ga * log((T)P.sigmah[jl - 1] / (T)P.sigmah[jl]);
            else zdh = -s.dt[0] * gascon / ga * log((T)P.sigma[0] / (T)P.sigmah[0]) * (T)0.5;
            T den = (T)P.dsigma[jl] * dp * (T)P.acpd * ((T)1. + (T)P.adv * s.dq[jl]);
            T zdtdt = -(ga * (fl1 - fl0) / den);
            ((T *)D.dtdt)[o] = ((T *)D.dtdt)[o] + zdtdt;
            ((T *)D.dtdtswr)[o] = -(ga * (s.sw[jl + 1] - s.sw[jl]) / den);
            ((T *)D.dtdtlwr)[o] = -(ga * (s.lw[jl + 1] - s.lw[jl]) / den);
            ((T *)D.dconv)[o] = (fl0 - fl1) / (zdh + (T)1.0e-9);
        }
        __syncwarp();
    }
}

}  // namespace exotx
