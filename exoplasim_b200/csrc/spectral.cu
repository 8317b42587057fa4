// Semi-implicit spectral time step on the device (plasim.f90 spectrala
// :2757-2918 and spectrald :3645-3999, one model state, without their
// diagnostic branches): host set-up of the level matrices (initsi
// :1709-1760, makebm :1683-1704) and the diffusion coefficients (:1617-1633),
// and the launchers.  The kernels are in spectral_kernel.cuh.
#include <cmath>
#include <cstring>
#include <vector>
#include "spectral_kernel.cuh"

struct exotx_specconst_s {
    exotx_spec_params h;
    int ntru = 0, nrsp = 0;
    double *d = nullptr;    // constants block (see SpecArgs::k)
    double *sak = nullptr;  // [L][NRSP]
    float *df = nullptr;    // the same two, rounded to FP32 once, for the FP32 step
    float *sakf = nullptr;
    int *nidx = nullptr;    // [NRSP]
};

namespace exotx {
exotx_status launch_spectral_fp64(const SpecBatch<double> &P, int n, bool d_part, cudaStream_t s);

static exotx_status launch_spectral_fp32(const SpecBatch<float> &P, int n, bool d_part, cudaStream_t s) {
    return spec_launch<float>(P, n, d_part, s);
}
}  // namespace exotx

using namespace exotx;

// the inverse of a small matrix (column major), Gauss-Jordan with partial pivoting
static bool invert(std::vector<double> &a, int n) {
    std::vector<double> inv((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) inv[i + (size_t)n * i] = 1.0;
    for (int c = 0; c < n; c++) {
        int piv = c;
        for (int r = c + 1; r < n; r++)
            if (fabs(a[r + (size_t)n * c]) > fabs(a[piv + (size_t)n * c])) piv = r;
        if (a[piv + (size_t)n * c] == 0.0) return false;
        if (piv != c)
            for (int k = 0; k < n; k++) {
                std::swap(a[c + (size_t)n * k], a[piv + (size_t)n * k]);
                std::swap(inv[c + (size_t)n * k], inv[piv + (size_t)n * k]);
            }
        const double d = a[c + (size_t)n * c];
        for (int k = 0; k < n; k++) { a[c + (size_t)n * k] /= d; inv[c + (size_t)n * k] /= d; }
        for (int r = 0; r < n; r++) {
            if (r == c) continue;
            const double f = a[r + (size_t)n * c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; k++) {
                a[r + (size_t)n * k] -= f * a[c + (size_t)n * k];
                inv[r + (size_t)n * k] -= f * inv[c + (size_t)n * k];
            }
        }
    }
    a.swap(inv);
    return true;
}

EXOTX_API exotx_status exotx_spec_params_default(int nlev, exotx_spec_params *p) {
    if (!p || nlev < 2 || nlev > 64) return EXOTX_BAD_ARG;
    memset(p, 0, sizeof(*p));
    p->nlev = nlev;
    p->nqspec = 1;
    p->nhdiff = 15;                                      // plasimmod.f90:199
    const double twopi = 2.0 * 3.14159265359, day = 86400.0, gascon = 287.0, plarad = 6371220.0,
                 sidereal_day = 86164.0;
    p->delt = twopi / 32.0;                              // 32 steps per rotation (plasim.f90:588)
    p->delt2 = p->delt + p->delt;
    p->pnu = 0.1;
    p->pnu21 = 1.0 - 2.0 * p->pnu;
    p->plavor = 1.63299310207;                           // EZ (plasimmod.f90:227)
    p->akap = 0.286;
    const double ww = twopi / sidereal_day, cv = plarad * ww, ct = cv * cv / gascon;
    for (int j = 0; j < nlev; j++) {
        const double z = (double)(j + 1) / nlev;
        p->sigmah[j] = 0.75 * z + 1.75 * z * z * z - 1.5 * z * z * z * z;   // plasim.f90:1554-1564
    }
    p->dsigma[0] = p->sigmah[0];
    for (int j = 1; j < nlev; j++) p->dsigma[j] = p->sigmah[j] - p->sigmah[j - 1];
    for (int j = 0; j < nlev; j++) {
        const double sig = j == 0 ? 0.5 * p->sigmah[0] : 0.5 * (p->sigmah[j - 1] + p->sigmah[j]);
        const double t = 288.0 * pow(sig, 0.0065 * gascon / 9.80665);
        p->t0[j] = (t < 216.65 ? 216.65 : t) / ct;
        // rates in units of 1/(time unit 1/ww): day / (2 pi timescale) (plasim.f90:1583-1615)
        p->tdissq[j] = day / (twopi * 0.1 * day);
        p->tdisst[j] = day / (twopi * 0.76 * day);
        p->tdissz[j] = day / (twopi * 0.3 * day);
        p->tdissd[j] = day / (twopi * 0.06 * day);
        p->ndel[j] = 2;
    }
    p->tfrc[0] = day / (twopi * 20.0 * day);
    p->tfrc[1] = day / (twopi * 100.0 * day);
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_specconst_create(exotx_plan pl, const exotx_spec_params *p, exotx_specconst *out) {
    if (!pl || !p || !out || p->nlev < 2 || p->nlev > 64) return EXOTX_BAD_ARG;
    const int L = p->nlev, ntru = pl->ntru, nrsp = 2 * pl->ncsp;
    if (p->nhdiff < 0 || p->nhdiff >= ntru) return EXOTX_BAD_ARG;
    // initsi (plasim.f90:1709-1760): g, c, tkp, t01s2, tau; rdsig (:1564)
    std::vector<double> g((size_t)L * L, 0.0), c((size_t)L * L), tau((size_t)L * L), zalp(L, 0.0), tkp(L),
        t01s2(L), rdsig(L);
    for (int j = 0; j < L; j++) tkp[j] = p->akap * p->t0[j];
    for (int j = 0; j < L - 1; j++) t01s2[j] = p->t0[j + 1] - p->t0[j];
    t01s2[L - 1] = 0.0;
    for (int j = 1; j < L; j++) zalp[j] = log(p->sigmah[j]) - log(p->sigmah[j - 1]);
    g[0] = 1.0;
    for (int jl = 1; jl < L; jl++) {
        g[jl + (size_t)L * jl] = 1.0 - zalp[jl] * p->sigmah[jl - 1] / p->dsigma[jl];
        for (int k = 0; k < jl; k++) g[jl + (size_t)L * k] = zalp[jl];
    }
    for (int jl = 0; jl < L; jl++)
        for (int k = 0; k < L; k++) c[jl + (size_t)L * k] = g[k + (size_t)L * jl] * (p->dsigma[jl] / p->dsigma[k]);
    for (int j = 0; j < L; j++) rdsig[j] = 0.5 / p->dsigma[j];
    {
        double zt01s2 = t01s2[0], zsig = p->sigmah[0];
        tau[0] = 0.5 * zt01s2 * (zsig - 1.0) + tkp[0];
        for (int j = 1; j < L; j++) tau[j] = 0.5 * zt01s2 * p->dsigma[j];
        for (int jl = 1; jl < L; jl++) {
            const double zttm = zt01s2, zsigm = zsig;
            zt01s2 = t01s2[jl];
            zsig = p->sigmah[jl];
            for (int j2 = 0; j2 < L; j2++) {
                const double ztm = j2 <= jl ? 1. : 0., ztmm = j2 < jl ? 1. : 0.;
                double z = zttm * (zsigm - ztmm);
                if (jl < L - 1) z = z + zt01s2 * (zsig - ztm);
                z = z * rdsig[jl] * p->dsigma[j2];
                if (j2 <= jl) z = z + tkp[jl] * c[j2 + (size_t)L * jl];
                tau[j2 + (size_t)L * jl] = z;
            }
        }
    }
    // makebm (plasim.f90:1683-1704): bm1(n) = (delt^2 (t0 dsigma^T + g^T tau^T) + I/(n(n+1)))^-1
    std::vector<double> base((size_t)L * L), bm1((size_t)(ntru + 1) * L * L, 0.0);
    const double zdeltsq = p->delt * p->delt;
    for (int j1 = 0; j1 < L; j1++)
        for (int j2 = 0; j2 < L; j2++) {
            double dot = 0.0;
            for (int i = 0; i < L; i++) dot += g[i + (size_t)L * j1] * tau[j2 + (size_t)L * i];
            base[j2 + (size_t)L * j1] = zdeltsq * (p->t0[j1] * p->dsigma[j2] + dot);
        }
    for (int jn = 1; jn <= ntru; jn++) {
        std::vector<double> b = base;
        for (int j = 0; j < L; j++) b[j + (size_t)L * j] += 1.0 / (jn * (jn + 1));
        if (!invert(b, L)) return EXOTX_BAD_ARG;
        memcpy(bm1.data() + (size_t)jn * L * L, b.data(), sizeof(double) * L * L);
    }
    // diffusion coefficients sak (plasim.f90:1617-1633) and the n of every real
    std::vector<double> sak((size_t)L * nrsp);
    std::vector<int> nidx(nrsp);
    for (int jl = 0; jl < L; jl++) {
        const int jdel = p->ndel[jl];
        const double zakk = 1. / pow((double)(ntru - p->nhdiff), jdel);
        int jr = 0;
        for (int jm = 0; jm <= ntru; jm++)
            for (int jn = jm; jn <= ntru; jn++) {
                const double v = jn >= p->nhdiff ? zakk * pow((double)(jn - p->nhdiff), jdel) : 0.;
                sak[(size_t)jl * nrsp + jr] = v;
                sak[(size_t)jl * nrsp + jr + 1] = v;
                nidx[jr] = nidx[jr + 1] = jn;
                jr += 2;
            }
    }
    std::vector<double> k((size_t)8 * L + 2 * (size_t)L * L + bm1.size());
    for (int j = 0; j < L; j++) {
        k[j] = p->t0[j]; k[L + j] = p->dsigma[j]; k[2 * L + j] = p->damp[j]; k[3 * L + j] = p->tdisst[j];
        k[4 * L + j] = p->tdissq[j]; k[5 * L + j] = p->tdissd[j]; k[6 * L + j] = p->tdissz[j];
        k[7 * L + j] = p->tfrc[j];
    }
    memcpy(k.data() + 8 * L, g.data(), sizeof(double) * L * L);
    memcpy(k.data() + 8 * L + L * L, tau.data(), sizeof(double) * L * L);
    memcpy(k.data() + 8 * L + 2 * L * L, bm1.data(), sizeof(double) * bm1.size());
    exotx_specconst sc = new exotx_specconst_s();
    sc->h = *p;
    sc->ntru = ntru;
    sc->nrsp = nrsp;
    const std::vector<float> kf(k.begin(), k.end()), sakf(sak.begin(), sak.end());   // rounded to nearest
    bool ok = cudaMalloc(&sc->d, sizeof(double) * k.size()) == cudaSuccess &&
              cudaMalloc(&sc->sak, sizeof(double) * sak.size()) == cudaSuccess &&
              cudaMalloc(&sc->df, sizeof(float) * kf.size()) == cudaSuccess &&
              cudaMalloc(&sc->sakf, sizeof(float) * sakf.size()) == cudaSuccess &&
              cudaMalloc(&sc->nidx, sizeof(int) * nidx.size()) == cudaSuccess &&
              cudaMemcpy(sc->d, k.data(), sizeof(double) * k.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(sc->sak, sak.data(), sizeof(double) * sak.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(sc->df, kf.data(), sizeof(float) * kf.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(sc->sakf, sakf.data(), sizeof(float) * sakf.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(sc->nidx, nidx.data(), sizeof(int) * nidx.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        cudaFree(sc->d); cudaFree(sc->sak); cudaFree(sc->df); cudaFree(sc->sakf); cudaFree(sc->nidx);
        delete sc;
        return EXOTX_NO_MEM;
    }
    *out = sc;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_specconst_destroy(exotx_specconst c) {
    if (!c) return EXOTX_BAD_ARG;
    cudaFree(c->d); cudaFree(c->sak); cudaFree(c->df); cudaFree(c->sakf); cudaFree(c->nidx);
    delete c;
    return EXOTX_OK;
}

template <typename T>
static SpecArgs<T> spec_args(exotx_specconst c, const exotx_spec_state *s) {
    SpecArgs<T> A;
    A.sdp = (T *)s->sdp; A.szp = (T *)s->szp; A.stp = (T *)s->stp; A.sqp = (T *)s->sqp; A.spp = (T *)s->spp;
    A.sdm = (T *)s->sdm; A.szm = (T *)s->szm; A.stm = (T *)s->stm; A.sqm = (T *)s->sqm; A.spm = (T *)s->spm;
    A.sdt = (T *)s->sdt; A.szt = (T *)s->szt; A.stt = (T *)s->stt; A.sqt = (T *)s->sqt; A.spt = (T *)s->spt;
    A.sop = (const T *)s->sop; A.srp = (const T *)s->srp;
    if constexpr (sizeof(T) == 8) { A.k = (const T *)c->d; A.sak = (const T *)c->sak; }
    else { A.k = (const T *)c->df; A.sak = (const T *)c->sakf; }
    A.nidx = c->nidx;
    A.L = c->h.nlev; A.nrsp = c->nrsp; A.ntru = c->ntru; A.nqspec = c->h.nqspec; A.nsponge = c->h.nsponge;
    A.delt = c->h.delt; A.delt2 = c->h.delt2; A.pnu = c->h.pnu; A.pnu21 = c->h.pnu21; A.plavor = c->h.plavor;
    A.dampsp = c->h.dampsp;
    return A;
}

static bool spec_state_ok(exotx_specconst c, const exotx_spec_state *s, bool d_part) {
    const void *need[] = {s->sdp, s->szp, s->stp, s->spp, s->sdm, s->szm, s->stm, s->spm,
                          s->sdt, s->szt, s->stt, s->spt};
    for (const void *q : need) if (!q) return false;
    if (c->h.nqspec == 1 && (!s->sqp || !s->sqm || !s->sqt)) return false;
    if (!d_part && !s->sop) return false;
    if (d_part && !s->srp) return false;
    return true;
}

template <typename T>
static exotx_status spec_run_t(exotx_specconst c, const exotx_spec_state *s, int n, bool d_part, cudaStream_t st) {
    for (int i0 = 0; i0 < n; i0 += SPEC_MAXB) {
        const int nb = n - i0 < SPEC_MAXB ? n - i0 : SPEC_MAXB;
        SpecBatch<T> P;
        for (int i = 0; i < nb; i++) P.s[i] = spec_args<T>(c, s + i0 + i);
        for (int i = nb; i < SPEC_MAXB; i++) P.s[i] = P.s[0];
        if constexpr (sizeof(T) == 8) EXOTX_TRY(launch_spectral_fp64(P, nb, d_part, st));
        else EXOTX_TRY(launch_spectral_fp32(P, nb, d_part, st));
    }
    return EXOTX_OK;
}

static exotx_status spec_run(exotx_specconst c, int prec, const exotx_spec_state *s, int n, bool d_part,
                             exotx_stream st) {
    if (!c || !s || n < 0 || (prec != EXOTX_FP64 && prec != EXOTX_FP32)) return EXOTX_BAD_ARG;
    for (int i = 0; i < n; i++)
        if (!spec_state_ok(c, s + i, d_part)) return EXOTX_BAD_ARG;
    if (n == 0) return EXOTX_OK;
    if (prec == EXOTX_FP64) return spec_run_t<double>(c, s, n, d_part, (cudaStream_t)st);
    return spec_run_t<float>(c, s, n, d_part, (cudaStream_t)st);
}

EXOTX_API exotx_status exotx_spectrala(exotx_specconst c, int prec, const exotx_spec_state *s, exotx_stream st) {
    return spec_run(c, prec, s, 1, false, st);
}
EXOTX_API exotx_status exotx_spectrald(exotx_specconst c, int prec, const exotx_spec_state *s, exotx_stream st) {
    return spec_run(c, prec, s, 1, true, st);
}
EXOTX_API exotx_status exotx_spectrala_batch(exotx_specconst c, int prec, const exotx_spec_state *states, int ninst,
                                             exotx_stream st) {
    return spec_run(c, prec, states, ninst, false, st);
}
EXOTX_API exotx_status exotx_spectrald_batch(exotx_specconst c, int prec, const exotx_spec_state *states, int ninst,
                                             exotx_stream st) {
    return spec_run(c, prec, states, ninst, true, st);
}
