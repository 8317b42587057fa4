// Plan construction: Gaussian grid and associated-Legendre tables built on
// the GPU in FP64, then laid out for the folded transform kernels.
//
// This file is compiled with -fmad=false so every product and sum is rounded
// separately, in the order the reference's 8-byte build evaluates them.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "exotx_internal.cuh"

namespace exotx {

static std::atomic<unsigned long long> g_launches{0};
void note_launch(unsigned n) { g_launches += n; }

// ---------------------------------------------------------------- inigau
// ql / qld follow gaussmod.f90:46-86; the Newton loop follows :23-37.
__device__ double ql_dev(int k, double p) {
    double z0 = acos(p), z1 = 1.0, z2 = 0.0, z3 = 0.0, z4;
    for (int j = k; j >= 0; j -= 2) {
        z3 = z1 * cos(z0 * j);
        z2 = z2 + z3;
        z4 = (double)((k - j + 1) * (k + j)) * 0.5;
        z1 = z1 * z4 / (z4 + (j - 1));
    }
    if (k % 2 == 0) z2 = z2 - 0.5 * z3;
    z0 = sqrt(2.0);
    for (int j = 1; j <= k; j++) z0 = z0 * sqrt(1.0 - 0.25 / (double)(j * j));
    return z0 * z2;
}

__device__ double qld_dev(int k, double p) {
    double z = p * ql_dev(k, p) - sqrt((k + k + 1.0) / (k + k - 1.0)) * ql_dev(k - 1, p);
    return (p * p - 1.0) / (k * z);
}

// one thread per northern latitude; writes both hemispheres
__global__ void k_inigau(int klat, double *pz0, double *pzw) {
    int jlat = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (jlat > klat / 2) return;
    const double PI = 3.14159265358979;
    const double ZEPS = 1.0e-16;
    double z0 = PI / (2 * klat + 1);
    double z1 = 1.0 / (double)(klat * klat * 8);
    double z4 = 2.0 / (double)(klat * klat);
    double z2 = z0 * (2 * jlat - 0.5);
    z2 = cos(z2 + z1 / tan(z2));
    for (int jiter = 1; jiter <= 50; jiter++) {
        double z3 = ql_dev(klat, z2) * qld_dev(klat, z2);
        z2 = z2 - z3;
        if (fabs(z3) < ZEPS) break;
    }
    double z5 = ql_dev(klat - 1, z2) / sqrt(klat - 0.5);
    pz0[jlat - 1] = z2;
    pzw[jlat - 1] = z4 * (1.0 - z2 * z2) / (z5 * z5);
    pz0[klat - jlat] = -z2;
    pzw[klat - jlat] = pzw[jlat - 1];
}

// ---------------------------------------------------------------- legini
// One block per latitude.  Thread 0 runs the sectoral chain f1m/f2m over m
// (legmod.f90:68-72, sequential by construction); then each thread runs the
// n-recurrence of its own m columns (:82-88) and writes the eight derived
// tables (:99-116) in the reference layout q(NCSP,NLAT).
__global__ void k_legini(int nlat, int ntru, int ncsp, const int *woff, const double *sid,
                         const double *gwd, double *qref) {
    extern __shared__ __align__(16) double sh[];
    double *f1 = sh, *f2 = sh + (ntru + 1);
    int jlat = blockIdx.x;
    double zsin = sid[jlat], zgwd = gwd[jlat];
    double zcsq = 1.0 - zsin * zsin;
    double zgwdcsq = zgwd / zcsq;
    if (threadIdx.x == 0) {
        double f1m = sqrt(1.5), f2m = 0.0;
        f1[0] = f1m;
        f2[0] = 0.0;
        for (int m = 1; m <= ntru; m++) {
            f2m = -f1m * sqrt(zcsq / (double)(m + m));
            f1m = f2m * sqrt(m + m + 3.0);
            f1[m] = f1m;
            f2[m] = f2m;
        }
    }
    __syncthreads();
    size_t tsz = (size_t)ncsp * nlat;
    double *qi = qref, *qj = qref + tsz, *qc = qref + 2 * tsz, *qe = qref + 3 * tsz;
    double *qm = qref + 4 * tsz, *qq = qref + 5 * tsz, *qu = qref + 6 * tsz, *qv = qref + 7 * tsz;
    size_t row = (size_t)jlat * ncsp;
    for (int m = threadIdx.x; m <= ntru; m += blockDim.x) {
        int w0 = woff[m];
        double amsq = (double)(m * m);
        // P(m,m), P(m,m+1), Q(m,m)
        double pm2 = (m == 0) ? sqrt(0.5) : f2[m];
        double pzd_prev = (m == 0) ? 0.0 : -m * f2[m] * zsin;
        double pm1 = 0.0;
        bool has2 = (m < ntru);
        if (has2) pm1 = ((m == 0) ? sqrt(1.5) : f1[m]) * zsin;
        // store helper
        auto store = [&](int n, double zpli, double zpld) {
            size_t o = row + w0 + (n - m);
            double znn1 = 0.0;
            if (n > 0) znn1 = 1.0 / (double)(n * (n + 1));
            qi[o] = zpli;
            qj[o] = zpld;
            qc[o] = zpli * zgwd;
            qu[o] = zpli * znn1 * m;
            qv[o] = zpld * znn1;
            qe[o] = zpld * zgwdcsq;
            qq[o] = zpli * zgwdcsq * n * (n + 1) * 0.5;
            qm[o] = zpli * zgwdcsq * m;
        };
        if (!has2) {  // mode (NTRU,NTRU)
            double zpld = -ntru * zsin * pm2;
            store(m, pm2, zpld);
            continue;
        }
        // pm2 = P(n-2), pm1 = P(n-1); Q(n-2) pending in pzd_prev
        for (int n = m + 2; n <= ntru; n++) {
            double z1 = sqrt(((n - 1) * (n - 1) - amsq) / (double)(4 * (n - 1) * (n - 1) - 1));
            double z2 = zsin * pm1 - z1 * pm2;
            double p = z2 * sqrt((4 * n * n - 1) / (n * n - amsq));
            double qd = (1 - n) * z2 + n * z1 * pm2;   // Q(n-1)
            store(n - 2, pm2, pzd_prev);
            pzd_prev = qd;
            pm2 = pm1;
            pm1 = p;
        }
        // now pm2 = P(NTRU-1), pm1 = P(NTRU), pzd_prev = Q(NTRU-1)
        double z3 = sqrt((ntru * ntru - amsq) / (double)(4 * ntru * ntru - 1));
        double qlast = -ntru * zsin * pm1 + (ntru + ntru + 1) * pm2 * z3;
        store(ntru - 1, pm2, pzd_prev);
        store(ntru, pm1, qlast);
    }
}

// inverse layout [t][w][j] for qi,qj,qu,qv (reference tables 0,1,6,7)
__global__ void k_layout_inv(int nlat, int ncsp, int nlath, const double *qref, double *inv64,
                             float *inv32) {
    size_t tsz = (size_t)ncsp * nlat;
    size_t total = (size_t)4 * ncsp * nlath;
    const int src[4] = {0, 1, 6, 7};
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        int j = (int)(i % nlath);
        size_t r = i / nlath;
        int w = (int)(r % ncsp);
        int t = (int)(r / ncsp);
        double v = qref[src[t] * tsz + (size_t)j * ncsp + w];
        inv64[i] = v;
        inv32[i] = (float)v;
    }
}

// forward layout per m block [t][woff(m)*nlath + j*K_m + (n-m)] for qc,qe,qm,qq (2,3,4,5)
__global__ void k_layout_fwd(int nlat, int ntru, int ncsp, int nlath, const int *woff,
                             const double *qref, double *fwd64, float *fwd32) {
    size_t tsz = (size_t)ncsp * nlat;
    size_t total = (size_t)4 * ncsp * nlath;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        int t = (int)(i / ((size_t)ncsp * nlath));
        size_t r = i % ((size_t)ncsp * nlath);
        // find m: woff[m]*nlath <= r < woff[m+1]*nlath (binary search)
        int lo = 0, hi = ntru;
        while (lo < hi) {
            int mid = (lo + hi + 1) / 2;
            if ((size_t)woff[mid] * nlath <= r) lo = mid; else hi = mid - 1;
        }
        int m = lo, K = ntru + 1 - m;
        size_t rr = r - (size_t)woff[m] * nlath;
        int j = (int)(rr / K), k = (int)(rr % K);
        double v = qref[(2 + t) * tsz + (size_t)j * ncsp + woff[m] + k];
        fwd64[i] = v;
        fwd32[i] = (float)v;
    }
}

// Filter coefficients (legmod.f90:124-155, pyfft.f90:152-156); index n-1.
static void host_filters(const exotx_grid_desc &d, int ntru, std::vector<double> &g,
                         std::vector<double> &s) {
    int ntp1 = ntru + 1;
    g.assign(ntp1, 1.0);
    s.assign(ntp1, 1.0);
    for (int n = 1; n <= ntp1; n++) {
        double gv = 1.0, sv = 1.0, rn = (double)n;
        if (d.pyfft_nfs >= 0) {
            // pyfft is compiled without -fdefault-real-8: 4-byte arithmetic
            float x = (float)n / (float)ntru;
            float x2 = x * x, x4 = x2 * x2, x8 = x4 * x4;
            float f = expf(-8.0f * x8);
            gv = sv = (double)(1 - d.pyfft_nfs) * 1.0 + (double)d.pyfft_nfs * (double)f;
        } else if (d.nfilter == 1) {
            gv = (1 - d.ngptfilter) * gv + d.ngptfilter * (1.0 - rn / ntp1);
            sv = (1 - d.nspvfilter) * sv + d.nspvfilter * (1.0 - rn / ntp1);
        } else if (d.nfilter == 2) {
            double e = exp(-d.filterkappa * pow(rn / ntru, d.nfilterexp));
            gv = (1 - d.ngptfilter) * gv + d.ngptfilter * e;
            sv = (1 - d.nspvfilter) * sv + d.nspvfilter * e;
        } else if (d.nfilter == 3) {
            double r = rn * (double)(n + 1) / (d.landhoskn0 * (d.landhoskn0 + 1));
            gv = (1 - d.ngptfilter) * gv + d.ngptfilter * exp(-(r * r));
            sv = (1 - d.nspvfilter) * sv + d.nspvfilter * exp(-(r * r));
        } else if (d.nfilter == 4) {
            double r = 1.0 - rn / ntp1;
            gv = (1 - d.ngptfilter) * gv + d.ngptfilter * (r * r);
            sv = (1 - d.nspvfilter) * sv + d.nspvfilter * (r * r);
        }
        g[n - 1] = gv;
        s[n - 1] = sv;
    }
}

exotx_status ensure_work(exotx_plan p, size_t bytes) {
    if (p->work_bytes >= bytes) return EXOTX_OK;
    if (p->d_work) {
        cudaDeviceSynchronize();
        cudaFree(p->d_work);
        p->d_work = nullptr;
        p->work_bytes = 0;
    }
    EXOTX_CUDA(cudaMalloc(&p->d_work, bytes));
    p->work_bytes = bytes;
    return EXOTX_OK;
}

static void plan_free(exotx_plan p) {
    if (!p) return;
    host_pipe_free(p);
    tc_free(p);
    cudaFree(p->d_woff);
    cudaFree(p->d_sid);
    cudaFree(p->d_gwd);
    cudaFree(p->d_qref);
    cudaFree(p->d_inv64);
    cudaFree(p->d_inv32);
    cudaFree(p->d_fwd64);
    cudaFree(p->d_fwd32);
    cudaFree(p->d_fs64);
    cudaFree(p->d_fg64);
    cudaFree(p->d_fs32);
    cudaFree(p->d_fg32);
    cudaFree(p->d_work);
    delete p;
}

}  // namespace exotx

using namespace exotx;

EXOTX_API unsigned long long exotx_launch_count(void) { return g_launches.load(); }

EXOTX_API const char *exotx_status_string(exotx_status st) {
    switch (st) {
        case EXOTX_OK: return "ok";
        case EXOTX_BAD_DIM: return "unsupported dimension";
        case EXOTX_UNSUPPORTED_N: return "FFT length not supported";
        case EXOTX_BAD_ARG: return "bad argument";
        case EXOTX_CUDA_ERR: return "CUDA error";
        case EXOTX_NO_MEM: return "out of device memory";
        case EXOTX_TIMEOUT: return "device wait timed out";
        case EXOTX_NOT_BUILT: return "path not available in this build";
    }
    return "unknown status";
}

EXOTX_API exotx_status exotx_grid_desc_default(int nlat, exotx_grid_desc *d) {
    if (!d) return EXOTX_BAD_ARG;
    memset(d, 0, sizeof(*d));
    d->nlat = nlat;
    d->nfilter = 0;
    d->ngptfilter = 0;
    d->nspvfilter = 0;
    d->landhoskn0 = 15.0;
    d->filterkappa = 8.0;
    d->nfilterexp = 8;
    d->pyfft_nfs = -1;
    d->plavor = 1.63299310207;  // EZ = 1/sqrt(3/8), plasimmod.f90:118,227
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_inigau(int nlat, double *sid, double *gwd, exotx_stream s) {
    if (nlat < 2 || nlat % 2 || !sid || !gwd) return EXOTX_BAD_ARG;
    int nh = nlat / 2;
    k_inigau<<<(nh + 63) / 64, 64, 0, (cudaStream_t)s>>>(nlat, sid, gwd);
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_plan_create(const exotx_grid_desc *d, exotx_plan *out) {
    if (!d || !out) return EXOTX_BAD_ARG;
    *out = nullptr;
    int nlat = d->nlat;
    // NLAT even, NLON = 2 NLAT a supported FFT length, NTRU >= 1
    if (nlat < 4 || nlat % 2 || nlat > 2048) return EXOTX_BAD_DIM;
    if (!exotx_fft_supported(2 * nlat)) return EXOTX_UNSUPPORTED_N;
    if (d->nfilter < 0 || d->nfilter > 4 || d->pyfft_nfs > 1) return EXOTX_BAD_ARG;
    exotx_plan p = new exotx_plan_s();
    p->desc = *d;
    p->nlat = nlat;
    p->nlon = 2 * nlat;
    p->ntru = (p->nlon - 1) / 3;
    p->ntp1 = p->ntru + 1;
    p->ncsp = p->ntp1 * (p->ntru + 2) / 2;
    p->nlath = nlat / 2;
    p->kmax = p->ntp1;
    int ntp1 = p->ntp1, ncsp = p->ncsp, nlath = p->nlath;
    std::vector<int> woff(ntp1 + 1);
    woff[0] = 0;
    for (int m = 0; m < ntp1; m++) woff[m + 1] = woff[m] + (ntp1 - m);
    std::vector<double> g, sv;
    host_filters(*d, p->ntru, g, sv);
    std::vector<float> g32(g.begin(), g.end()), s32(sv.begin(), sv.end());
    size_t tsz = (size_t)ncsp * nlat;
    size_t half = (size_t)4 * ncsp * nlath;
    exotx_status st = EXOTX_OK;
#define PALLOC(ptr, bytes)                                           \
    do {                                                             \
        if (cudaMalloc(&(ptr), (bytes)) != cudaSuccess) {            \
            st = EXOTX_NO_MEM;                                       \
            goto fail;                                               \
        }                                                            \
    } while (0)
    PALLOC(p->d_woff, sizeof(int) * (ntp1 + 1));
    PALLOC(p->d_sid, sizeof(double) * nlat);
    PALLOC(p->d_gwd, sizeof(double) * nlat);
    PALLOC(p->d_qref, sizeof(double) * 8 * tsz);
    PALLOC(p->d_inv64, sizeof(double) * half);
    PALLOC(p->d_inv32, sizeof(float) * half);
    PALLOC(p->d_fwd64, sizeof(double) * half);
    PALLOC(p->d_fwd32, sizeof(float) * half);
    PALLOC(p->d_fs64, sizeof(double) * ntp1);
    PALLOC(p->d_fg64, sizeof(double) * ntp1);
    PALLOC(p->d_fs32, sizeof(float) * ntp1);
    PALLOC(p->d_fg32, sizeof(float) * ntp1);
#undef PALLOC
    {
        cudaStream_t s = 0;
        if (cudaMemcpy(p->d_woff, woff.data(), sizeof(int) * (ntp1 + 1), cudaMemcpyHostToDevice) ||
            cudaMemcpy(p->d_fg64, g.data(), sizeof(double) * ntp1, cudaMemcpyHostToDevice) ||
            cudaMemcpy(p->d_fs64, sv.data(), sizeof(double) * ntp1, cudaMemcpyHostToDevice) ||
            cudaMemcpy(p->d_fg32, g32.data(), sizeof(float) * ntp1, cudaMemcpyHostToDevice) ||
            cudaMemcpy(p->d_fs32, s32.data(), sizeof(float) * ntp1, cudaMemcpyHostToDevice)) {
            st = EXOTX_CUDA_ERR;
            goto fail;
        }
        k_inigau<<<(nlath + 63) / 64, 64, 0, s>>>(nlat, p->d_sid, p->d_gwd);
        note_launch();
        k_legini<<<nlat, 128, sizeof(double) * 2 * ntp1, s>>>(nlat, p->ntru, ncsp, p->d_woff, p->d_sid,
                                                              p->d_gwd, p->d_qref);
        note_launch();
        int blocks = (int)std::min<size_t>((half + 255) / 256, 148 * 16);
        k_layout_inv<<<blocks, 256, 0, s>>>(nlat, ncsp, nlath, p->d_qref, p->d_inv64, p->d_inv32);
        note_launch();
        k_layout_fwd<<<blocks, 256, 0, s>>>(nlat, p->ntru, ncsp, nlath, p->d_woff, p->d_qref, p->d_fwd64,
                                            p->d_fwd32);
        note_launch();
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
            st = EXOTX_CUDA_ERR;
            goto fail;
        }
    }
    *out = p;
    return EXOTX_OK;
fail:
    plan_free(p);
    return st;
}

EXOTX_API exotx_status exotx_plan_destroy(exotx_plan p) {
    if (!p) return EXOTX_BAD_ARG;
    cudaDeviceSynchronize();
    plan_free(p);
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_plan_dims(exotx_plan p, int *nlat, int *nlon, int *ntru, int *ncsp) {
    if (!p) return EXOTX_BAD_ARG;
    if (nlat) *nlat = p->nlat;
    if (nlon) *nlon = p->nlon;
    if (ntru) *ntru = p->ntru;
    if (ncsp) *ncsp = p->ncsp;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_plan_gauss(exotx_plan p, double *sid, double *gwd) {
    if (!p || !sid || !gwd) return EXOTX_BAD_ARG;
    EXOTX_CUDA(cudaMemcpy(sid, p->d_sid, sizeof(double) * p->nlat, cudaMemcpyDeviceToHost));
    EXOTX_CUDA(cudaMemcpy(gwd, p->d_gwd, sizeof(double) * p->nlat, cudaMemcpyDeviceToHost));
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_plan_table(exotx_plan p, int which, double *out) {
    if (!p || !out || which < 0 || which > 7) return EXOTX_BAD_ARG;
    size_t tsz = (size_t)p->ncsp * p->nlat;
    EXOTX_CUDA(cudaMemcpy(out, p->d_qref + which * tsz, sizeof(double) * tsz, cudaMemcpyDeviceToHost));
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_plan_tune(exotx_plan p, int key, long long value) {
    if (!p || value < 0) return EXOTX_BAD_ARG;
    switch (key) {
        case EXOTX_TUNE_CHUNK_INV: p->chunk_inv = (size_t)value; return EXOTX_OK;
        case EXOTX_TUNE_CHUNK_FWD: p->chunk_fwd = (size_t)value; return EXOTX_OK;
        case EXOTX_TUNE_INV_HALF:
            if (value > 1) return EXOTX_BAD_ARG;
            if (p->inv_half_ok != (int)value) {
                // the cached inverse job lists follow the mode: rebuild them
                // (after the work that may still read them)
                EXOTX_CUDA(cudaDeviceSynchronize());
                tc_free(p);
                p->inv_half_ok = (int)value;
            }
            return EXOTX_OK;
    }
    return EXOTX_BAD_ARG;
}
