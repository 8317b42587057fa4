// Uneven ensembles of transform sets (no counterpart in the reference, which
// runs one model state per process, plasim.f90 gridpointa :2396-2486).
// Instances of different truncations and level counts are grouped into
// segments of one resolution and level count; each half of the round trip is
// one tensor-core Legendre launch plus one FFT launch over all segments, and
// the forward half one small launch more for the FP64 global means, so the
// whole ensemble step is five kernels (and one CUDA graph when captured).
// Segments whose rows have a register-resident FFT kernel (NLON 384) take one
// FFT launch more per half when they are mixed with other lengths.
#include <algorithm>
#include <cmath>
#include <map>
#include <vector>
#include "exotx_internal.cuh"

struct exotx_ensemble_s {
    int ninst = 0;
    std::vector<exotx_plan> plans;                  // one per distinct nlat
    std::vector<int> seg_plan, seg_L, seg_n;        // per segment
    std::vector<long long> seg_spec, seg_gin, seg_gout, seg_W;  // segment offsets (floats)
    std::vector<long long> spec_off, gin_off, gout_off;          // per instance, caller order
    long long totals[3] = {0, 0, 0};
    float *W = nullptr;
    int4 *jobs[2] = {nullptr, nullptr};
    int njobs[2] = {0, 0};
    size_t smem[2] = {0, 0};
    int nc_qi = 128, nc_uv = 64, nprod = 6;
    int sorted = 1;
};

namespace exotx {

static std::vector<EnsSeg> ens_segs(exotx_ensemble e, const float *spin, float *spout) {
    std::vector<EnsSeg> v(e->seg_L.size());
    for (size_t s = 0; s < v.size(); s++) {
        v[s].p = e->plans[e->seg_plan[s]];
        v[s].L = e->seg_L[s];
        v[s].ninst = e->seg_n[s];
        v[s].spin = spin ? spin + e->seg_spec[s] : nullptr;
        v[s].spout = spout ? spout + e->seg_spec[s] : nullptr;
        v[s].W = e->W + e->seg_W[s];
    }
    return v;
}

static exotx_status ens_build_jobs(exotx_ensemble e) {
    std::vector<EnsSeg> v = ens_segs(e, nullptr, nullptr);
    for (int d = 0; d < 2; d++) {
        cudaFree(e->jobs[d]);
        e->jobs[d] = nullptr;
        EXOTX_TRY(tc_ens_jobs(v.data(), (int)v.size(), d, e->nc_qi, e->nc_uv, e->sorted != 0, &e->jobs[d],
                              &e->njobs[d], &e->smem[d]));
    }
    return EXOTX_OK;
}

static exotx_status ens_inverse(exotx_ensemble e, const float *spin, float *gpout, cudaStream_t s) {
    std::vector<EnsSeg> v = ens_segs(e, spin, nullptr);
    EXOTX_TRY(tc_ens_run(v.data(), (int)v.size(), 0, e->jobs[0], e->njobs[0], e->smem[0], e->nprod, s));
    std::vector<FftEnsSeg> f(v.size());
    for (size_t i = 0; i < v.size(); i++) {
        const exotx_plan p = v[i].p;
        const long long rows = (long long)v[i].ninst * (6 * v[i].L + 3) * p->nlat;
        f[i] = FftEnsSeg{v[i].W, gpout + e->seg_gout[i], rows, 1, rows, p->nlon, p->ntp1};
    }
    return fft_ens(false, f.data(), (int)f.size(), s);
}

static exotx_status ens_forward(exotx_ensemble e, const float *gpin, float *spout, cudaStream_t s) {
    std::vector<EnsSeg> v = ens_segs(e, nullptr, spout);
    std::vector<FftEnsSeg> f(v.size());
    const bool folded = tc_ens_fwd_folded(v.data(), (int)v.size());   // persistent kernel: folded intermediate
    for (size_t i = 0; i < v.size(); i++) {
        const exotx_plan p = v[i].p;
        const long long rows = (long long)v[i].ninst * (9 * v[i].L + 1) * p->nlat;
        f[i] = FftEnsSeg{gpin + e->seg_gin[i], v[i].W, rows, 1, rows, p->nlon, p->ntp1, folded ? p->nlat : 0};
    }
    EXOTX_TRY(fft_ens(true, f.data(), (int)f.size(), s));
    EXOTX_TRY(tc_ens_run(v.data(), (int)v.size(), 1, e->jobs[1], e->njobs[1], e->smem[1], e->nprod, s));
    std::vector<const float *> g(v.size());
    for (size_t i = 0; i < v.size(); i++) g[i] = gpin + e->seg_gin[i];
    return tc_ens_n0(v.data(), g.data(), (int)v.size(), s);   // global means in FP64
}

// acc[0] += sum (a-b)^2, acc[1] += sum b^2
__global__ void k_ens_diff(const float *a, const float *b, long long n, double *acc) {
    __shared__ double r0[256], r1[256];
    double s0 = 0, s1 = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double d = (double)a[i] - (double)b[i];
        s0 += d * d;
        s1 += (double)b[i] * (double)b[i];
    }
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) { r0[threadIdx.x] += r0[threadIdx.x + w]; r1[threadIdx.x] += r1[threadIdx.x + w]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { atomicAdd(acc, r0[0]); atomicAdd(acc + 1, r1[0]); }
}

static exotx_status rel_l2(const float *a, const float *b, long long n, double *acc_dev, double *out,
                           cudaStream_t s) {
    EXOTX_CUDA(cudaMemsetAsync(acc_dev, 0, 2 * sizeof(double), s));
    k_ens_diff<<<(unsigned)std::min<long long>((n + 255) / 256, 148 * 8), 256, 0, s>>>(a, b, n, acc_dev);
    EXOTX_CHECK_LAUNCH();
    double h[2];
    EXOTX_CUDA(cudaMemcpyAsync(h, acc_dev, sizeof(h), cudaMemcpyDeviceToHost, s));
    EXOTX_CUDA(cudaStreamSynchronize(s));
    *out = std::sqrt(h[0] / std::max(h[1], 1e-300));
    return EXOTX_OK;
}

}  // namespace exotx

using namespace exotx;

EXOTX_API exotx_status exotx_ensemble_create(int ninst, const int *nlat, const int *nlev, exotx_ensemble *out) {
    if (ninst < 1 || !nlat || !nlev || !out) return EXOTX_BAD_ARG;
    for (int i = 0; i < ninst; i++)
        if (nlat[i] < 4 || nlev[i] < 1) return EXOTX_BAD_ARG;
    exotx_ensemble e = new exotx_ensemble_s();
    e->ninst = ninst;
    // segments: distinct (nlat, nlev) in increasing order; instances keep caller order inside
    std::map<std::pair<int, int>, std::vector<int>> groups;
    for (int i = 0; i < ninst; i++) groups[{nlat[i], nlev[i]}].push_back(i);
    if ((int)groups.size() > std::min(TC_MAXSEG, FFT_ENS_MAXSEG)) { delete e; return EXOTX_BAD_DIM; }
    std::map<int, int> plan_of;
    e->spec_off.assign(ninst, 0);
    e->gin_off.assign(ninst, 0);
    e->gout_off.assign(ninst, 0);
    long long so = 0, gi = 0, go = 0, wo = 0;
    exotx_status st = EXOTX_OK;
    for (auto &kv : groups) {
        const int nl = kv.first.first, L = kv.first.second;
        if (!plan_of.count(nl)) {
            exotx_grid_desc d;
            exotx_plan p = nullptr;
            st = exotx_grid_desc_default(nl, &d);
            if (st == EXOTX_OK) st = exotx_plan_create(&d, &p);
            if (st != EXOTX_OK) break;
            plan_of[nl] = (int)e->plans.size();
            e->plans.push_back(p);
        }
        const exotx_plan p = e->plans[plan_of[nl]];
        const long long nrsp = 2LL * p->ncsp, nhor = (long long)p->nlat * p->nlon;
        e->seg_plan.push_back(plan_of[nl]);
        e->seg_L.push_back(L);
        e->seg_n.push_back((int)kv.second.size());
        e->seg_spec.push_back(so);
        e->seg_gin.push_back(gi);
        e->seg_gout.push_back(go);
        e->seg_W.push_back(wo);
        for (int i : kv.second) {
            e->spec_off[i] = so; so += (4LL * L + 1) * nrsp;
            e->gin_off[i] = gi; gi += (9LL * L + 1) * nhor;
            e->gout_off[i] = go; go += (6LL * L + 3) * nhor;
        }
        wo += (long long)kv.second.size() * (9LL * L + 1) * p->nlat * p->ntp1 * 2;
    }
    if (st == EXOTX_OK && cudaMalloc(&e->W, sizeof(float) * wo) != cudaSuccess) st = EXOTX_NO_MEM;
    e->totals[0] = so; e->totals[1] = gi; e->totals[2] = go;
    if (st == EXOTX_OK) st = ens_build_jobs(e);
    if (st != EXOTX_OK) { exotx_ensemble_destroy(e); return st; }
    *out = e;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_ensemble_destroy(exotx_ensemble e) {
    if (!e) return EXOTX_BAD_ARG;
    cudaFree(e->W);
    cudaFree(e->jobs[0]);
    cudaFree(e->jobs[1]);
    for (exotx_plan p : e->plans) exotx_plan_destroy(p);
    delete e;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_ensemble_layout(exotx_ensemble e, long long *spec_off, long long *gin_off,
                                             long long *gout_off, long long *totals) {
    if (!e) return EXOTX_BAD_ARG;
    for (int i = 0; i < e->ninst; i++) {
        if (spec_off) spec_off[i] = e->spec_off[i];
        if (gin_off) gin_off[i] = e->gin_off[i];
        if (gout_off) gout_off[i] = e->gout_off[i];
    }
    if (totals) for (int k = 0; k < 3; k++) totals[k] = e->totals[k];
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_ensemble_configure(exotx_ensemble e, int nc_qi, int nc_uv, int sorted, int nprod) {
    if (!e || nc_qi < 16 || nc_uv < 16 || (nprod != 3 && nprod != 6)) return EXOTX_BAD_ARG;
    e->nc_qi = nc_qi; e->nc_uv = nc_uv; e->sorted = sorted != 0; e->nprod = nprod;
    return ens_build_jobs(e);
}

EXOTX_API exotx_status exotx_ensemble_inverse(exotx_ensemble e, const float *spin, float *gpout, exotx_stream s) {
    if (!e || !spin || !gpout) return EXOTX_BAD_ARG;
    return ens_inverse(e, spin, gpout, (cudaStream_t)s);
}

EXOTX_API exotx_status exotx_ensemble_forward(exotx_ensemble e, const float *gpin, float *spout, exotx_stream s) {
    if (!e || !gpin || !spout) return EXOTX_BAD_ARG;
    return ens_forward(e, gpin, spout, (cudaStream_t)s);
}

EXOTX_API exotx_status exotx_ensemble_tune(exotx_ensemble e, const float *spin, float *gpout, const float *gpin,
                                           float *spout, int reps, exotx_stream sv, int *choice, float *best_ms) {
    if (!e || !spin || !gpout || !gpin || !spout || reps < 1) return EXOTX_BAD_ARG;
    cudaStream_t s = (cudaStream_t)sv;
    // reference outputs: 3-term split (6 products), default tiles
    EXOTX_TRY(exotx_ensemble_configure(e, 128, 64, 1, 6));
    float *ref_g = nullptr, *ref_s = nullptr;
    double *acc = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    exotx_status st = EXOTX_OK;
    const long long ng = e->totals[2], ns = e->totals[0];
    if (cudaMalloc(&ref_g, sizeof(float) * ng) != cudaSuccess || cudaMalloc(&ref_s, sizeof(float) * ns) != cudaSuccess ||
        cudaMalloc(&acc, 2 * sizeof(double)) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess)
        st = EXOTX_NO_MEM;
    if (st == EXOTX_OK) st = ens_inverse(e, spin, ref_g, s);
    if (st == EXOTX_OK) st = ens_forward(e, gpin, ref_s, s);
    int best[4] = {128, 64, 1, 6};
    float bms = 1e30f;
    const int qi[2] = {64, 128}, uv[2] = {32, 64}, so[2] = {0, 1}, np[2] = {6, 3};
    for (int a = 0; a < 2 && st == EXOTX_OK; a++)
        for (int b = 0; b < 2 && st == EXOTX_OK; b++)
            for (int c = 0; c < 2 && st == EXOTX_OK; c++)
                for (int d = 0; d < 2 && st == EXOTX_OK; d++) {
                    st = exotx_ensemble_configure(e, qi[a], uv[b], so[c], np[d]);
                    if (st != EXOTX_OK) break;
                    // warm-up and accuracy against the reference (relative L2, both halves)
                    st = ens_inverse(e, spin, gpout, s);
                    if (st == EXOTX_OK) st = ens_forward(e, gpin, spout, s);
                    double eg = 0, es = 0;
                    if (st == EXOTX_OK) st = rel_l2(gpout, ref_g, ng, acc, &eg, s);
                    if (st == EXOTX_OK) st = rel_l2(spout, ref_s, ns, acc, &es, s);
                    if (st != EXOTX_OK) break;
                    if (eg > 1e-6 || es > 1e-6) continue;  // the split choice must hold the 1e-6 bar
                    cudaEventRecord(e0, s);
                    for (int r = 0; r < reps && st == EXOTX_OK; r++) {
                        st = ens_inverse(e, spin, gpout, s);
                        if (st == EXOTX_OK) st = ens_forward(e, gpin, spout, s);
                    }
                    cudaEventRecord(e1, s);
                    if (cudaEventSynchronize(e1) != cudaSuccess) st = EXOTX_CUDA_ERR;
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    ms /= reps;
                    if (st == EXOTX_OK && ms < bms) {
                        bms = ms;
                        best[0] = qi[a]; best[1] = uv[b]; best[2] = so[c]; best[3] = np[d];
                    }
                }
    cudaFree(ref_g);
    cudaFree(ref_s);
    cudaFree(acc);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st != EXOTX_OK) return st;
    EXOTX_TRY(exotx_ensemble_configure(e, best[0], best[1], best[2], best[3]));
    if (choice) for (int k = 0; k < 4; k++) choice[k] = best[k];
    if (best_ms) *best_ms = bms;
    return EXOTX_OK;
}
