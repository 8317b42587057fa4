// Tensor-core (tcgen05) Legendre transforms with 3-term BF16 splits.
#include <algorithm>
#include <cstdio>
#include <vector>
#include "exotx_internal.cuh"
#include "tc_prims.cuh"

namespace exotx {

// error word written by tensor-core kernels when a bounded wait gives up
__device__ int g_tc_error;

// split-product schedule: pairs (i,j) of split terms with i + j <= 2
__constant__ int c_pair_a[6] = {0, 0, 1, 0, 1, 2};
__constant__ int c_pair_b[6] = {0, 1, 0, 2, 1, 0};

// Self-test GEMM: C(128 x N) = A(128 x K) * B(N x K)^T with FP32 inputs split
// into three BF16 terms and nprod (1, 3 or 6) split products accumulated in
// TMEM.  One CTA of 128 threads; N multiple of 16 (<= 256), K multiple of 16 (<= 64).
__global__ void __launch_bounds__(128) k_tc_selftest(const float *A, const float *B, float *C, int N, int K,
                                                    int nprod) {
    extern __shared__ __align__(128) unsigned char smraw[];
    __nv_bfloat16 *sa = reinterpret_cast<__nv_bfloat16 *>(smraw);              // 3 x 128 x K
    __nv_bfloat16 *sb = sa + 3 * 128 * K;                                       // 3 x N x K
    uint64_t *bar = reinterpret_cast<uint64_t *>(sb + 3 * N * K);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc::tmem_alloc(slot, 256);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_fence_init();
    }
    // stage split operands
    for (int i = tid; i < 128 * K; i += blockDim.x) {
        int r = i / K, k = i % K;
        __nv_bfloat16 h, m, l;
        tc::split3(A[i], h, m, l);
        uint32_t o = tc::kmajor_off(r, k, K) / 2;
        sa[o] = h; sa[128 * K + o] = m; sa[2 * 128 * K + o] = l;
    }
    for (int i = tid; i < N * K; i += blockDim.x) {
        int r = i / K, k = i % K;
        __nv_bfloat16 h, m, l;
        tc::split3(B[i], h, m, l);
        uint32_t o = tc::kmajor_off(r, k, K) / 2;
        sb[o] = h; sb[N * K + o] = m; sb[2 * N * K + o] = l;
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    if (tid == 0) {
        const uint32_t idesc = tc::idesc_bf16(128, N);
        bool acc = false;
        for (int kc = 0; kc < K / 16; kc++) {
            for (int p = 0; p < nprod; p++) {
                const __nv_bfloat16 *a = sa + c_pair_a[p] * 128 * K + kc * 128;  // 2 core matrices = 256 B
                const __nv_bfloat16 *b = sb + c_pair_b[p] * N * K + kc * 128;
                uint64_t da = tc::smem_desc(a, 128, (K / 8) * 128);
                uint64_t db = tc::smem_desc(b, 128, (K / 8) * 128);
                tc::mma_bf16(tmem, da, db, idesc, acc);
                acc = true;
            }
        }
        tc::mma_commit(bar);
    }
    bool ok = tc::mbar_wait(bar, 0);
    if (!ok && lane == 0) atomicExch(&g_tc_error, 1);
    tc::fence_after_sync();
    if (ok) {
        const int row = warp * 32 + lane;
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
#pragma unroll
            for (int i = 0; i < 16; i++) C[row * N + c0 + i] = v[i];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

// ===================================================================
// Mixed-precision Legendre transforms on the tensor cores.
//
// Per zonal wavenumber m the transforms are small dense contractions.  Both
// directions are split by the parity of n-m (north/south folding):
//   inverse  D_t,p[j][c] = sum_k'  T_t(m, m+2k'+p, lat j) * X_c(m, m+2k'+p)
//            (M = latitude pairs j, N = field columns c, K = modes k' of parity p)
//   forward  D_t,p[k'][c] = sum_j T_t(m, m+2k'+p, lat j) * F_c^{S|D}(j)
//            (M = modes k', N = field columns, K = latitude pairs; F^S = N+S, F^D = N-S)
// T is the TMA-staged table (A operand), the field data the B operand; both
// are split into three BF16 terms and the six products with split-order
// sum <= 2 accumulate in FP32 in tensor memory.  Each epilogue thread owns one
// TMEM lane (a latitude pair or a mode), combines the table/parity
// accumulators exactly as legmod.f90 combines its terms, and stores.
// ===================================================================

constexpr int TCT = 128;  // threads per CTA (4 warps = the 4 TMEM lane quarters)

// inverse tables: t = 0..3 -> qi, qj, qu, qv (reference tables 0, 1, 6, 7)
// forward tables: t = 0..3 -> qc, qe, qm, qq (reference tables 2, 3, 4, 5)
static const int kInvRef[4] = {0, 1, 6, 7};
static const int kFwdRef[4] = {2, 3, 4, 5};

struct TcTables {
    int nj8;                          // inverse rows: latitude pairs rounded up to 8
    int njc;                          // forward K extent: latitude pairs rounded up to 16
    std::vector<long long> inv_off;   // byte offset of block (m, t), [m*4+t]
    std::vector<int> inv_bytes;
    std::vector<long long> fwd_off;
    std::vector<int> fwd_bytes;
    unsigned char *inv = nullptr, *fwd = nullptr;
    long long *d_inv_off = nullptr, *d_fwd_off = nullptr;
    // cached job lists, keyed by (direction, nlev, ninst)
    struct Jobs { int dir, nlev, ninst, njobs; int4 *d = nullptr; };
    std::vector<Jobs> jobs;
    ~TcTables() {
        cudaFree(inv); cudaFree(fwd); cudaFree(d_inv_off); cudaFree(d_fwd_off);
        for (auto &j : jobs) cudaFree(j.d);
    }
};

__host__ __device__ inline int pad16(int x) { return (x + 15) & ~15; }
__host__ __device__ inline int pad8(int x) { return (x + 7) & ~7; }
// modes of parity p among K = ntp1 - m modes
__host__ __device__ inline int kpar(int K, int p) { return p == 0 ? (K + 1) / 2 : K / 2; }

__device__ __forceinline__ void split3d(double x, __nv_bfloat16 &h, __nv_bfloat16 &m, __nv_bfloat16 &l) {
    h = __double2bfloat16(x);
    double r1 = x - (double)__bfloat162float(h);
    m = __double2bfloat16(r1);
    double r2 = r1 - (double)__bfloat162float(m);
    l = __double2bfloat16(r2);
}

// inverse block (m, t) = [p][split][rows nj8][Kp_p] (K-major core matrices)
__global__ void k_build_tc_inv(const double *qref, const int *woff, const long long *off, int nlat, int nlath,
                               int ncsp, int ntp1, int nj8, int t, int tref, unsigned char *base) {
    const int m = blockIdx.x;
    const int K = ntp1 - m;
    unsigned char *blk = base + off[m * 4 + t];
    const double *q = qref + (size_t)tref * ncsp * nlat;
    size_t poff = 0;
    for (int p = 0; p < 2; p++) {
        const int Kq = kpar(K, p), Kp = pad16(Kq);
        if (Kq == 0) break;
        const size_t tile = (size_t)nj8 * Kp * 2;
        for (int idx = threadIdx.x; idx < nj8 * Kp; idx += blockDim.x) {
            const int r = idx / Kp, k = idx % Kp;
            double v = 0.0;
            if (r < nlath && k < Kq) v = q[(size_t)r * ncsp + woff[m] + 2 * k + p];
            __nv_bfloat16 h, mm, l;
            split3d(v, h, mm, l);
            const uint32_t o = tc::kmajor_off(r, k, Kp);
            *reinterpret_cast<__nv_bfloat16 *>(blk + poff + o) = h;
            *reinterpret_cast<__nv_bfloat16 *>(blk + poff + tile + o) = mm;
            *reinterpret_cast<__nv_bfloat16 *>(blk + poff + 2 * tile + o) = l;
        }
        poff += 3 * tile;
    }
}

// forward block (m, t) = [p][j-chunk][split][rows pad8(Kq)][chunk width] (K-major, K = j)
__global__ void k_build_tc_fwd(const double *qref, const int *woff, const long long *off, int nlat, int nlath,
                               int ncsp, int ntp1, int njc, int t, int tref, unsigned char *base) {
    const int m = blockIdx.x;
    const int K = ntp1 - m;
    unsigned char *blk = base + off[m * 4 + t];
    const double *q = qref + (size_t)tref * ncsp * nlat;
    size_t poff = 0;
    for (int p = 0; p < 2; p++) {
        const int Kq = kpar(K, p), R = pad8(Kq);
        if (Kq == 0) break;
        for (int j0 = 0; j0 < njc; j0 += 32) {
            const int jw = min(32, njc - j0);
            const size_t tile = (size_t)R * jw * 2;
            for (int idx = threadIdx.x; idx < R * jw; idx += blockDim.x) {
                const int r = idx / jw, jj = idx % jw, j = j0 + jj;
                double v = 0.0;
                if (r < Kq && j < nlath) v = q[(size_t)j * ncsp + woff[m] + 2 * r + p];
                __nv_bfloat16 h, mm, l;
                split3d(v, h, mm, l);
                const uint32_t o = tc::kmajor_off(r, jj, jw);
                *reinterpret_cast<__nv_bfloat16 *>(blk + poff + o) = h;
                *reinterpret_cast<__nv_bfloat16 *>(blk + poff + tile + o) = mm;
                *reinterpret_cast<__nv_bfloat16 *>(blk + poff + 2 * tile + o) = l;
            }
            poff += 3 * tile;
        }
    }
}

static exotx_status tc_tables(exotx_plan p, TcTables **out) {
    if (p->tc) { *out = p->tc; return EXOTX_OK; }
    if (p->nlath > 128) return EXOTX_BAD_DIM;  // inverse M tile = 128 latitude pairs
    TcTables *T = new TcTables();
    T->nj8 = pad8(p->nlath);
    T->njc = pad16(p->nlath);
    const int ntp1 = p->ntp1;
    T->inv_off.assign(ntp1 * 4, 0);
    T->inv_bytes.assign(ntp1 * 4, 0);
    T->fwd_off.assign(ntp1 * 4, 0);
    T->fwd_bytes.assign(ntp1 * 4, 0);
    long long io = 0, fo = 0;
    for (int m = 0; m < ntp1; m++) {
        const int K = ntp1 - m;
        for (int t = 0; t < 4; t++) {
            long long bi = 0, bf = 0;
            for (int q = 0; q < 2; q++) {
                const int Kq = kpar(K, q);
                if (!Kq) continue;
                bi += 3LL * T->nj8 * pad16(Kq) * 2;
                bf += 3LL * pad8(Kq) * T->njc * 2;
            }
            T->inv_off[m * 4 + t] = io; T->inv_bytes[m * 4 + t] = (int)bi; io += bi;
            T->fwd_off[m * 4 + t] = fo; T->fwd_bytes[m * 4 + t] = (int)bf; fo += bf;
        }
    }
    bool ok = cudaMalloc(&T->inv, io) == cudaSuccess && cudaMalloc(&T->fwd, fo) == cudaSuccess &&
              cudaMalloc(&T->d_inv_off, sizeof(long long) * ntp1 * 4) == cudaSuccess &&
              cudaMalloc(&T->d_fwd_off, sizeof(long long) * ntp1 * 4) == cudaSuccess;
    ok = ok && cudaMemcpy(T->d_inv_off, T->inv_off.data(), sizeof(long long) * ntp1 * 4, cudaMemcpyHostToDevice) ==
                   cudaSuccess &&
         cudaMemcpy(T->d_fwd_off, T->fwd_off.data(), sizeof(long long) * ntp1 * 4, cudaMemcpyHostToDevice) ==
             cudaSuccess;
    if (!ok) { delete T; return EXOTX_NO_MEM; }
    for (int t = 0; t < 4; t++) {
        k_build_tc_inv<<<ntp1, 256>>>(p->d_qref, p->d_woff, T->d_inv_off, p->nlat, p->nlath, p->ncsp, ntp1, T->nj8,
                                      t, kInvRef[t], T->inv);
        note_launch();
        k_build_tc_fwd<<<ntp1, 256>>>(p->d_qref, p->d_woff, T->d_fwd_off, p->nlat, p->nlath, p->ncsp, ntp1, T->njc,
                                      t, kFwdRef[t], T->fwd);
        note_launch();
    }
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        delete T;
        return EXOTX_CUDA_ERR;
    }
    p->tc = T;
    *out = T;
    return EXOTX_OK;
}

void tc_free(exotx_plan p) {
    delete p->tc;
    p->tc = nullptr;
}
exotx_status tc_available() { return EXOTX_OK; }

// ------------------------------------------------------------------ jobs
// inverse groups: 0 = qi on sd,st,sz,sq,sp; 1 = qj on sp; 2 = qu,qv on (D,Z)
// forward groups: 0 = qc,qe,qm,qq on the mktend/qtend/fc2sp inputs (one level slab)
// job = (m, group, first column, number of columns)
static constexpr int FWD_LEV_TILE = 4;  // levels per forward job (shared-memory bound)
static constexpr size_t TC_SMEM_MAX = 227 * 1024;

static size_t inv_smem(int nj8, int K, int ncp);

// inverse column tiles: as wide as shared memory (both parities of one table
// plus the staged columns) and TMEM (tables x parities x columns <= 256) allow
static void inv_tiles(int nj8, int ntp1, int *nc_qi, int *nc_uv) {
    int a = 128, b = 64;
    while (a > 16 && inv_smem(nj8, ntp1, a) > TC_SMEM_MAX) a -= 16;
    while (b > 16 && inv_smem(nj8, ntp1, b) > TC_SMEM_MAX) b -= 16;
    *nc_qi = a;
    *nc_uv = b;
}

static exotx_status tc_jobs(exotx_plan p, TcTables *T, int dir, int L, int ninst, const int4 **d, int *njobs) {
    for (auto &j : T->jobs)
        if (j.dir == dir && j.nlev == L && j.ninst == ninst) { *d = j.d; *njobs = j.njobs; return EXOTX_OK; }
    std::vector<int4> v;
    int INV_NC_QI, INV_NC_UV;
    inv_tiles(T->nj8, p->ntp1, &INV_NC_QI, &INV_NC_UV);
    for (int m = 0; m < p->ntp1; m++) {
        if (dir == 0) {
            const int n0 = ninst * (4 * L + 1) * 2, n1 = ninst * 2, n2 = ninst * L * 4;
            for (int c = 0; c < n0; c += INV_NC_QI) v.push_back(make_int4(m, 0, c, std::min(INV_NC_QI, n0 - c)));
            for (int c = 0; c < n1; c += INV_NC_QI) v.push_back(make_int4(m, 1, c, std::min(INV_NC_QI, n1 - c)));
            for (int c = 0; c < n2; c += INV_NC_UV) v.push_back(make_int4(m, 2, c, std::min(INV_NC_UV, n2 - c)));
        } else {
            // slabs of FWD_LEV_TILE levels of one instance; the level-independent gvpp rides with slab 0
            for (int i = 0; i < ninst; i++)
                for (int l0 = 0; l0 < L; l0 += FWD_LEV_TILE)
                    v.push_back(make_int4(m, i, l0, std::min(FWD_LEV_TILE, L - l0)));
        }
    }
    TcTables::Jobs J;
    J.dir = dir; J.nlev = L; J.ninst = ninst; J.njobs = (int)v.size();
    if (cudaMalloc(&J.d, sizeof(int4) * v.size()) != cudaSuccess) return EXOTX_NO_MEM;
    if (cudaMemcpy(J.d, v.data(), sizeof(int4) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess) return EXOTX_CUDA_ERR;
    T->jobs.push_back(J);
    *d = J.d;
    *njobs = J.njobs;
    return EXOTX_OK;
}

// ------------------------------------------------------------ inverse
struct TcInvArgs {
    const unsigned char *tab;
    const long long *off;
    const int *woff;
    const float *spin;      // [inst][4L+1][NRSP]
    const float *filt;      // skspgp
    float2 *W;              // [m][row], row = (inst*(6L+3) + field)*nlat + lat
    long long nrows;
    const int4 *jobs;
    int L, nlat, nlath, nj8, ntp1, nrsp;
    float plavor;
};

// spectral input column -> value (already filtered); returns false for pads
__device__ __forceinline__ float inv_input(const TcInvArgs &A, int group, int gc, int m, int k) {
    const int L = A.L, nf = 4 * L + 1;
    int inst, f, ri;
    bool zvort = false;
    if (group == 0) { inst = gc / (2 * nf); f = (gc >> 1) % nf; ri = gc & 1; }
    else if (group == 1) { inst = gc >> 1; f = 4 * L; ri = gc & 1; }
    else {
        inst = gc / (4 * L);
        const int l = (gc % (4 * L)) >> 2, q = gc & 3;
        zvort = q >= 2;
        f = zvort ? 2 * L + l : l;
        ri = q & 1;
    }
    const int w = A.woff[m] + k;
    float x = A.spin[((size_t)inst * nf + f) * A.nrsp + 2 * w + ri];
    if (zvort && m == 0 && k == 1 && ri == 0) x -= A.plavor;  // dv2uv, legmod.f90:332
    return x * A.filt[m + k];
}

__global__ void __launch_bounds__(TCT) k_tc_inverse(TcInvArgs A) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int4 jb = A.jobs[blockIdx.x];
    const int m = jb.x, group = jb.y, c0 = jb.z, nc = jb.w;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int K = A.ntp1 - m;
    const int Kq[2] = {kpar(K, 0), kpar(K, 1)};
    const int Kp[2] = {pad16(Kq[0]), pad16(Kq[1])};
    const int ncp = pad16(nc);
    const int ntab = group == 2 ? 2 : 1;
    const int nj8 = A.nj8;
    // shared layout: [table tiles p0,p1 x 3 splits][data p0,p1 x 3 splits][overrun][bars]
    const size_t ttile[2] = {(size_t)nj8 * Kp[0] * 2, (size_t)nj8 * Kp[1] * 2};
    const size_t tbytes = 3 * (ttile[0] + ttile[1]);
    const size_t dtile[2] = {(size_t)ncp * Kp[0] * 2, (size_t)ncp * Kp[1] * 2};
    unsigned char *tab = sm;
    unsigned char *dat = sm + tbytes;
    unsigned char *tail = dat + 3 * (dtile[0] + dtile[1]) + (size_t)(128 - nj8) * 64 * 2 + 128;
    uint64_t *bar_tma = reinterpret_cast<uint64_t *>((reinterpret_cast<uintptr_t>(tail) + 15) & ~(uintptr_t)15);
    uint64_t *bar_mma = bar_tma + 1;
    uint64_t *bar_done = bar_tma + 2;
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar_tma + 3);
    if (warp == 0) tc::tmem_alloc(slot, 512);
    if (tid == 0) {
        tc::mbar_init(bar_tma, 1);
        tc::mbar_init(bar_mma, 1);
        tc::mbar_init(bar_done, 1);
        tc::mbar_fence_init();
    }
    // stage the spectral columns of both parities, split into three BF16 terms
    size_t doff = 0;
    for (int p = 0; p < 2; p++) {
        if (!Kq[p]) break;
        const int kp = Kp[p];
        for (int idx = tid; idx < ncp * kp; idx += TCT) {
            const int c = idx / kp, k = idx % kp;
            float x = 0.f;
            if (c < nc && k < Kq[p]) x = inv_input(A, group, c0 + c, m, 2 * k + p);
            __nv_bfloat16 h, mm, l;
            tc::split3(x, h, mm, l);
            const uint32_t o = tc::kmajor_off(c, k, kp);
            *reinterpret_cast<__nv_bfloat16 *>(dat + doff + o) = h;
            *reinterpret_cast<__nv_bfloat16 *>(dat + doff + dtile[p] + o) = mm;
            *reinterpret_cast<__nv_bfloat16 *>(dat + doff + 2 * dtile[p] + o) = l;
        }
        doff += 3 * dtile[p];
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    bool ok = true;
    if (tid == 0) {
        const uint32_t idesc = tc::idesc_bf16(128, ncp);
        for (int ti = 0; ti < ntab && ok; ti++) {
            const int t = group == 0 ? 0 : (group == 1 ? 1 : 2 + ti);
            if (ti > 0) ok = tc::mbar_wait(bar_mma, (ti - 1) & 1);  // table buffer free again
            if (!ok) break;
            const uint32_t bytes = (uint32_t)tbytes;
            tc::mbar_arrive_expect_tx(bar_tma, bytes);
            tc::bulk_g2s(tab, A.tab + A.off[m * 4 + t], bytes, bar_tma);
            ok = tc::mbar_wait(bar_tma, ti & 1);
            if (!ok) break;
            tc::fence_after_sync();
            size_t to = 0, dd = 0;
            for (int p = 0; p < 2; p++) {
                if (!Kq[p]) break;
                // hi*hi products and the five smaller correction products go to
                // separate accumulators (the tensor-core adder truncates; keeping the
                // large term's chain short bounds that error), summed in the epilogue
                const uint32_t dm = tmem + (uint32_t)(((ti * 2 + p) * 2 + 0) * ncp);
                const uint32_t dc = tmem + (uint32_t)(((ti * 2 + p) * 2 + 1) * ncp);
                const uint32_t sbo = (uint32_t)(Kp[p] / 8) * 128;
                bool accm = false, accc = false;
                for (int kc = 0; kc < Kp[p] / 16; kc++)
                    for (int pr = 0; pr < 6; pr++) {
                        const unsigned char *a = tab + to + c_pair_a[pr] * ttile[p] + kc * 256;
                        const unsigned char *b = dat + dd + c_pair_b[pr] * dtile[p] + kc * 256;
                        const bool main = (pr == 0);
                        tc::mma_bf16(main ? dm : dc, tc::smem_desc(a, 128, sbo), tc::smem_desc(b, 128, sbo), idesc,
                                     main ? accm : accc);
                        if (main) accm = true; else accc = true;
                    }
                to += 3 * ttile[p];
                dd += 3 * dtile[p];
            }
            // intermediate batches recycle the table buffer; the last one releases the epilogue
            tc::mma_commit(ti == ntab - 1 ? bar_done : bar_mma);
        }
        if (!ok) atomicExch(&g_tc_error, 1);
    }
    __syncthreads();
    // every thread waits for the last MMA batch (single-phase barrier, bounded)
    ok = tc::mbar_wait(bar_done, 0);
    if (!ok && (tid & 31) == 0) atomicExch(&g_tc_error, 2);
    tc::fence_after_sync();
    if (ok) {
        const int j = tid;  // TMEM lane = latitude pair
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        const int L = A.L, nfo = 6 * L + 3, nf = 4 * L + 1;
        const bool has1 = Kq[1] > 0;
        for (int cc = 0; cc < ncp; cc += 16) {
            float d[4][16];
            for (int r = 0; r < 2 * ntab; r++) {
                const int ti = r >> 1, p = r & 1;
                if (p == 1 && !has1) {
#pragma unroll
                    for (int i = 0; i < 16; i++) d[r][i] = 0.f;
                } else {
                    float e[16];
                    tc::tmem_ld16(tmem + lane_addr + (uint32_t)(((ti * 2 + p) * 2 + 0) * ncp + cc), d[r]);
                    tc::tmem_ld16(tmem + lane_addr + (uint32_t)(((ti * 2 + p) * 2 + 1) * ncp + cc), e);
#pragma unroll
                    for (int i = 0; i < 16; i++) d[r][i] += e[i];
                }
            }
            if (j >= A.nlath) continue;
            const int latN = j, latS = A.nlat - 1 - j;
            if (group < 2) {
                // P-type qi: N = D0 + D1, S = D0 - D1; Q-type qj: S = D1 - D0
                const float ss = group == 0 ? 1.f : -1.f;
                for (int i = 0; i < 16 && cc + i < nc; i += 2) {
                    const int gc = c0 + cc + i;
                    int inst, f;
                    if (group == 0) { inst = gc / (2 * nf); f = (gc >> 1) % nf; }
                    else { inst = gc >> 1; f = 4 * L; }
                    float2 vn = make_float2(d[0][i] + d[1][i], d[0][i + 1] + d[1][i + 1]);
                    float2 vs = make_float2(ss * (d[0][i] - d[1][i]), ss * (d[0][i + 1] - d[1][i + 1]));
                    int F;
                    if (group == 1) F = 6 * L;                    // gpj
                    else if (f < L) F = 3 * L + f;                // sd -> gd
                    else if (f < 2 * L) F = f + L;                // st -> gt
                    else if (f < 4 * L) F = f + 2 * L;            // sz -> gz, sq -> gq
                    else F = 6 * L + 2;                           // sp -> gp
                    const size_t rb = (size_t)m * A.nrows + (size_t)(inst * nfo + F) * A.nlat;
                    A.W[rb + latN] = vn;
                    A.W[rb + latS] = vs;
                    if (group == 0 && f == 4 * L) {               // gpmt = i*m*gp
                        const float fm = (float)m;
                        const size_t rt = (size_t)m * A.nrows + (size_t)(inst * nfo + 6 * L + 1) * A.nlat;
                        A.W[rt + latN] = make_float2(-fm * vn.y, fm * vn.x);
                        A.W[rt + latS] = make_float2(-fm * vs.y, fm * vs.x);
                    }
                }
            } else {
                // dv2uv: u = qv*Z - i*qu*D, v = -i*qu*Z - qv*D; qu P-type, qv Q-type
                // d[0]=qu p0, d[1]=qu p1, d[2]=qv p0, d[3]=qv p1; columns Dr,Di,Zr,Zi per level
                for (int i = 0; i < 16 && cc + i < nc; i += 4) {
                    const int gc = c0 + cc + i;
                    const int inst = gc / (4 * L), l = (gc % (4 * L)) >> 2;
                    const int Dr = i, Di = i + 1, Zr = i + 2, Zi = i + 3;
                    const float urs = d[0][Di] + d[3][Zr], ura = d[1][Di] + d[2][Zr];
                    const float uis = -d[0][Dr] + d[3][Zi], uia = -d[1][Dr] + d[2][Zi];
                    const float vrs = d[0][Zi] - d[3][Dr], vra = d[1][Zi] - d[2][Dr];
                    const float vis = -d[0][Zr] - d[3][Di], via = -d[1][Zr] - d[2][Di];
                    const size_t ru = (size_t)m * A.nrows + (size_t)(inst * nfo + l) * A.nlat;
                    const size_t rv = (size_t)m * A.nrows + (size_t)(inst * nfo + L + l) * A.nlat;
                    A.W[ru + latN] = make_float2(urs + ura, uis + uia);
                    A.W[ru + latS] = make_float2(urs - ura, uis - uia);
                    A.W[rv + latN] = make_float2(vrs + vra, vis + via);
                    A.W[rv + latS] = make_float2(vrs - vra, vis - via);
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

static size_t inv_smem(int nj8, int K, int ncp) {
    const int Kp0 = pad16(kpar(K, 0)), Kp1 = pad16(kpar(K, 1));
    return 3 * (size_t)nj8 * (Kp0 + Kp1) * 2 + 3 * (size_t)ncp * (Kp0 + Kp1) * 2 + (size_t)(128 - nj8) * 64 * 2 +
           128 + 80;
}

// ------------------------------------------------------------ forward
struct TcFwdArgs {
    const unsigned char *tab;
    const long long *off;
    const int *woff;
    const float2 *W;        // [m][row], row = (inst*(9L+1) + field)*nlat + lat
    long long nrows;
    const float *filt;      // skgpsp
    float *spout;           // [inst][4L+1][NRSP]
    const int4 *jobs;
    int L, nlat, nlath, njc, ntp1, nrsp;
};

// Forward columns of one job (levels l0..l0+nl-1 of one instance), per table:
//   qc: tn, qn (per level) [+ gvpp once]   qe: fv, vt, fu, vq   qm: fu, ut, fv, uq   qq: ke
// each column is (field, level, re|im).  Input field indices in gpin order:
// gtn 0, gqn 1, gut 2, gvt 3, guz 4, gvz 5, gke 6, gvpp 7 (single), guq 8, gvq 9
// mktend call: tn=gtn, fu=gvz, fv=guz, ke=gke, ut=gut, vt=gvt; qtend: qn=gqn, uq=guq, vq=gvq
__device__ __constant__ int c_fwd_nf[4] = {2, 4, 4, 1};
__device__ __constant__ int c_fwd_fields[4][4] = {{0, 1, -1, -1}, {4, 3, 5, 9}, {5, 2, 4, 8}, {6, -1, -1, -1}};

__device__ __forceinline__ long long fwd_row(int L, int inst, int kind, int l) {
    // gpin field -> row base (without lat)
    const int nfi = 9 * L + 1;
    int F;
    if (kind == 7) F = 7 * L;
    else if (kind < 7) F = kind * L + l;
    else F = 7 * L + 1 + (kind - 8) * L + l;
    return (long long)inst * nfi + F;
}

__global__ void __launch_bounds__(TCT) k_tc_forward(TcFwdArgs A) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int4 jb = A.jobs[blockIdx.x];
    const int m = jb.x, inst = jb.y, l0 = jb.z, nl = jb.w;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int K = A.ntp1 - m;
    const int Kq[2] = {kpar(K, 0), kpar(K, 1)};
    const int R[2] = {pad8(Kq[0]), pad8(Kq[1])};
    const int njc = A.njc, L = A.L, nlat = A.nlat;
    const bool with_vpp = (l0 == 0);
    // columns per table: nf fields x nl levels x 2 (+2 for gvpp on qc)
    int ncol[4], ncp[4], colbase[4];
    int tot = 0;
    for (int t = 0; t < 4; t++) {
        ncol[t] = c_fwd_nf[t] * nl * 2 + ((t == 0 && with_vpp) ? 2 : 0);
        ncp[t] = pad16(ncol[t]);
        colbase[t] = tot;
        tot += 4 * ncp[t];  // 2 parities x (main, correction) accumulators
    }
    // shared: [table block (both parities, all j-chunks, 3 splits)][data: per table, per sel(S/D), 3 splits, ncp x njc]
    size_t tblk = 0;
    for (int p = 0; p < 2; p++) if (Kq[p]) tblk += 3 * (size_t)R[p] * njc * 2;
    // rows >= R of the M=128 table tiles read past the block: keep a margin
    // before the data so those reads (whose TMEM lanes are never used) stay in bounds
    unsigned char *tab = sm;
    unsigned char *dat = sm + tblk + 128 * 32 * 2;
    size_t dbytes = 0;
    size_t doffs[4];
    for (int t = 0; t < 4; t++) { doffs[t] = dbytes; dbytes += 2 * 3 * (size_t)ncp[t] * njc * 2; }
    unsigned char *tail = dat + dbytes;
    uint64_t *bar_tma = reinterpret_cast<uint64_t *>((reinterpret_cast<uintptr_t>(tail) + 15) & ~(uintptr_t)15);
    uint64_t *bar_mma = bar_tma + 1;
    uint64_t *bar_done = bar_tma + 2;
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar_tma + 3);
    if (warp == 0) tc::tmem_alloc(slot, 512);
    if (tid == 0) {
        tc::mbar_init(bar_tma, 1);
        tc::mbar_init(bar_mma, 1);
        tc::mbar_init(bar_done, 1);
        tc::mbar_fence_init();
    }
    // stage folded Fourier columns: for each table, S (= N+S) and D (= N-S) versions
    for (int t = 0; t < 4; t++) {
        const int nf = c_fwd_nf[t];
        const size_t dt = (size_t)ncp[t] * njc * 2;  // one split tile
        for (int idx = tid; idx < ncp[t] * njc; idx += TCT) {
            const int c = idx / njc, j = idx % njc;
            float2 vn = make_float2(0.f, 0.f), vs = vn;
            int ri = c & 1;
            if (c < ncol[t] && j < A.nlath) {
                long long rb;
                if (t == 0 && with_vpp && c >= nf * nl * 2) rb = fwd_row(L, inst, 7, 0);
                else {
                    const int fl = c >> 1, fi = fl / nl, l = l0 + fl % nl;
                    rb = fwd_row(L, inst, c_fwd_fields[t][fi], l);
                }
                const size_t base = (size_t)m * A.nrows + (size_t)rb * nlat;
                vn = A.W[base + j];
                vs = A.W[base + nlat - 1 - j];
            }
            const float xn = ri ? vn.y : vn.x, xs = ri ? vs.y : vs.x;
            const float S = xn + xs, D = xn - xs;
            const uint32_t o = tc::kmajor_off(c, j, njc);
            __nv_bfloat16 h, mm, l;
            tc::split3(S, h, mm, l);
            unsigned char *bS = dat + doffs[t];
            *reinterpret_cast<__nv_bfloat16 *>(bS + o) = h;
            *reinterpret_cast<__nv_bfloat16 *>(bS + dt + o) = mm;
            *reinterpret_cast<__nv_bfloat16 *>(bS + 2 * dt + o) = l;
            tc::split3(D, h, mm, l);
            unsigned char *bD = bS + 3 * dt;
            *reinterpret_cast<__nv_bfloat16 *>(bD + o) = h;
            *reinterpret_cast<__nv_bfloat16 *>(bD + dt + o) = mm;
            *reinterpret_cast<__nv_bfloat16 *>(bD + 2 * dt + o) = l;
        }
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    bool ok = true;
    if (tid == 0) {
        for (int t = 0; t < 4 && ok; t++) {
            if (t > 0) ok = tc::mbar_wait(bar_mma, (t - 1) & 1);
            if (!ok) break;
            tc::mbar_arrive_expect_tx(bar_tma, (uint32_t)tblk);
            tc::bulk_g2s(tab, A.tab + A.off[m * 4 + t], (uint32_t)tblk, bar_tma);
            ok = tc::mbar_wait(bar_tma, t & 1);
            if (!ok) break;
            tc::fence_after_sync();
            const uint32_t idesc = tc::idesc_bf16(128, ncp[t]);
            const size_t dt = (size_t)ncp[t] * njc * 2;
            size_t to = 0;
            for (int p = 0; p < 2; p++) {
                if (!Kq[p]) break;
                // P-type (qc, qm, qq) use N+S on even n-m and N-S on odd; Q-type (qe) the reverse
                const bool ptype = (t != 1);
                const int sel = (ptype ? p : 1 - p);  // 0 -> S, 1 -> D
                const unsigned char *dsel = dat + doffs[t] + (size_t)sel * 3 * dt;
                const uint32_t dm = tmem + (uint32_t)(colbase[t] + (2 * p + 0) * ncp[t]);
                const uint32_t dc = tmem + (uint32_t)(colbase[t] + (2 * p + 1) * ncp[t]);
                bool accm = false, accc = false;
                size_t jo = 0;
                for (int j0 = 0; j0 < njc; j0 += 32) {
                    const int jw = njc - j0 < 32 ? njc - j0 : 32;
                    const size_t tt = (size_t)R[p] * jw * 2;
                    for (int kc = 0; kc < jw / 16; kc++)
                        for (int pr = 0; pr < 6; pr++) {
                            const unsigned char *a = tab + to + jo + c_pair_a[pr] * tt + kc * 256;
                            const unsigned char *b = dsel + c_pair_b[pr] * dt + (size_t)(j0 / 8) * 128 + kc * 256;
                            const bool main = (pr == 0);
                            tc::mma_bf16(main ? dm : dc, tc::smem_desc(a, 128, (uint32_t)(jw / 8) * 128),
                                         tc::smem_desc(b, 128, (uint32_t)(njc / 8) * 128), idesc,
                                         main ? accm : accc);
                            if (main) accm = true; else accc = true;
                        }
                    jo += 3 * tt;
                }
                to += jo;
            }
            tc::mma_commit(t == 3 ? bar_done : bar_mma);
        }
        if (!ok) atomicExch(&g_tc_error, 3);
    }
    __syncthreads();
    ok = tc::mbar_wait(bar_done, 0);
    if (!ok && (tid & 31) == 0) atomicExch(&g_tc_error, 4);
    tc::fence_after_sync();
    if (ok) {
        // TMEM lane = mode index k' of each parity; epilogue per parity
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        const int kk = tid;
        const int nfo = 4 * L + 1;
        for (int p = 0; p < 2; p++) {
            if (!Kq[p]) break;
            const bool valid = kk < Kq[p];
            const int k = 2 * kk + p;               // n - m
            const float fl = valid ? A.filt[m + k] : 0.f;
            const size_t wo = 2 * (size_t)(A.woff[m] + k);
            // level loop over the columns of this job
            for (int li = 0; li < nl; li++) {
                // gather the products needed for level li: per table, column (field fi, level li, ri)
                // qc: tn(fi0), qn(fi1); qe: fv(0), vt(1), fu(2), vq(3); qm: fu(0), ut(1), fv(2), uq(3); qq: ke(0)
                float v[4][4][2];
                for (int t = 0; t < 4; t++) {
                    const int nf = c_fwd_nf[t];
                    for (int fi = 0; fi < nf; fi++) {
                        const int c = (fi * nl + li) * 2;
                        float x[16], y[16];
                        const int cb = c & ~15;
                        tc::tmem_ld16(tmem + lane_addr + (uint32_t)(colbase[t] + (2 * p) * ncp[t] + cb), x);
                        tc::tmem_ld16(tmem + lane_addr + (uint32_t)(colbase[t] + (2 * p + 1) * ncp[t] + cb), y);
                        v[t][fi][0] = x[c - cb] + y[c - cb];
                        v[t][fi][1] = x[c - cb + 1] + y[c - cb + 1];
                    }
                }
                if (!valid) continue;
                const int l = l0 + li;
                float *sd = A.spout + ((size_t)inst * nfo + l) * A.nrsp + wo;
                float *st = A.spout + ((size_t)inst * nfo + L + l) * A.nrsp + wo;
                float *sz = A.spout + ((size_t)inst * nfo + 2 * L + l) * A.nrsp + wo;
                float *sq = A.spout + ((size_t)inst * nfo + 3 * L + l) * A.nrsp + wo;
                // d = qq*ke - qe*fv + i*qm*fu
                sd[0] = (v[3][0][0] - v[1][0][0] - v[2][0][1]) * fl;
                sd[1] = (v[3][0][1] - v[1][0][1] + v[2][0][0]) * fl;
                // t = qe*vt + qc*tn - i*qm*ut
                st[0] = (v[1][1][0] + v[0][0][0] + v[2][1][1]) * fl;
                st[1] = (v[1][1][1] + v[0][0][1] - v[2][1][0]) * fl;
                // z = qe*fu + i*qm*fv
                sz[0] = (v[1][2][0] - v[2][2][1]) * fl;
                sz[1] = (v[1][2][1] + v[2][2][0]) * fl;
                // q = qe*vq + qc*qn - i*qm*uq
                sq[0] = (v[1][3][0] + v[0][1][0] + v[2][3][1]) * fl;
                sq[1] = (v[1][3][1] + v[0][1][1] - v[2][3][0]) * fl;
            }
            if (with_vpp) {
                const int c = c_fwd_nf[0] * nl * 2;
                const int cb = c & ~15;
                float x[16], y[16];
                tc::tmem_ld16(tmem + lane_addr + (uint32_t)(colbase[0] + (2 * p) * ncp[0] + cb), x);
                tc::tmem_ld16(tmem + lane_addr + (uint32_t)(colbase[0] + (2 * p + 1) * ncp[0] + cb), y);
                if (valid) {
                    float *sp = A.spout + ((size_t)inst * nfo + 4 * L) * A.nrsp + wo;
                    sp[0] = (x[c - cb] + y[c - cb]) * fl;
                    sp[1] = (x[c - cb + 1] + y[c - cb + 1]) * fl;
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

static size_t fwd_smem(int K, int njc, int nl, bool with_vpp) {
    size_t tblk = 0;
    for (int p = 0; p < 2; p++) {
        const int Kq = kpar(K, p);
        if (Kq) tblk += 3 * (size_t)pad8(Kq) * njc * 2;
    }
    size_t d = 0;
    const int nf[4] = {2, 4, 4, 1};
    for (int t = 0; t < 4; t++) {
        int ncol = nf[t] * nl * 2 + ((t == 0 && with_vpp) ? 2 : 0);
        d += 2 * 3 * (size_t)pad16(ncol) * njc * 2;
    }
    return tblk + 128 * 32 * 2 + d + 80;
}

// ---------------------------------------------------------- set drivers
exotx_status tc_inverse_batch(exotx_plan p, const float *spin, float *gpout, int L, int ninst, cudaStream_t s) {
    TcTables *T;
    EXOTX_TRY(tc_tables(p, &T));
    const long long nrsp = 2LL * p->ncsp, nhor = (long long)p->nlat * p->nlon;
    const int nfo = 6 * L + 3;
    // chunk instances so the m-major Fourier intermediate stays L2-resident (<= 48 MB)
    const size_t per_inst = (size_t)nfo * p->nlat * p->ntp1 * sizeof(float2);
    int chunk = (int)std::max<size_t>(1, (48u << 20) / per_inst);
    chunk = std::min(chunk, ninst);
    EXOTX_TRY(ensure_work(p, per_inst * chunk));
    const int4 *jobs;
    int njobs;
    EXOTX_TRY(tc_jobs(p, T, 0, L, chunk, &jobs, &njobs));
    int nc_qi, nc_uv;
    inv_tiles(T->nj8, p->ntp1, &nc_qi, &nc_uv);
    size_t smem = std::max(inv_smem(T->nj8, p->ntp1, nc_qi), inv_smem(T->nj8, p->ntp1, nc_uv));
    if (smem > TC_SMEM_MAX) return EXOTX_BAD_DIM;
    EXOTX_CUDA(cudaFuncSetAttribute(k_tc_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    for (int i0 = 0; i0 < ninst; i0 += chunk) {
        const int ni = std::min(chunk, ninst - i0);
        const int4 *jl = jobs;
        int nj = njobs;
        if (ni != chunk) EXOTX_TRY(tc_jobs(p, T, 0, L, ni, &jl, &nj));
        TcInvArgs A;
        A.tab = T->inv; A.off = T->d_inv_off; A.woff = p->d_woff;
        A.spin = spin + (size_t)i0 * (4 * L + 1) * nrsp;
        A.filt = p->d_fs32;
        A.W = (float2 *)p->d_work;
        A.nrows = (long long)ni * nfo * p->nlat;
        A.jobs = jl;
        A.L = L; A.nlat = p->nlat; A.nlath = p->nlath; A.nj8 = T->nj8; A.ntp1 = p->ntp1; A.nrsp = (int)nrsp;
        A.plavor = (float)p->desc.plavor;
        k_tc_inverse<<<nj, TCT, smem, s>>>(A);
        EXOTX_CHECK_LAUNCH();
        EXOTX_TRY(fft_inverse_l<float>((const float *)p->d_work, gpout + (size_t)i0 * nfo * nhor, p->nlon, A.nrows,
                                       p->ntp1, 1, A.nrows, s));
    }
    return EXOTX_OK;
}

exotx_status tc_forward_batch(exotx_plan p, const float *gpin, float *spout, int L, int ninst, cudaStream_t s) {
    TcTables *T;
    EXOTX_TRY(tc_tables(p, &T));
    const long long nrsp = 2LL * p->ncsp, nhor = (long long)p->nlat * p->nlon;
    const int nfi = 9 * L + 1;
    const size_t per_inst = (size_t)nfi * p->nlat * p->ntp1 * sizeof(float2);
    int chunk = (int)std::max<size_t>(1, (48u << 20) / per_inst);
    chunk = std::min(chunk, ninst);
    EXOTX_TRY(ensure_work(p, per_inst * chunk));
    const int4 *jobs;
    int njobs;
    EXOTX_TRY(tc_jobs(p, T, 1, L, chunk, &jobs, &njobs));
    size_t smem = fwd_smem(p->ntp1, T->njc, std::min(FWD_LEV_TILE, L), true);
    if (smem > TC_SMEM_MAX) return EXOTX_BAD_DIM;
    EXOTX_CUDA(cudaFuncSetAttribute(k_tc_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    for (int i0 = 0; i0 < ninst; i0 += chunk) {
        const int ni = std::min(chunk, ninst - i0);
        const int4 *jl = jobs;
        int nj = njobs;
        if (ni != chunk) EXOTX_TRY(tc_jobs(p, T, 1, L, ni, &jl, &nj));
        const long long nrows = (long long)ni * nfi * p->nlat;
        EXOTX_TRY(fft_forward_l<float>(gpin + (size_t)i0 * nfi * nhor, (float *)p->d_work, p->nlon, nrows, p->ntp1,
                                       1, nrows, s));
        TcFwdArgs A;
        A.tab = T->fwd; A.off = T->d_fwd_off; A.woff = p->d_woff;
        A.W = (const float2 *)p->d_work;
        A.nrows = nrows;
        A.filt = p->d_fg32;
        A.spout = spout + (size_t)i0 * (4 * L + 1) * nrsp;
        A.jobs = jl;
        A.L = L; A.nlat = p->nlat; A.nlath = p->nlath; A.njc = T->njc; A.ntp1 = p->ntp1; A.nrsp = (int)nrsp;
        k_tc_forward<<<nj, TCT, smem, s>>>(A);
        EXOTX_CHECK_LAUNCH();
    }
    return EXOTX_OK;
}

exotx_status tc_inverse_set(exotx_plan p, const float *spin, float *gpout, int L, cudaStream_t s) {
    return tc_inverse_batch(p, spin, gpout, L, 1, s);
}
exotx_status tc_forward_set(exotx_plan p, const float *gpin, float *spout, int L, cudaStream_t s) {
    return tc_forward_batch(p, gpin, spout, L, 1, s);
}

exotx_status tc_error_reset(cudaStream_t s) {
    int zero = 0;
    EXOTX_CUDA(cudaMemcpyToSymbolAsync(g_tc_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s));
    return EXOTX_OK;
}
exotx_status tc_error_read(int *err, cudaStream_t s) {
    EXOTX_CUDA(cudaMemcpyFromSymbolAsync(err, g_tc_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    EXOTX_CUDA(cudaStreamSynchronize(s));
    return EXOTX_OK;
}
}  // namespace exotx

using namespace exotx;

EXOTX_API exotx_status exotx_tc_selftest(const float *A, const float *B, float *C, int N, int K, int nprod,
                                         exotx_stream s) {
    if (!A || !B || !C || N < 16 || N > 256 || (N % 16) || K < 16 || K > 64 || (K % 16)) return EXOTX_BAD_ARG;
    if (nprod != 1 && nprod != 3 && nprod != 6) return EXOTX_BAD_ARG;
    int zero = 0;
    EXOTX_CUDA(cudaMemcpyToSymbolAsync(g_tc_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, (cudaStream_t)s));
    size_t smem = (size_t)3 * (128 + N) * K * 2 + 16;
    if (smem > 48 * 1024)
        EXOTX_CUDA(cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tc_selftest<<<1, 128, smem, (cudaStream_t)s>>>(A, B, C, N, K, nprod);
    EXOTX_CHECK_LAUNCH();
    int err = 0;
    EXOTX_CUDA(cudaMemcpyFromSymbolAsync(&err, g_tc_error, sizeof(int), 0, cudaMemcpyDeviceToHost, (cudaStream_t)s));
    EXOTX_CUDA(cudaStreamSynchronize((cudaStream_t)s));
    return err ? EXOTX_TIMEOUT : EXOTX_OK;
}
