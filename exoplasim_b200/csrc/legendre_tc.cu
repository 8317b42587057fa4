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
    bool ok = __all_sync(0xffffffffu, tc::mbar_wait(bar, 0));
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
    // stacked-split forward tables (NTRU+1 <= 128): block (m, t, p) at [(m*4+t)*2+p]
    bool has3 = false;
    std::vector<long long> fwd3_off;
    unsigned char *fwd3 = nullptr;
    long long *d_fwd3_off = nullptr;
    // cached job lists, keyed by (direction, nlev, ninst)
    struct Jobs { int dir, nlev, ninst, njobs, dset; int4 *d = nullptr; };
    std::vector<Jobs> jobs;
    ~TcTables() {
        cudaFree(inv); cudaFree(fwd); cudaFree(d_inv_off); cudaFree(d_fwd_off);
        cudaFree(fwd3); cudaFree(d_fwd3_off);
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

// inverse block (m, t) = [p][split][rows nj8][Kp_p] (K-major core matrices); the
// spectral filter skspgp(n) (legmod.f90:241) is folded into the table entries
__global__ void k_build_tc_inv(const double *qref, const int *woff, const long long *off, const double *filt,
                               int nlat, int nlath, int ncsp, int ntp1, int nj8, int t, int tref,
                               unsigned char *base) {
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
            if (r < nlath && k < Kq) v = q[(size_t)r * ncsp + woff[m] + 2 * k + p] * filt[m + 2 * k + p];
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

// stacked-split forward block (m, t, p) = per latitude chunk of 32:
// [S01: 2R rows (a0 of modes 0..R-1, then a1)][S2: 2R rows (zeros, then a2)] x chunk width
__global__ void k_build_tc_fwd3(const double *qref, const int *woff, const long long *off3, int nlat, int nlath,
                                int ncsp, int ntp1, int njc, int t, int tref, unsigned char *base) {
    const int m = blockIdx.x, p = blockIdx.y;
    const int K = ntp1 - m, Kq = kpar(K, p), R = pad8(Kq);
    if (Kq == 0) return;
    unsigned char *blk = base + off3[(m * 4 + t) * 2 + p];
    const double *q = qref + (size_t)tref * ncsp * nlat;
    size_t co = 0;
    for (int j0 = 0; j0 < njc; j0 += 32) {
        const int jw = min(32, njc - j0);
        const size_t tt = (size_t)2 * R * jw * 2;
        for (int idx = threadIdx.x; idx < 2 * R * jw; idx += blockDim.x) {
            const int row = idx / jw, jj = idx % jw, j = j0 + jj;
            const int mode = row < R ? row : row - R;
            double v = 0.0;
            if (mode < Kq && j < nlath) v = q[(size_t)j * ncsp + woff[m] + 2 * mode + p];
            __nv_bfloat16 h, mm, l;
            split3d(v, h, mm, l);
            const uint32_t o = tc::kmajor_off(row, jj, jw);
            *reinterpret_cast<__nv_bfloat16 *>(blk + co + o) = row < R ? h : mm;
            *reinterpret_cast<__nv_bfloat16 *>(blk + co + tt + o) = row < R ? __float2bfloat16_rn(0.f) : l;
        }
        co += 2 * tt;
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
    if (ntp1 <= 128) {
        // every parity has at most 64 modes: the stacked-split forward tables
        T->fwd3_off.assign(ntp1 * 8, 0);
        long long o3 = 0;
        for (int m = 0; m < ntp1; m++)
            for (int t = 0; t < 4; t++)
                for (int q = 0; q < 2; q++) {
                    T->fwd3_off[(m * 4 + t) * 2 + q] = o3;
                    o3 += 8LL * pad8(kpar(ntp1 - m, q)) * T->njc;
                }
        T->has3 = cudaMalloc(&T->fwd3, o3) == cudaSuccess &&
                  cudaMalloc(&T->d_fwd3_off, sizeof(long long) * ntp1 * 8) == cudaSuccess &&
                  cudaMemcpy(T->d_fwd3_off, T->fwd3_off.data(), sizeof(long long) * ntp1 * 8,
                             cudaMemcpyHostToDevice) == cudaSuccess;
        if (!T->has3) { delete T; return EXOTX_NO_MEM; }
        for (int t = 0; t < 4; t++) {
            k_build_tc_fwd3<<<dim3(ntp1, 2), 256>>>(p->d_qref, p->d_woff, T->d_fwd3_off, p->nlat, p->nlath, p->ncsp,
                                                    ntp1, T->njc, t, kFwdRef[t], T->fwd3);
            note_launch();
        }
    }
    for (int t = 0; t < 4; t++) {
        k_build_tc_inv<<<ntp1, 256>>>(p->d_qref, p->d_woff, T->d_inv_off, p->d_fs64, p->nlat, p->nlath, p->ncsp,
                                      ntp1, T->nj8, t, kInvRef[t], T->inv);
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
static constexpr size_t TC_SMEM_MAX = 227 * 1024;
// the persistent kernel sizes its grid to the SM count and allocates all 512
// TMEM columns, so it asks for enough shared memory that two CTAs never share an SM
static constexpr size_t kPersistSmemMin = 116 * 1024;

#include "legendre_tc_kernels.cuh"

// the half-table inverse mode runs where two CTAs fit an SM with 64-column
// qi tiles (and 32-column qu/qv tiles, 256 TMEM columns each)
static constexpr size_t kInvHalfSmemMax = 112 * 1024;
static bool inv_half(exotx_plan p, int nj8) {
    return p->inv_half_ok && inv_smem_half(nj8, p->ntp1, 64) <= kInvHalfSmemMax;
}

// inverse column tiles: as wide as shared memory (both parities of one table
// plus the staged columns) and TMEM (tables x parities x columns <= 256) allow;
// in the half-table mode 64 (qi, qj) and 32 (qu/qv) columns
static void inv_tiles_full(int nj8, int ntp1, int *nc_qi, int *nc_uv) {
    int a = 128, b = 64;
    while (a > 16 && inv_smem(nj8, ntp1, a) + TCI_BARS > TC_SMEM_MAX) a -= 16;
    while (b > 16 && inv_smem(nj8, ntp1, b) + TCI_BARS > TC_SMEM_MAX) b -= 16;
    *nc_qi = a;
    *nc_uv = b;
}
static void inv_tiles(exotx_plan p, int nj8, int *nc_qi, int *nc_uv) {
    if (inv_half(p, nj8)) {
        *nc_qi = 64;
        *nc_uv = 32;
        return;
    }
    inv_tiles_full(nj8, p->ntp1, nc_qi, nc_uv);
}

// forward kernel variants, tried in order until the widest job fits shared memory:
// 4 levels per job with both table halves resident, 4 levels with one half
// buffer, 2 levels with one half buffer
static const int kFwdNlt[3] = {4, 4, 2};
static const bool kFwdOne[3] = {false, true, true};
static int fwd_level(exotx_plan p, const TcTables *T) {
    for (int v = 0; v < 3; v++)
        if (fwd_smem(p->ntp1, T->njc, kFwdNlt[v], kFwdOne[v]) <= TC_SMEM_MAX) return v;
    return -1;
}
// the persistent stacked-split forward kernel runs wherever its tables exist and fit
static bool use_fwd3(const TcTables *T) { return T->has3 && fpipe_smem(T->njc) <= TC_SMEM_MAX; }
// SMs of the current device (the grid of the persistent kernels)
static exotx_status sm_count(int *nsm) {
    int dev = 0;
    EXOTX_CUDA(cudaGetDevice(&dev));
    EXOTX_CUDA(cudaDeviceGetAttribute(nsm, cudaDevAttrMultiProcessorCount, dev));
    if (*nsm < 1) *nsm = 1;
    return EXOTX_OK;
}
// the persistent stacked-split forward kernel: one CTA per SM walks the job list
static exotx_status launch_fwd_pipe(TcFwd3Launch &P, int njobs, int njmax, bool folded, cudaStream_t s) {
    int nsm = 0;
    EXOTX_TRY(sm_count(&nsm));
    const size_t smem = std::max(fpipe_smem(njmax), kPersistSmemMin);   // one CTA per SM
    if (smem > TC_SMEM_MAX) return EXOTX_BAD_DIM;
    P.njobs = njobs;
    P.njmax = njmax;
    auto kern = folded ? k_tc_forward_pipe<F3_NLT, true> : k_tc_forward_pipe<F3_NLT, false>;
    EXOTX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    const int grid = std::max(1, std::min(njobs, nsm));
    cudaEvent_t ev = ktimer_start(EXOTX_K_TC_FORWARD, s);
    EXOTX_CUDA(launch_pdl(kern, dim3(grid), dim3(FP_THREADS), smem, s, P));   // set-up overlaps the FFT's tail
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_TC_FORWARD, s, ev);
    return EXOTX_OK;
}
static void fwd3_args(TcFwd3Args &A, exotx_plan p, const TcTables *T, int L, const float2 *W, long long nrows,
                      float *spout) {
    A.tab = T->fwd3; A.off = T->d_fwd3_off; A.woff = p->d_woff; A.W = W; A.nrows = nrows;
    A.filt = p->d_fg32; A.spout = spout;
    A.L = L; A.nlat = p->nlat; A.nlath = p->nlath; A.njc = T->njc; A.ntp1 = p->ntp1; A.nrsp = 2 * p->ncsp;
}
// stacked-split forward jobs of one instance range: (m, inst | seg << 16, l0, nl | parity << 8),
// with a cost estimate (modes x latitude pairs) for ordering
static void fwd3_jobs(exotx_plan p, const TcTables *T, int L, int ninst, int seg,
                      std::vector<std::pair<long long, int4>> &v) {
    for (int m = 0; m < p->ntp1; m++)
        for (int q = 0; q < 2; q++) {
            const int Kq = kpar(p->ntp1 - m, q);
            if (!Kq) continue;
            const long long cost = (long long)pad8(Kq) * T->njc;
            for (int i = 0; i < ninst; i++)
                for (int l0 = 0; l0 < L; l0 += F3_NLT)
                    v.push_back({cost, make_int4(m, i | (seg << 16), l0, std::min(F3_NLT, L - l0) | (q << 8))});
        }
}

static exotx_status launch_fwd(const TcFwdLaunch &P, int level, int njobs, size_t smem, cudaStream_t s) {
    cudaEvent_t ev = nullptr;
    if (kFwdNlt[level] == 4) {
        EXOTX_CUDA(cudaFuncSetAttribute(k_tc_forward<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
        ev = ktimer_start(EXOTX_K_TC_FORWARD, s);
        k_tc_forward<4><<<njobs, TCT2, smem, s>>>(P);
    } else {
        EXOTX_CUDA(cudaFuncSetAttribute(k_tc_forward<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
        ev = ktimer_start(EXOTX_K_TC_FORWARD, s);
        k_tc_forward<2><<<njobs, TCT2, smem, s>>>(P);
    }
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_TC_FORWARD, s, ev);
    return EXOTX_OK;
}

// dset = 1: the gridpointd inverse set (qi on st, sq, sp; no qj job), whose
// forward jobs are the gridpointa ones
static exotx_status tc_jobs(exotx_plan p, TcTables *T, int dir, int L, int ninst, const int4 **d, int *njobs,
                            int dset = 0) {
    if (dir == 1) dset = 0;
    for (auto &j : T->jobs)
        if (j.dir == dir && j.nlev == L && j.ninst == ninst && j.dset == dset) {
            *d = j.d; *njobs = j.njobs; return EXOTX_OK;
        }
    std::vector<int4> v;
    int INV_NC_QI, INV_NC_UV;
    inv_tiles(p, T->nj8, &INV_NC_QI, &INV_NC_UV);
    for (int m = 0; m < p->ntp1; m++) {
        if (dir == 0) {
            const int n0 = ninst * (dset ? 2 * L + 1 : 4 * L + 1) * 2, n1 = dset ? 0 : ninst * 2, n2 = ninst * L * 4;
            for (int c = 0; c < n0; c += INV_NC_QI) v.push_back(make_int4(m, 0, c, std::min(INV_NC_QI, n0 - c)));
            for (int c = 0; c < n1; c += INV_NC_QI) v.push_back(make_int4(m, 1, c, std::min(INV_NC_QI, n1 - c)));
            for (int c = 0; c < n2; c += INV_NC_UV) v.push_back(make_int4(m, 2, c, std::min(INV_NC_UV, n2 - c)));
        } else {
            // slabs of nlt levels of one instance; the level-independent gvpp rides with slab 0
            if (use_fwd3(T)) {
                if (m == 0) {
                    std::vector<std::pair<long long, int4>> w;
                    fwd3_jobs(p, T, L, ninst, 0, w);
                    std::stable_sort(w.begin(), w.end(), [](const std::pair<long long, int4> &x,
                                                            const std::pair<long long, int4> &y) {
                        return x.first > y.first;
                    });
                    for (auto &e : w) v.push_back(e.second);
                }
                continue;
            }
            const int lv = fwd_level(p, T), nlt = lv < 0 ? 2 : kFwdNlt[lv];
            for (int i = 0; i < ninst; i++)
                for (int l0 = 0; l0 < L; l0 += nlt)
                    v.push_back(make_int4(m, i, l0, std::min(nlt, L - l0)));
        }
    }
    TcTables::Jobs J;
    J.dir = dir; J.nlev = L; J.ninst = ninst; J.njobs = (int)v.size(); J.dset = dset;
    if (cudaMalloc(&J.d, sizeof(int4) * v.size()) != cudaSuccess) return EXOTX_NO_MEM;
    if (cudaMemcpy(J.d, v.data(), sizeof(int4) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess) return EXOTX_CUDA_ERR;
    T->jobs.push_back(J);
    *d = J.d;
    *njobs = J.njobs;
    return EXOTX_OK;
}

// ---------------------------------------------------------- set drivers
static exotx_status tc_inverse_run(exotx_plan p, const float *spin, float *gpout, int L, int ninst, int dset,
                                   cudaStream_t s) {
    TcTables *T;
    EXOTX_TRY(tc_tables(p, &T));
    const long long nrsp = 2LL * p->ncsp, nhor = (long long)p->nlat * p->nlon;
    const int nfo = dset ? 4 * L + 1 : 6 * L + 3;
    // chunk instances so the m-major Fourier intermediate stays L2-resident
    const size_t per_inst = (size_t)nfo * p->nlat * p->ntp1 * sizeof(float2);
    int chunk = (int)std::max<size_t>(1, p->chunk_inv / per_inst);
    chunk = std::min(chunk, ninst);
    EXOTX_TRY(ensure_work(p, per_inst * chunk));
    const int4 *jobs;
    int njobs;
    EXOTX_TRY(tc_jobs(p, T, 0, L, chunk, &jobs, &njobs, dset));
    int nc_qi, nc_uv;
    inv_tiles(p, T->nj8, &nc_qi, &nc_uv);
    const bool half = inv_half(p, T->nj8);
    size_t smem = half ? std::max(inv_smem_half(T->nj8, p->ntp1, nc_qi), inv_smem_half(T->nj8, p->ntp1, nc_uv))
                       : std::max(inv_smem(T->nj8, p->ntp1, nc_qi), inv_smem(T->nj8, p->ntp1, nc_uv));
    // the persistent kernel keeps its barriers in front of the tables, and asks
    // for enough shared memory that two of its CTAs never share an SM (TMEM)
    if (!half) smem = std::max(smem + TCI_BARS, kPersistSmemMin);
    if (smem > TC_SMEM_MAX) return EXOTX_BAD_DIM;
    if (half)
        EXOTX_CUDA(cudaFuncSetAttribute(k_tc_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    else
        EXOTX_CUDA(cudaFuncSetAttribute(k_tc_inverse_p, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    int nsm = 0;
    EXOTX_TRY(sm_count(&nsm));
    for (int i0 = 0; i0 < ninst; i0 += chunk) {
        const int ni = std::min(chunk, ninst - i0);
        const int4 *jl = jobs;
        int nj = njobs;
        if (ni != chunk) EXOTX_TRY(tc_jobs(p, T, 0, L, ni, &jl, &nj, dset));
        TcInvLaunch P;
        P.jobs = jl;
        P.nprod = 6;
        P.half = half ? 1 : 0;
        TcInvArgs &A = P.seg[0];
        A.tab = T->inv; A.off = T->d_inv_off; A.woff = p->d_woff;
        A.spin = spin + (size_t)i0 * (4 * L + 1) * nrsp;
        A.filt = p->d_fs32;
        A.W = (float2 *)p->d_work;
        A.nrows = (long long)ni * nfo * p->nlat;
        A.L = L; A.nlat = p->nlat; A.nlath = p->nlath; A.nj8 = T->nj8; A.ntp1 = p->ntp1; A.nrsp = (int)nrsp;
        A.plavor = (float)p->desc.plavor;
        A.dset = dset;
        cudaEvent_t ev = ktimer_start(EXOTX_K_TC_INVERSE, s);
        if (half)
            EXOTX_CUDA(launch_pdl(k_tc_inverse, dim3(nj), dim3(TCI_HALF), smem, s, P));   // set-up overlaps the last tail
        else
            EXOTX_CUDA(launch_pdl(k_tc_inverse_p, dim3(std::min(nj, nsm)), dim3(TCI), smem, s, P, nj));
        EXOTX_CHECK_LAUNCH();
        ktimer_stop(EXOTX_K_TC_INVERSE, s, ev);
        EXOTX_TRY(fft_inverse_l<float>((const float *)p->d_work, gpout + (size_t)i0 * nfo * nhor, p->nlon, A.nrows,
                                       p->ntp1, 1, A.nrows, s));
    }
    return EXOTX_OK;
}

exotx_status tc_inverse_batch(exotx_plan p, const float *spin, float *gpout, int L, int ninst, cudaStream_t s) {
    return tc_inverse_run(p, spin, gpout, L, ninst, 0, s);
}
exotx_status tc_inverse_batch_d(exotx_plan p, const float *spin, float *gpout, int L, int ninst, cudaStream_t s) {
    return tc_inverse_run(p, spin, gpout, L, ninst, 1, s);
}

// The global means (the n = 0 coefficients) of the mixed forward set in FP64.
// For m = n = 0 the tables qe, qm and qq vanish (Q_00 = 0, m = 0, n(n+1) = 0),
// so mktend's temperature, qtend's humidity and fc2sp(gvpp) reduce to
// sum_lat qc_00(lat) A0(lat) skgpsp(0), A0 the zonal mean of the grid row
// (fc2sp legmod.f90:178-223, mktend :555-602).  One block per (instance,
// field) sums its grid rows in FP64 from the FP32 grid input and overwrites
// the coefficient the tensor cores wrote: the model's mass (ln ps) and
// energy budgets then close in FP64 (the reference keeps spp(1:2) conserved,
// plasim.f90:2937-2938).  Field f of an instance: 0..L-1 temperature, L..2L-1
// humidity, 2L the ln ps tendency (gridpointa only).  One launch covers the
// segments of an ensemble as well.
struct N0Seg {
    const float *gpin;
    const double *rowsum; // FP64 grid-row sums from the forward FFT (may be null: summed here)
    float *spout;
    const double *qc00;   // qc(w = 0, lat), stride qstride
    const double *fg;     // skgpsp
    int qstride, L, nfi, nfo, nlat, nlon, nrsp, dset, nf, blk0;
};
struct N0Launch {
    N0Seg seg[TC_MAXSEG];
    int nseg;
};

constexpr int N0_MAXLAT = 1024;

__global__ void __launch_bounds__(256) k_n0_fp64(const __grid_constant__ N0Launch P) {
    __shared__ double rs[N0_MAXLAT];
    pdl_trigger();
    int si = 0;
    while (si + 1 < P.nseg && (int)blockIdx.x >= P.seg[si + 1].blk0) si++;
    const N0Seg &S = P.seg[si];
    const int b = blockIdx.x - S.blk0, L = S.L;
    const int inst = b / S.nf, f = b - inst * S.nf;
    int fin, fout;
    if (f < L) { fin = f; fout = L + f; }                                    // tn (gtdt) -> stf
    else if (f < 2 * L) { fin = S.dset ? 2 * L + f : f; fout = 2 * L + f; }  // qn (gqdt) -> sqf
    else { fin = 7 * L; fout = 4 * L; }                                      // gvpp -> spf
    const long long row0 = ((long long)inst * S.nfi + fin) * S.nlat;
    pdl_wait();   // the grid, the row sums and the tensor cores' outputs come from earlier kernels
    if (S.rowsum) {
        for (int lat = threadIdx.x; lat < S.nlat; lat += blockDim.x) rs[lat] = S.rowsum[row0 + lat];
    } else {
        // eight lanes per row in the order of the forward FFT's row sums: lane t
        // adds the complex elements t + 8 j (real part first), then an xor butterfly
        const int t = threadIdx.x & 7, g = threadIdx.x >> 3, ng = blockDim.x >> 3, h = S.nlon / 2;
        for (int lat0 = 0; lat0 < S.nlat; lat0 += ng) {
            const int lat = lat0 + g;
            double a = 0.0;
            if (lat < S.nlat) {
                const float2 *row = reinterpret_cast<const float2 *>(S.gpin + (size_t)(row0 + lat) * S.nlon);
                for (int e = t; e < h; e += 8) {
                    const float2 x = row[e];
                    a += (double)x.x;
                    a += (double)x.y;
                }
            }
            for (int o = 1; o < 8; o <<= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            if (lat < S.nlat && t == 0) rs[lat] = a;
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        double acc = 0.0;
        for (int lat = threadIdx.x; lat < S.nlat; lat += 32) acc += S.qc00[(size_t)lat * S.qstride] * (rs[lat] / (double)S.nlon);
        for (int o = 1; o < 32; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) {
            float *o = S.spout + ((size_t)inst * S.nfo + fout) * S.nrsp;
            o[0] = (float)(acc * S.fg[0]);
            o[1] = 0.0f;
        }
    }
}

static void n0_seg(N0Seg &g, exotx_plan p, const float *gpin, const double *rowsum, float *spout, int L, int dset,
                   int blk0) {
    g.gpin = gpin;
    g.rowsum = rowsum;
    g.spout = spout;
    // qc(w = 0, lat) of the FP64 reference tables [t][lat][w] (qc is table 2)
    g.qc00 = p->d_qref + (size_t)2 * p->nlat * p->ncsp;
    g.qstride = p->ncsp;
    g.fg = p->d_fg64;
    g.L = L;
    g.nfi = dset ? 4 * L : 9 * L + 1;
    g.nfo = dset ? 4 * L : 4 * L + 1;
    g.nlat = p->nlat;
    g.nlon = p->nlon;
    g.nrsp = 2 * p->ncsp;
    g.dset = dset;
    g.nf = dset ? 2 * L : 2 * L + 1;
    g.blk0 = blk0;
}

static exotx_status n0_launch(const N0Launch &P, int nblk, cudaStream_t s) {
    if (nblk == 0) return EXOTX_OK;
    for (int i = 0; i < P.nseg; i++)
        if (P.seg[i].nlat > N0_MAXLAT) return EXOTX_BAD_DIM;
    EXOTX_CUDA(launch_pdl(k_n0_fp64, dim3((unsigned)nblk), dim3(256), 0, s, P));
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}

static exotx_status n0_fp64(exotx_plan p, const float *gsrc, const double *rowsum, float *sout, int L, int ni,
                            int dset, cudaStream_t s) {
    N0Launch P;
    P.nseg = 1;
    n0_seg(P.seg[0], p, gsrc, rowsum, sout, L, dset, 0);
    return n0_launch(P, ni * P.seg[0].nf, s);
}

// the FP64 global means of every segment of an ensemble's forward set (gridpointa)
exotx_status tc_ens_n0(const EnsSeg *segs, const float *const *gpin, int nseg, cudaStream_t s) {
    if (nseg < 1 || nseg > TC_MAXSEG) return EXOTX_BAD_ARG;
    N0Launch P;
    P.nseg = nseg;
    int nblk = 0;
    for (int i = 0; i < nseg; i++) {
        n0_seg(P.seg[i], segs[i].p, gpin[i], nullptr, segs[i].spout, segs[i].L, 0, nblk);
        nblk += segs[i].ninst * P.seg[i].nf;
    }
    return n0_launch(P, nblk, s);
}

static exotx_status tc_forward_run(exotx_plan p, const float *gpin, float *spout, int L, int ninst, int dset,
                                   cudaStream_t s) {
    TcTables *T;
    EXOTX_TRY(tc_tables(p, &T));
    const long long nrsp = 2LL * p->ncsp, nhor = (long long)p->nlat * p->nlon;
    const int nfi = dset ? 4 * L : 9 * L + 1, nfo = dset ? 4 * L : 4 * L + 1;
    const size_t per_inst = (size_t)nfi * p->nlat * p->ntp1 * sizeof(float2);
    int chunk = (int)std::max<size_t>(1, p->chunk_fwd / per_inst);
    chunk = std::min(chunk, ninst);
    // the FP64 grid-row sums of the n = 0 coefficients follow the intermediate,
    // where the folded FFT forms them (register-resident lengths)
    const bool with_rs = fft_fold_rowsum(p->nlon);
    const size_t rs_off = (per_inst * chunk + 255) & ~(size_t)255;
    EXOTX_TRY(ensure_work(p, with_rs ? rs_off + (size_t)chunk * nfi * p->nlat * sizeof(double) : per_inst * chunk));
    const int4 *jobs;
    int njobs;
    EXOTX_TRY(tc_jobs(p, T, 1, L, chunk, &jobs, &njobs));
    const bool v3 = use_fwd3(T);
    const int lv = fwd_level(p, T);
    if (!v3 && lv < 0) return EXOTX_BAD_DIM;
    const size_t smem = v3 ? 0 : fwd_smem(p->ntp1, T->njc, kFwdNlt[lv], kFwdOne[lv]);
    for (int i0 = 0; i0 < ninst; i0 += chunk) {
        const int ni = std::min(chunk, ninst - i0);
        const int4 *jl = jobs;
        int nj = njobs;
        if (ni != chunk) EXOTX_TRY(tc_jobs(p, T, 1, L, ni, &jl, &nj));
        const long long nrows = (long long)ni * nfi * p->nlat;
        const float *gsrc = gpin + (size_t)i0 * nfi * nhor;
        // the persistent kernel reads the intermediate folded about the equator where
        // the grid length has a specialised FFT; otherwise as north and south rows
        bool folded = false;
        double *rowsum = nullptr;
        if (v3) {
            double *rs = with_rs ? reinterpret_cast<double *>(static_cast<char *>(p->d_work) + rs_off) : nullptr;
            const exotx_status sf = fft_forward_fold(gsrc, (float *)p->d_work, p->nlon, p->nlat, nrows, p->ntp1,
                                                     nrows, rs, s);
            if (sf != EXOTX_OK && sf != EXOTX_NOT_BUILT) return sf;
            folded = sf == EXOTX_OK;
            if (folded) rowsum = rs;
        }
        if (!folded)
            EXOTX_TRY(fft_forward_l<float>(gsrc, (float *)p->d_work, p->nlon, nrows, p->ntp1, 1, nrows, s));
        if (v3) {
            TcFwd3Launch P3;
            P3.jobs = jl;
            P3.nprod = 6;
            fwd3_args(P3.seg[0], p, T, L, (const float2 *)p->d_work, nrows, spout + (size_t)i0 * nfo * nrsp);
            P3.seg[0].dset = dset;
            EXOTX_TRY(launch_fwd_pipe(P3, nj, T->njc, folded, s));
            EXOTX_TRY(n0_fp64(p, gsrc, rowsum, spout + (size_t)i0 * nfo * nrsp, L, ni, dset, s));
            continue;
        }
        TcFwdLaunch P;
        P.jobs = jl;
        P.nprod = 6;
        P.onebuf = kFwdOne[lv];
        TcFwdArgs &A = P.seg[0];
        A.tab = T->fwd; A.off = T->d_fwd_off; A.woff = p->d_woff;
        A.W = (const float2 *)p->d_work;
        A.nrows = nrows;
        A.filt = p->d_fg32;
        A.spout = spout + (size_t)i0 * nfo * nrsp;
        A.L = L; A.nlat = p->nlat; A.nlath = p->nlath; A.njc = T->njc; A.ntp1 = p->ntp1; A.nrsp = (int)nrsp;
        A.dset = dset;
        EXOTX_TRY(launch_fwd(P, lv, nj, smem, s));
        EXOTX_TRY(n0_fp64(p, gsrc, nullptr, spout + (size_t)i0 * nfo * nrsp, L, ni, dset, s));
    }
    return EXOTX_OK;
}
exotx_status tc_forward_batch(exotx_plan p, const float *gpin, float *spout, int L, int ninst, cudaStream_t s) {
    return tc_forward_run(p, gpin, spout, L, ninst, 0, s);
}
exotx_status tc_forward_batch_d(exotx_plan p, const float *gpin, float *spout, int L, int ninst, cudaStream_t s) {
    return tc_forward_run(p, gpin, spout, L, ninst, 1, s);
}

// ---------------------------------------------------------- ensembles
// Merged job list of an uneven ensemble: every segment's jobs, with the
// inverse column tiles capped at nc_qi_cap / nc_uv_cap, optionally ordered by
// decreasing work so the longest jobs start first.
exotx_status tc_ens_jobs(const EnsSeg *segs, int nseg, int dir, int nc_qi_cap, int nc_uv_cap, bool sort,
                         int4 **d_jobs, int *njobs, size_t *smem) {
    if (nseg < 1 || nseg > TC_MAXSEG) return EXOTX_BAD_ARG;
    std::vector<std::pair<long long, int4>> v;
    size_t smax = 0;
    int lv = 0;       // forward variant shared by every segment of the launch
    bool v3 = true;   // stacked-split forward kernel when every segment has its tables
    for (int sgi = 0; sgi < nseg && dir == 1; sgi++) {
        TcTables *T;
        EXOTX_TRY(tc_tables(segs[sgi].p, &T));
        v3 = v3 && use_fwd3(T);
        const int l = fwd_level(segs[sgi].p, T);
        if (l < 0) return EXOTX_BAD_DIM;
        lv = std::max(lv, l);
    }
    for (int sgi = 0; sgi < nseg; sgi++) {
        const EnsSeg &g = segs[sgi];
        exotx_plan p = g.p;
        TcTables *T;
        EXOTX_TRY(tc_tables(p, &T));
        const int L = g.L, ni = g.ninst;
        if (dir == 0) {
            int a, b;
            inv_tiles_full(T->nj8, p->ntp1, &a, &b);   // ensembles run the one-CTA-per-SM mode
            a = std::max(16, std::min(a, nc_qi_cap) & ~15);
            b = std::max(16, std::min(b, nc_uv_cap) & ~15);
            smax = std::max(smax, std::max(inv_smem(T->nj8, p->ntp1, a), inv_smem(T->nj8, p->ntp1, b)));
            for (int m = 0; m < p->ntp1; m++) {
                const int K = p->ntp1 - m;
                const long long kw = pad16(kpar(K, 0)) + pad16(kpar(K, 1));
                const int n0 = ni * (4 * L + 1) * 2, n1 = ni * 2, n2 = ni * L * 4;
                for (int c = 0; c < n0; c += a)
                    v.push_back({kw * a, make_int4(m, 0 | (sgi << 2), c, std::min(a, n0 - c))});
                for (int c = 0; c < n1; c += a)
                    v.push_back({kw * a, make_int4(m, 1 | (sgi << 2), c, std::min(a, n1 - c))});
                for (int c = 0; c < n2; c += b)
                    v.push_back({2 * kw * b, make_int4(m, 2 | (sgi << 2), c, std::min(b, n2 - c))});
            }
        } else if (v3) {
            smax = std::max(smax, fpipe_smem(T->njc));
            fwd3_jobs(p, T, L, ni, sgi, v);
        } else {
            const int nlt = kFwdNlt[lv];
            smax = std::max(smax, fwd_smem(p->ntp1, T->njc, nlt, kFwdOne[lv]));
            for (int m = 0; m < p->ntp1; m++) {
                const int K = p->ntp1 - m;
                const long long kw = (long long)(pad8(kpar(K, 0)) + pad8(kpar(K, 1))) * T->njc;
                for (int i = 0; i < ni; i++)
                    for (int l0 = 0; l0 < L; l0 += nlt)
                        v.push_back({kw, make_int4(m, i | (sgi << 16), l0, std::min(nlt, L - l0))});
            }
        }
    }
    if (smax > TC_SMEM_MAX) return EXOTX_BAD_DIM;
    if (sort)
        std::stable_sort(v.begin(), v.end(), [](const std::pair<long long, int4> &x,
                                               const std::pair<long long, int4> &y) { return x.first > y.first; });
    std::vector<int4> jobs(v.size());
    for (size_t i = 0; i < v.size(); i++) jobs[i] = v[i].second;
    int4 *d = nullptr;
    EXOTX_CUDA(cudaMalloc(&d, sizeof(int4) * jobs.size()));
    if (cudaMemcpy(d, jobs.data(), sizeof(int4) * jobs.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return EXOTX_CUDA_ERR;
    }
    *d_jobs = d;
    *njobs = (int)jobs.size();
    *smem = smax;
    return EXOTX_OK;
}

// whether the forward tensor-core launch over these segments is the persistent
// kernel, which reads the intermediate folded about the equator
bool tc_ens_fwd_folded(const EnsSeg *segs, int nseg) {
    for (int i = 0; i < nseg; i++) {
        TcTables *T;
        if (tc_tables(segs[i].p, &T) != EXOTX_OK || !use_fwd3(T)) return false;
    }
    return nseg > 0;
}

// one tensor-core launch over every segment: inverse (spin -> W) or forward (W -> spout)
exotx_status tc_ens_run(const EnsSeg *segs, int nseg, int dir, const int4 *d_jobs, int njobs, size_t smem,
                        int nprod, cudaStream_t s) {
    if (nseg < 1 || nseg > TC_MAXSEG || (nprod != 3 && nprod != 6)) return EXOTX_BAD_ARG;
    if (njobs == 0) return EXOTX_OK;
    if (dir == 0) {
        TcInvLaunch P;
        P.jobs = d_jobs;
        P.nprod = nprod;
        for (int i = 0; i < nseg; i++) {
            const EnsSeg &g = segs[i];
            exotx_plan p = g.p;
            TcTables *T;
            EXOTX_TRY(tc_tables(p, &T));
            TcInvArgs &A = P.seg[i];
            A.tab = T->inv; A.off = T->d_inv_off; A.woff = p->d_woff;
            A.spin = g.spin; A.filt = p->d_fs32; A.W = (float2 *)g.W;
            A.nrows = (long long)g.ninst * (6 * g.L + 3) * p->nlat;
            A.L = g.L; A.nlat = p->nlat; A.nlath = p->nlath; A.nj8 = T->nj8; A.ntp1 = p->ntp1;
            A.nrsp = 2 * p->ncsp; A.plavor = (float)p->desc.plavor;
        }
        // the persistent kernel: barriers in front of the tables, one CTA per SM
        const size_t smem_p = std::max(smem + TCI_BARS, kPersistSmemMin);
        if (smem_p > TC_SMEM_MAX) return EXOTX_BAD_DIM;
        int nsm = 0;
        EXOTX_TRY(sm_count(&nsm));
        EXOTX_CUDA(cudaFuncSetAttribute(k_tc_inverse_p, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
        cudaEvent_t ev = ktimer_start(EXOTX_K_TC_INVERSE, s);
        k_tc_inverse_p<<<std::min(njobs, nsm), TCI, smem_p, s>>>(P, njobs);
        EXOTX_CHECK_LAUNCH();
        ktimer_stop(EXOTX_K_TC_INVERSE, s, ev);
    } else {
        TcFwdLaunch P;
        P.jobs = d_jobs;
        P.nprod = nprod;
        int lv = 0;
        bool v3 = true;
        for (int i = 0; i < nseg; i++) {
            TcTables *T;
            EXOTX_TRY(tc_tables(segs[i].p, &T));
            v3 = v3 && use_fwd3(T);
            const int l = fwd_level(segs[i].p, T);
            if (l < 0) return EXOTX_BAD_DIM;
            lv = std::max(lv, l);
        }
        if (v3) {
            TcFwd3Launch P3;
            P3.jobs = d_jobs;
            P3.nprod = nprod;
            int njmax = 16;
            for (int i = 0; i < nseg; i++) {
                const EnsSeg &g = segs[i];
                TcTables *T;
                EXOTX_TRY(tc_tables(g.p, &T));
                fwd3_args(P3.seg[i], g.p, T, g.L, (const float2 *)g.W,
                          (long long)g.ninst * (9 * g.L + 1) * g.p->nlat, g.spout);
                njmax = std::max(njmax, T->njc);
            }
            return launch_fwd_pipe(P3, njobs, njmax, true, s);   // the ensemble FFT writes the folded form
        }
        P.onebuf = kFwdOne[lv];
        for (int i = 0; i < nseg; i++) {
            const EnsSeg &g = segs[i];
            exotx_plan p = g.p;
            TcTables *T;
            EXOTX_TRY(tc_tables(p, &T));
            TcFwdArgs &A = P.seg[i];
            A.tab = T->fwd; A.off = T->d_fwd_off; A.woff = p->d_woff;
            A.W = (const float2 *)g.W;
            A.nrows = (long long)g.ninst * (9 * g.L + 1) * p->nlat;
            A.filt = p->d_fg32; A.spout = g.spout;
            A.L = g.L; A.nlat = p->nlat; A.nlath = p->nlath; A.njc = T->njc; A.ntp1 = p->ntp1;
            A.nrsp = 2 * p->ncsp;
        }
        EXOTX_TRY(launch_fwd(P, lv, njobs, smem, s));
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
