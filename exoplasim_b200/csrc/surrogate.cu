// Learned radiation surrogate (no counterpart in the reference): an MLP that
// maps one radmod column (radmod.f90 radstep :927-1110) to its heating-rate
// profile and its four surface fluxes.  Training runs in FP32 on the
// library's own GEMM/activation/Adam kernels; inference runs in BF16 on the
// tensor cores (tcgen05, FP32 accumulation in TMEM) with the features built
// in the same kernel.  Columns whose inputs leave the training ranges are
// collected on the device and computed by the plain radstep kernel instead.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "exotx_internal.cuh"
#include "tc_prims.cuh"

namespace exotx {

constexpr int MLP_MAX_LAYERS = 8;
constexpr int SURR_TILE = 128;          // columns per tile (MMA M)
constexpr int SURR_THREADS = 512;      // 4 warp groups x the 4 TMEM lane quarters
constexpr int SURR_WIDTH = 256;         // hidden width of the tensor-core inference path
constexpr int SURR_KIN = 80;            // padded input features (nin <= 80)
constexpr int SURR_NOUT = 32;           // padded outputs (nout <= 32)

// error word of the inference kernel: nonzero when a bounded wait gave up
__device__ int g_surr_error;

}  // namespace exotx

struct exotx_mlp_s {
    int nin, width, nhid, nout, nl, maxb;
    int din[exotx::MLP_MAX_LAYERS], dout[exotx::MLP_MAX_LAYERS];
    long long woff[exotx::MLP_MAX_LAYERS], boff[exotx::MLP_MAX_LAYERS];
    long long nparams = 0;
    float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
    float *ws = nullptr;     // training activations
    float *norm = nullptr;   // xm, xs, xlo, xhi (nin each), ym, ys (nout each)
    bool has_norm = false;
    unsigned char *tw = nullptr;   // BF16 weight tiles for inference
    long long twoff[exotx::MLP_MAX_LAYERS + 1];
    bool prepared = false;
    int *fb = nullptr;       // [0] = fallback count, [1..] = column list
    int fb_cap = 0;
    float *split = nullptr;  // split-K workspace of the weight-gradient GEMMs
    size_t split_elems = 0;
};

namespace exotx {

// ------------------------------------------------------------ features
// Raw features of one column (L levels), in this order:
//   T(k) k<L, T surface, ln q(k) k<=L, cc(k) k<L, ln ps, albedo, cos zenith,
//   ln CO2 (ppmv), zsolar1, rcoeff, sin(latitude)          -> 3L + 9 values
// Targets: per level the heating rate (K/day) times (ps / 1e5 Pa) (1 + ADV q),
// which removes the exact 1 / (ps (1 + ADV q)) factor of radstep's heating
// (radmod.f90:1100-1110) from what the network learns; then SW down, SW up,
// LW down, LW up at the surface (dfd, dfu, dftd, dftu at NLEP) -> L + 4 values.
template <typename T> struct SurrIn {
    const T *dt, *dq, *dcc, *dp, *dalb, *gmu0, *dqco2, *zsol, *sid;
    double zsolar1, rcoeff, adv;
    int L, nhor, nlon;
};

__host__ __device__ inline int surr_nin(int L) { return 3 * L + 9; }
__host__ __device__ inline int surr_nout(int L) { return L + 4; }

template <bool FAST> __device__ __forceinline__ float surr_log(float x) { return FAST ? __logf(x) : logf(x); }

template <typename T, bool FAST = false>
__device__ __forceinline__ float surr_feature(const SurrIn<T> &in, int col, int f) {
    const int L = in.L;
    const size_t n = (size_t)in.nhor;
    if (f < L + 1) return (float)in.dt[(size_t)f * n + col];
    f -= L + 1;
    if (f < L + 1) return surr_log<FAST>(fmaxf((float)in.dq[(size_t)f * n + col], 1e-12f));
    f -= L + 1;
    if (f < L) return (float)in.dcc[(size_t)f * n + col];
    f -= L;
    switch (f) {
        case 0: return surr_log<FAST>(fmaxf((float)in.dp[col], 1.f));
        case 1: return (float)in.dalb[col];
        case 2: return (float)in.gmu0[col];
        case 3: return surr_log<FAST>(fmaxf((float)in.dqco2[col], 1e-6f));
        case 4: return in.zsol ? (float)in.zsol[col] : (float)in.zsolar1;
        case 5: return in.zsol ? (float)in.zsol[2 * n + col] : (float)in.rcoeff;
        default: return (float)in.sid[col / in.nlon];
    }
}

template <typename T>
__global__ void k_surr_features(SurrIn<T> in, float *X) {
    const int nin = surr_nin(in.L);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)in.nhor * nin;
         i += (long long)gridDim.x * blockDim.x) {
        const int col = (int)(i % in.nhor), f = (int)(i / in.nhor);
        X[(size_t)col * nin + f] = surr_feature(in, col, f);
    }
}

// heating-rate scale of level k: 86400 s/day x (ps / 1e5 Pa) x (1 + ADV q_k)
template <typename T>
__device__ __forceinline__ T surr_hscale(const SurrIn<T> &in, int col, int k) {
    return (T)86400 * (in.dp[col] / (T)1e5) * ((T)1 + (T)in.adv * in.dq[(size_t)k * in.nhor + col]);
}

template <typename T>
__global__ void k_surr_targets(SurrIn<T> in, const T *dtdt, const T *dfd, const T *dfu, const T *dftd,
                               const T *dftu, float *Y) {
    const int L = in.L, nhor = in.nhor;
    const int nout = surr_nout(L);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)nhor * nout;
         i += (long long)gridDim.x * blockDim.x) {
        const int col = (int)(i % nhor), o = (int)(i / nhor);
        float v;
        if (o < L) v = (float)(dtdt[(size_t)o * nhor + col] * surr_hscale(in, col, o));
        else {
            const T *src = o == L ? dfd : o == L + 1 ? dfu : o == L + 2 ? dftd : dftu;
            v = (float)src[(size_t)L * nhor + col];
        }
        Y[(size_t)col * nout + o] = v;
    }
}

// ------------------------------------------------------------ training (FP32)
// The three GEMMs of a layer's forward and backward pass run on the tensor
// cores in FP32-accurate split form (tc_sgemm, tc_gemm.cu); the element-wise
// parts are the kernels below.

__device__ __forceinline__ float silu(float z) { return z / (1.f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    const float sg = 1.f / (1.f + expf(-z));
    return sg * (1.f + z * (1.f - sg));
}

// inference activation: fast exponential and division (the result is rounded to BF16)
// silu(z) = z sigmoid(z) = h + h tanh(h) with h = z/2: one MUFU operation (tanh.approx, max relative
// error about 2^-11), half the special-function work of the exp + reciprocal form
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float silu_fast(float z) {
    const float h = 0.5f * z;
    return fmaf(h, tanh_approx(h), h);
}

__global__ void k_silu(const float *Z, float *H, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        H[i] = silu(Z[i]);
}
__global__ void k_silu_bwd(const float *dH, const float *Z, float *dZ, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dZ[i] = dH[i] * silu_grad(Z[i]);
}
// mean (optionally weighted: Wt per element, may be null) squared error over
// n x nout; dY = d(loss)/dY; loss accumulated into *loss
__global__ void k_mse(const float *Y, const float *T, const float *Wt, float *dY, long long n, float scale,
                      float *loss) {
    __shared__ float red[256];
    float acc = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i], w = Wt ? Wt[i] : 1.f;
        dY[i] = 2.f * w * d * scale;
        acc += w * d * d;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss) atomicAdd(loss, red[0] * scale);
}
// db[o] = sum_b dZ[b][o]
__global__ void k_colsum(const float *dZ, float *db, int n, int nc) {
    const int o = blockIdx.x * 32 + (threadIdx.x & 31);
    const int r0 = threadIdx.x >> 5, nr = blockDim.x >> 5;
    __shared__ float red[8][33];
    float acc = 0.f;
    if (o < nc)
        for (int b = r0; b < n; b += nr) acc += dZ[(size_t)b * nc + o];
    red[r0][threadIdx.x & 31] = acc;
    __syncthreads();
    if (r0 == 0 && o < nc) {
        float t = 0.f;
        for (int r = 0; r < nr; r++) t += red[r][threadIdx.x & 31];
        db[o] = t;
    }
}
__global__ void k_adam(float *P, const float *G, float *M, float *V, long long n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float g = G[i];
        const float m = b1 * M[i] + (1.f - b1) * g;
        const float v = b2 * V[i] + (1.f - b2) * g * g;
        M[i] = m;
        V[i] = v;
        P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
}

static unsigned grid_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148 * 16); }

// activations: Z_l, H_l (maxb x width) for hidden l, then Y, dY (maxb x nout), dA, dZa, dZb (maxb x width)
static float *ws_Z(exotx_mlp net, int l) { return net->ws + (size_t)2 * l * net->maxb * net->width; }
static float *ws_H(exotx_mlp net, int l) { return ws_Z(net, l) + (size_t)net->maxb * net->width; }
static float *ws_Y(exotx_mlp net) { return net->ws + (size_t)2 * net->nhid * net->maxb * net->width; }
static float *ws_dY(exotx_mlp net) { return ws_Y(net) + (size_t)net->maxb * net->nout; }
static float *ws_dA(exotx_mlp net) { return ws_dY(net) + (size_t)net->maxb * net->nout; }
static float *ws_dZ(exotx_mlp net, int i) { return ws_dA(net) + (size_t)(1 + i) * net->maxb * net->width; }

static exotx_status gemm(exotx_mlp net, int M, int N, int K, const float *A, long long am, long long ak,
                         const float *B, long long bk, long long bn, float *C, long long ldc, const float *bias,
                         cudaStream_t s) {
    return tc_sgemm(M, N, K, A, am, ak, B, bk, bn, C, ldc, bias, net->split, net->split_elems, s);
}

static exotx_status mlp_forward(exotx_mlp net, const float *X, int n, cudaStream_t s) {
    const float *H = X;
    for (int l = 0; l < net->nl; l++) {
        const int din = net->din[l], dout = net->dout[l];
        float *Z = l < net->nhid ? ws_Z(net, l) : ws_Y(net);
        EXOTX_TRY(gemm(net, n, dout, din, H, din, 1, net->P + net->woff[l], 1, din, Z, dout, net->P + net->boff[l], s));
        if (l < net->nhid) {
            k_silu<<<grid_for((long long)n * dout), 256, 0, s>>>(Z, ws_H(net, l), (long long)n * dout);
            EXOTX_CHECK_LAUNCH();
            H = ws_H(net, l);
        }
    }
    return EXOTX_OK;
}

// ------------------------------------------------------------ inference (tcgen05)
template <typename T> struct SurrArgs {
    SurrIn<T> in;
    const unsigned char *tw;
    long long twoff[MLP_MAX_LAYERS];
    const float *bias[MLP_MAX_LAYERS];
    int nl, nin, nout;
    const float *norm;
    T *dtdt, *dfd, *dfu, *dftd, *dftu, *dswfl, *dlwfl;
    int *fb;   // [0] count, [1..] list
};

// layer geometry of the inference tiles
__host__ __device__ inline int surr_layer_N(int l, int nl) { return l == nl - 1 ? SURR_NOUT : SURR_WIDTH; }
__host__ __device__ inline int surr_layer_K(int l) { return l == 0 ? SURR_KIN : SURR_WIDTH; }
__host__ __device__ inline int surr_layer_KC(int l) { return l == 0 ? SURR_KIN : 128; }

template <typename T>
__global__ void __launch_bounds__(SURR_THREADS) k_surr_infer(SurrArgs<T> A) {
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char *abuf = sm;                       // 128 rows x 256 K, BF16 K-major (64 KB)
    unsigned char *wbuf = sm + 65536;               // 2 chunks x 64 KB of layer weights
    uint64_t *bar_w = reinterpret_cast<uint64_t *>(sm + 65536 + 131072);   // [2]: weight chunk c arrived
    uint64_t *bar_mma = bar_w + 2;
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar_w + 3);
    int *flags = reinterpret_cast<int *>(bar_w + 4);   // 128 out-of-range flags
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, quarter = warp & 3, grp = warp >> 2;
    const int row = quarter * 32 + lane;  // TMEM lane = column of the tile
    const int nhor = A.in.nhor, nl = A.nl;
    const int ntiles = (nhor + SURR_TILE - 1) / SURR_TILE;
    if (warp == 0) tc::tmem_alloc(slot, 2 * SURR_WIDTH);   // two layer accumulators
    uint32_t wi0 = 0, wi1 = 0;   // weight chunks 0 and 1 issued (thread 0)
    auto issue_weights = [&](int l) {
        const int N = surr_layer_N(l, nl), K = surr_layer_K(l), KC = surr_layer_KC(l);
        const uint32_t cbytes = (uint32_t)N * KC * 2;
        // one barrier per K chunk: the MMAs over a chunk start as soon as it is in
        for (int c = 0; c < K / KC; c++) {
            (c == 0 ? wi0 : wi1)++;
            tc::mbar_arrive_expect_tx(bar_w + c, cbytes);
            tc::bulk_g2s(wbuf + c * 65536, A.tw + A.twoff[l] + (size_t)c * cbytes, cbytes, bar_w + c);
        }
    };
    if (tid == 0) {
        tc::mbar_init(bar_w, 1);
        tc::mbar_init(bar_w + 1, 1);
        tc::mbar_init(bar_mma, 1);
        tc::mbar_fence_init();
        if (blockIdx.x < ntiles) issue_weights(0);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    const float *xm = A.norm, *xs = A.norm + A.nin, *xlo = A.norm + 2 * A.nin, *xhi = A.norm + 3 * A.nin;
    const float *ym = A.norm + 4 * A.nin, *ys = ym + A.nout;
    // per input feature: source array (read at the column, or at its latitude
    // row for kind 5), transform kind (0 none, 1-3 log with floors 1e-12, 1,
    // 1e-6, -1 a constant), the constant, and 1 / the normalisation scale
    struct __align__(16) Feat {
        const T *src;
        int kind;
        float cst, xr, xm, lo, hi;
    };
    __shared__ Feat ftab[SURR_KIN];
    // every layer's biases (hidden layers: SURR_WIDTH each; output: SURR_NOUT)
    __shared__ __align__(16) float bias_s[MLP_MAX_LAYERS][SURR_WIDTH];
    for (int i = tid; i < MLP_MAX_LAYERS * SURR_WIDTH; i += SURR_THREADS) {
        const int l = i / SURR_WIDTH, c = i - l * SURR_WIDTH;
        bias_s[l][c] = (l < nl && c < surr_layer_N(l, nl) && c < (l == nl - 1 ? A.nout : SURR_WIDTH)) ? A.bias[l][c] : 0.f;
    }
    if (tid < SURR_KIN) {
        const int L = A.in.L, n = A.in.nhor;
        int f = tid, kd = -1;
        const T *src = nullptr;
        float cv = 0.f;
        if (f < A.nin) {
            if (f < L + 1) { src = A.in.dt + (size_t)f * n; kd = 0; }
            else if (f < 2 * L + 2) { src = A.in.dq + (size_t)(f - L - 1) * n; kd = 1; }
            else if (f < 3 * L + 2) { src = A.in.dcc + (size_t)(f - 2 * L - 2) * n; kd = 0; }
            else {
                switch (f - 3 * L - 2) {
                    case 0: src = A.in.dp; kd = 2; break;
                    case 1: src = A.in.dalb; kd = 0; break;
                    case 2: src = A.in.gmu0; kd = 0; break;
                    case 3: src = A.in.dqco2; kd = 3; break;
                    case 4: if (A.in.zsol) { src = A.in.zsol; kd = 0; } else cv = (float)A.in.zsolar1; break;
                    case 5: if (A.in.zsol) { src = A.in.zsol + 2 * (size_t)n; kd = 0; } else cv = (float)A.in.rcoeff; break;
                    default: src = A.in.sid; kd = 5; break;
                }
            }
            ftab[f].xr = 1.f / xs[f];
            ftab[f].xm = xm[f]; ftab[f].lo = xlo[f]; ftab[f].hi = xhi[f];
        } else {
            ftab[f].xr = 0.f;
            ftab[f].xm = 0.f; ftab[f].lo = -INFINITY; ftab[f].hi = INFINITY;
        }
        ftab[f].src = src; ftab[f].kind = kd; ftab[f].cst = cv;
    }
    __syncthreads();
    uint32_t pw0 = 0, pw1 = 0, pm = 0;   // completed phases of the two weight barriers and the MMA barrier
    bool ok = true;  // cleared on every thread when a wait gives up
    // thread 0: MMAs of layer l over the 16-wide K steps [k0, k1) (within one weight
    // chunk) into the layer's accumulator (layers alternate between two 256-column
    // TMEM regions); a call that starts a chunk waits for it; commit arrives on bar_mma
    auto issue_mma = [&](int l, int k0, int k1, bool commit) -> bool {
        const int N = surr_layer_N(l, nl), K = surr_layer_K(l), KC = surr_layer_KC(l);
        if ((k0 * 16) % KC == 0) {
            const int c = (k0 * 16) / KC;
            uint32_t &ph = c == 0 ? pw0 : pw1;
            if (!tc::mbar_wait(bar_w + c, ph & 1)) {
                atomicExch(&g_surr_error, 1);
                return false;
            }
            ph++;
            tc::fence_after_sync();
        }
        const uint32_t idesc = tc::idesc_bf16(SURR_TILE, N);
        const uint64_t da = tc::smem_desc(abuf, 128, (uint32_t)(K / 8) * 128);
        const uint64_t db = tc::smem_desc(wbuf, 128, (uint32_t)(KC / 8) * 128);
        const uint32_t d = tmem + (uint32_t)((l & 1) * SURR_WIDTH);
        for (int kc = k0; kc < k1; kc++) {
            const int c = (kc * 16) / KC, kin = (kc * 16) % KC;
            tc::mma_bf16(d, tc::desc_add(da, kc * 256), tc::desc_add(db, c * 65536 + (kin / 8) * 128), idesc, kc > 0);
        }
        if (commit) tc::mma_commit(bar_mma);
        return true;
    };
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int col = tile * SURR_TILE + row;
        const bool live = col < nhor;
        if (grp == 0) flags[row] = 0;
        __syncthreads();
        // features: warp group g builds the 8-input blocks g, g+4, ... of its row,
        // normalised, as BF16; the block's eight raw loads are issued together
        {
            int bad = 0;
            const int crow = col / A.in.nlon;   // latitude row, for the kind-5 feature
#pragma unroll 1
            for (int g = grp; g < SURR_KIN / 8; g += 4) {
                const int f0 = 8 * g;
                float raw[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const Feat &F = ftab[f0 + e];
                    raw[e] = F.cst;
                    if (live && F.kind >= 0) raw[e] = (float)F.src[F.kind == 5 ? crow : col];
                }
                float v[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int f = f0 + e;
                    const Feat &F = ftab[f];
                    float x = raw[e];
                    if (F.kind == 1) x = __logf(fmaxf(x, 1e-12f));
                    else if (F.kind == 2) x = __logf(fmaxf(x, 1.f));
                    else if (F.kind == 3) x = __logf(fmaxf(x, 1e-6f));
                    if (live && f < A.nin) bad |= (x < F.lo) | (x > F.hi) | (x != x);
                    v[e] = (live && f < A.nin) ? (x - F.xm) * F.xr : 0.f;
                }
                uint32_t w[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                    w[i] = *reinterpret_cast<const uint32_t *>(&b2);
                }
                *reinterpret_cast<uint4 *>(abuf + tc::kmajor_off(row, f0, SURR_KIN)) = make_uint4(w[0], w[1], w[2], w[3]);
            }
            if (bad) atomicOr(&flags[row], 1);
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        // layer 0 (the input features) in one go; each hidden epilogue below
        // issues the next layer's MMAs in two K halves, the first while the
        // second half of the activations is still being written
        if (tid == 0 && ok) ok = issue_mma(0, 0, SURR_KIN / 16, true);
        for (int l = 0; l < nl; l++) {
            const uint32_t acc = tmem + (uint32_t)((l & 1) * SURR_WIDTH);
            const bool mok = __all_sync(0xffffffffu, tc::mbar_wait(bar_mma, pm & 1));
            pm++;
            if (!mok) { if (lane == 0) atomicExch(&g_surr_error, 2); ok = false; }
            tc::fence_after_sync();
            // the weight buffer is free: fetch the next layer (or the next tile's first)
            if (tid == 0 && mok) {
                if (l + 1 < nl) issue_weights(l + 1);
                else if (tile + (int)gridDim.x < ntiles) issue_weights(0);
            }
            if (!mok) break;
            if (l + 1 < nl) {
                // hidden epilogue: bias + SiLU, BF16, into the next layer's A operand;
                // in half h warp group g takes columns [128h + 32g, 128h + 32g + 32)
                const float *b = bias_s[l];
#pragma unroll 1
                for (int h = 0; h < 2; h++) {
                    const int c0 = 128 * h + 32 * grp;
                    uint32_t r[32];
                    tc::tmem_ld32_nw(acc + lane_addr + (uint32_t)c0, r);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        uint32_t w[4];
#pragma unroll
                        for (int i = 0; i < 4; i++) {
                            const int c = 8 * q + 2 * i;
                            const float2 bb = *reinterpret_cast<const float2 *>(b + c0 + c);
                            const float h0 = silu_fast(__uint_as_float(r[c]) + bb.x);
                            const float h1 = silu_fast(__uint_as_float(r[c + 1]) + bb.y);
                            const __nv_bfloat162 b2 = __floats2bfloat162_rn(h0, h1);
                            w[i] = *reinterpret_cast<const uint32_t *>(&b2);
                        }
                        *reinterpret_cast<uint4 *>(abuf + tc::kmajor_off(row, c0 + 8 * q, SURR_WIDTH)) =
                            make_uint4(w[0], w[1], w[2], w[3]);
                    }
                    tc::fence_proxy_async();
                    tc::fence_before_sync();
                    __syncthreads();
                    tc::fence_after_sync();
                    // K half h of the next layer's A operand is complete
                    constexpr int KH = SURR_WIDTH / 32;   // 16-wide K steps per half
                    if (tid == 0 && ok) ok = issue_mma(l + 1, KH * h, KH * h + KH, h == 1);
                }
            } else {
                // output epilogue: de-normalise and write the in-range columns; warp
                // group g writes the levels k = g (mod 4), group 0 the surface fluxes
                uint32_t r[32];
                tc::tmem_ld32_nw(acc + lane_addr, r);
                tc::tmem_wait_ld();
                if (live && !flags[row]) {
                    const float *b = bias_s[l];
                    const int L = A.in.L;
                    const size_t n = (size_t)nhor;
                    const float ps = (float)A.in.dp[col] * 1e-5f, adv = (float)A.in.adv;
                    // this group's levels k = grp (mod 4): their humidities and heating
                    // rates are read together before the updates
                    constexpr int KMAX = SURR_NOUT / 4;
                    T qk[KMAX], hk[KMAX];
#pragma unroll
                    for (int j = 0; j < KMAX; j++) {
                        const int o = grp + 4 * j;
                        if (o < L && o < A.nout) {
                            qk[j] = A.in.dq[(size_t)o * n + col];
                            hk[j] = A.dtdt[(size_t)o * n + col];
                        }
                    }
#pragma unroll
                    for (int j = 0; j < KMAX; j++) {
                        const int o = grp + 4 * j;
                        if (o < L && o < A.nout) {
                            // r[4j + grp] with constant register indices
                            const uint32_t rv = grp == 0 ? r[4 * j] : grp == 1 ? r[4 * j + 1] : grp == 2 ? r[4 * j + 2] : r[4 * j + 3];
                            const float y = (__uint_as_float(rv) + b[o]) * ys[o] + ym[o];
                            A.dtdt[(size_t)o * n + col] = hk[j] + (T)__fdividef(y, 86400.f * ps * (1.f + adv * (float)qk[j]));
                        }
                    }
                    if (grp == 0) {
                        float f4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                        for (int o = 0; o < SURR_NOUT; o++) {
                            const int i = o - L;
                            if (i < 0 || i > 3 || o >= A.nout) continue;
                            const float y = (__uint_as_float(r[o]) + b[o]) * ys[o] + ym[o];
                            if (i == 0) f4[0] = y; else if (i == 1) f4[1] = y; else if (i == 2) f4[2] = y; else f4[3] = y;
                        }
                        A.dfd[(size_t)L * n + col] = (T)f4[0];
                        A.dfu[(size_t)L * n + col] = (T)f4[1];
                        A.dftd[(size_t)L * n + col] = (T)f4[2];
                        A.dftu[(size_t)L * n + col] = (T)f4[3];
                        A.dswfl[(size_t)L * n + col] = (T)f4[0] + (T)f4[1];
                        A.dlwfl[(size_t)L * n + col] = (T)f4[2] + (T)f4[3];
                    }
                }
                if (live && flags[row] && grp == 0) {
                    const int idx = atomicAdd(A.fb, 1);
                    A.fb[1 + idx] = col;
                }
            }
            if (l + 1 == nl) {
                tc::fence_before_sync();
                __syncthreads();  // TMEM and flags reused by the next tile
                tc::fence_after_sync();
            }
        }
    }
    // after a timeout, a weight load still in flight lands before the block leaves
    if (tid == 0 && !ok) {
        if (wi0 > pw0) tc::mbar_wait(bar_w, pw0 & 1);
        if (wi1 > pw1) tc::mbar_wait(bar_w + 1, pw1 & 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 2 * SURR_WIDTH);
}

}  // namespace exotx

namespace exotx {

// BF16 weight tiles of layer l: [K/KC chunks][N rows][KC], K-major core matrices
__global__ void k_surr_tiles(const float *P, long long woff, int din, int dout, int N, int K, int KC,
                             unsigned char *dst) {
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < N * K; idx += gridDim.x * blockDim.x) {
        const int n = idx / K, k = idx - n * K;
        const float v = (n < dout && k < din) ? P[woff + (long long)n * din + k] : 0.f;
        const int c = k / KC, kk = k - c * KC;
        *reinterpret_cast<__nv_bfloat16 *>(dst + (size_t)c * N * KC * 2 + tc::kmajor_off(n, kk, KC)) =
            __float2bfloat16_rn(v);
    }
}

template <typename T>
static SurrIn<T> surr_in(const exotx_rad_params *p, const exotx_rad_io *io) {
    SurrIn<T> in;
    in.dt = (const T *)io->dt; in.dq = (const T *)io->dq; in.dcc = (const T *)io->dcc; in.dp = (const T *)io->dp;
    in.dalb = (const T *)io->dalb; in.gmu0 = (const T *)io->gmu0; in.dqco2 = (const T *)io->dqco2;
    in.zsol = (const T *)io->zsol; in.sid = (const T *)io->sid;
    in.zsolar1 = p->zsolar1; in.rcoeff = p->rcoeff; in.adv = p->adv;
    in.L = p->nlev; in.nhor = p->nhor; in.nlon = p->nlon;
    return in;
}

static bool surr_io_ok(const exotx_rad_params *p, const exotx_rad_io *io) {
    return p && io && io->dt && io->dq && io->dcc && io->dp && io->dalb && io->gmu0 && io->dqco2 && io->sid &&
           p->nlev >= 2 && p->nlev <= 64 && p->nhor >= 1 && p->nlon >= 1 && p->nhor % p->nlon == 0;
}

static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
    }
    return n;
}

template <typename T>
static exotx_status surr_launch(exotx_mlp net, const exotx_rad_params *p, int prec, const exotx_rad_io *io,
                                cudaStream_t s) {
    SurrArgs<T> A;
    A.in = surr_in<T>(p, io);
    A.tw = net->tw;
    for (int l = 0; l < MLP_MAX_LAYERS; l++) {
        A.twoff[l] = l < net->nl ? net->twoff[l] : 0;
        A.bias[l] = l < net->nl ? net->P + net->boff[l] : nullptr;
    }
    A.nl = net->nl; A.nin = net->nin; A.nout = net->nout; A.norm = net->norm;
    A.dtdt = (T *)io->dtdt; A.dfd = (T *)io->dfd; A.dfu = (T *)io->dfu; A.dftd = (T *)io->dftd;
    A.dftu = (T *)io->dftu; A.dswfl = (T *)io->dswfl; A.dlwfl = (T *)io->dlwfl;
    A.fb = net->fb;
    const size_t smem = 65536 + 131072 + 1024;
    EXOTX_CUDA(cudaFuncSetAttribute(k_surr_infer<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int ntiles = (p->nhor + SURR_TILE - 1) / SURR_TILE;
    const int grid = std::min(ntiles, sm_count());
    cudaEvent_t ev = ktimer_start(EXOTX_K_SURROGATE, s);
    k_surr_infer<T><<<grid, SURR_THREADS, smem, s>>>(A);
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_SURROGATE, s, ev);
    (void)prec;
    return EXOTX_OK;
}

}  // namespace exotx

using namespace exotx;

EXOTX_API exotx_status exotx_mlp_create(int nin, int width, int nhidden, int nout, int max_batch, exotx_mlp *out) {
    if (!out || nin < 1 || width < 1 || nhidden < 1 || nhidden > MLP_MAX_LAYERS - 1 || nout < 1 || max_batch < 1)
        return EXOTX_BAD_ARG;
    exotx_mlp net = new exotx_mlp_s();
    net->nin = nin; net->width = width; net->nhid = nhidden; net->nout = nout; net->nl = nhidden + 1;
    net->maxb = max_batch;
    long long off = 0;
    for (int l = 0; l < net->nl; l++) {
        net->din[l] = l == 0 ? nin : width;
        net->dout[l] = l == net->nl - 1 ? nout : width;
        net->woff[l] = off; off += (long long)net->din[l] * net->dout[l];
        net->boff[l] = off; off += net->dout[l];
    }
    net->nparams = off;
    const size_t wsf = (size_t)2 * nhidden * max_batch * width + (size_t)2 * max_batch * nout +
                       (size_t)3 * max_batch * width;
    net->split_elems = tc_sgemm_work(std::max(width, nout), std::max(nin, width), max_batch);
    bool ok = cudaMalloc(&net->P, off * 4) == cudaSuccess && cudaMalloc(&net->G, off * 4) == cudaSuccess &&
              cudaMalloc(&net->M, off * 4) == cudaSuccess && cudaMalloc(&net->V, off * 4) == cudaSuccess &&
              cudaMalloc(&net->ws, wsf * 4) == cudaSuccess &&
              cudaMalloc(&net->norm, sizeof(float) * (4 * nin + 2 * nout)) == cudaSuccess &&
              (net->split_elems == 0 || cudaMalloc(&net->split, net->split_elems * 4) == cudaSuccess);
    ok = ok && cudaMemset(net->P, 0, off * 4) == cudaSuccess && cudaMemset(net->G, 0, off * 4) == cudaSuccess &&
         cudaMemset(net->M, 0, off * 4) == cudaSuccess && cudaMemset(net->V, 0, off * 4) == cudaSuccess;
    if (!ok) {
        cudaFree(net->P); cudaFree(net->G); cudaFree(net->M); cudaFree(net->V); cudaFree(net->ws); cudaFree(net->norm);
        cudaFree(net->split);
        delete net;
        return EXOTX_NO_MEM;
    }
    *out = net;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_destroy(exotx_mlp net) {
    if (!net) return EXOTX_BAD_ARG;
    cudaFree(net->P); cudaFree(net->G); cudaFree(net->M); cudaFree(net->V); cudaFree(net->ws);
    cudaFree(net->norm); cudaFree(net->tw); cudaFree(net->fb); cudaFree(net->split);
    delete net;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_params(exotx_mlp net, float **params, float **grads, long long *nparams) {
    if (!net || !params || !grads || !nparams) return EXOTX_BAD_ARG;
    *params = net->P; *grads = net->G; *nparams = net->nparams;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_layer(exotx_mlp net, int l, long long *w_off, long long *b_off, int *din,
                                       int *dout) {
    if (!net || l < 0 || l >= net->nl || !w_off || !b_off || !din || !dout) return EXOTX_BAD_ARG;
    *w_off = net->woff[l]; *b_off = net->boff[l]; *din = net->din[l]; *dout = net->dout[l];
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_set_norm(exotx_mlp net, const float *host_norm) {
    if (!net || !host_norm) return EXOTX_BAD_ARG;
    const int n = 4 * net->nin + 2 * net->nout;
    std::vector<float> v(host_norm, host_norm + n);
    for (int f = 0; f < net->nin; f++) v[net->nin + f] = std::max(v[net->nin + f], 1e-6f);          // xs
    for (int o = 0; o < net->nout; o++) v[4 * net->nin + net->nout + o] = std::max(v[4 * net->nin + net->nout + o], 1e-6f);
    EXOTX_CUDA(cudaMemcpy(net->norm, v.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    net->has_norm = true;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_forward(exotx_mlp net, const float *X, float *Y, int n, exotx_stream s) {
    if (!net || !X || !Y || n < 0 || n > net->maxb) return EXOTX_BAD_ARG;
    if (n == 0) return EXOTX_OK;
    EXOTX_TRY(mlp_forward(net, X, n, (cudaStream_t)s));
    EXOTX_CUDA(cudaMemcpyAsync(Y, ws_Y(net), sizeof(float) * n * net->nout, cudaMemcpyDeviceToDevice,
                               (cudaStream_t)s));
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_backward(exotx_mlp net, const float *X, const float *Tt, int n, float *loss,
                                          exotx_stream sv) {
    return exotx_mlp_backward_weighted(net, X, Tt, nullptr, n, loss, sv);
}

EXOTX_API exotx_status exotx_mlp_backward_weighted(exotx_mlp net, const float *X, const float *Tt, const float *Wt,
                                                   int n, float *loss, exotx_stream sv) {
    if (!net || !X || !Tt || n < 1 || n > net->maxb) return EXOTX_BAD_ARG;
    cudaStream_t s = (cudaStream_t)sv;
    EXOTX_TRY(mlp_forward(net, X, n, s));
    const long long ny = (long long)n * net->nout;
    k_mse<<<grid_for(ny), 256, 0, s>>>(ws_Y(net), Tt, Wt, ws_dY(net), ny, 1.f / (float)ny, loss);
    EXOTX_CHECK_LAUNCH();
    const float *dZ = ws_dY(net);
    int cur = 0;
    for (int l = net->nl - 1; l >= 0; l--) {
        const int din = net->din[l], dout = net->dout[l];
        const float *Hp = l > 0 ? ws_H(net, l - 1) : X;
        // dW = dZ^T H_prev, db = column sums of dZ
        EXOTX_TRY(gemm(net, dout, din, n, dZ, 1, dout, Hp, din, 1, net->G + net->woff[l], din, nullptr, s));
        k_colsum<<<(dout + 31) / 32, 256, 0, s>>>(dZ, net->G + net->boff[l], n, dout);
        EXOTX_CHECK_LAUNCH();
        if (l > 0) {
            // dH_prev = dZ W, then through the SiLU of layer l-1
            EXOTX_TRY(gemm(net, n, din, dout, dZ, dout, 1, net->P + net->woff[l], din, 1, ws_dA(net), din, nullptr, s));
            float *dZn = ws_dZ(net, cur);
            k_silu_bwd<<<grid_for((long long)n * din), 256, 0, s>>>(ws_dA(net), ws_Z(net, l - 1), dZn,
                                                                  (long long)n * din);
            EXOTX_CHECK_LAUNCH();
            dZ = dZn;
            cur ^= 1;
        }
    }
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_check(exotx_mlp net, exotx_stream s) {
    if (!net) return EXOTX_BAD_ARG;
    int err = 0;
    EXOTX_TRY(tc_sgemm_error(&err, (cudaStream_t)s));
    return err ? EXOTX_TIMEOUT : EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_adam(exotx_mlp net, float lr, float b1, float b2, float eps, int step,
                                      exotx_stream s) {
    if (!net || step < 1) return EXOTX_BAD_ARG;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<grid_for(net->nparams), 256, 0, (cudaStream_t)s>>>(net->P, net->G, net->M, net->V, net->nparams, lr,
                                                                 b1, b2, eps, c1, c2);
    EXOTX_CHECK_LAUNCH();
    net->prepared = false;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_mlp_prepare(exotx_mlp net, exotx_stream sv) {
    if (!net) return EXOTX_BAD_ARG;
    if (net->width != SURR_WIDTH || net->nin > SURR_KIN || net->nout > SURR_NOUT) return EXOTX_NOT_BUILT;
    cudaStream_t s = (cudaStream_t)sv;
    long long off = 0;
    for (int l = 0; l < net->nl; l++) {
        net->twoff[l] = off;
        off += (long long)surr_layer_N(l, net->nl) * surr_layer_K(l) * 2;
    }
    net->twoff[net->nl] = off;
    if (!net->tw) EXOTX_CUDA(cudaMalloc(&net->tw, off));
    for (int l = 0; l < net->nl; l++) {
        const int N = surr_layer_N(l, net->nl), K = surr_layer_K(l);
        k_surr_tiles<<<(N * K + 255) / 256, 256, 0, s>>>(net->P, net->woff[l], net->din[l], net->dout[l], N, K,
                                                          surr_layer_KC(l), net->tw + net->twoff[l]);
        EXOTX_CHECK_LAUNCH();
    }
    net->prepared = true;
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_surr_features(const exotx_rad_params *p, int prec, const exotx_rad_io *io, float *X,
                                           exotx_stream s) {
    if (!surr_io_ok(p, io) || !X) return EXOTX_BAD_ARG;
    const long long n = (long long)p->nhor * surr_nin(p->nlev);
    if (prec == EXOTX_FP64)
        k_surr_features<double><<<grid_for(n), 256, 0, (cudaStream_t)s>>>(surr_in<double>(p, io), X);
    else if (prec == EXOTX_FP32)
        k_surr_features<float><<<grid_for(n), 256, 0, (cudaStream_t)s>>>(surr_in<float>(p, io), X);
    else
        return EXOTX_BAD_ARG;
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_surr_targets(const exotx_rad_params *p, int prec, const exotx_rad_io *io, float *Y,
                                          exotx_stream s) {
    if (!surr_io_ok(p, io) || !Y || !io->dtdt || !io->dfd || !io->dfu || !io->dftd || !io->dftu) return EXOTX_BAD_ARG;
    const long long n = (long long)p->nhor * surr_nout(p->nlev);
    if (prec == EXOTX_FP64)
        k_surr_targets<double><<<grid_for(n), 256, 0, (cudaStream_t)s>>>(
            surr_in<double>(p, io), (const double *)io->dtdt, (const double *)io->dfd, (const double *)io->dfu,
            (const double *)io->dftd, (const double *)io->dftu, Y);
    else if (prec == EXOTX_FP32)
        k_surr_targets<float><<<grid_for(n), 256, 0, (cudaStream_t)s>>>(
            surr_in<float>(p, io), (const float *)io->dtdt, (const float *)io->dfd, (const float *)io->dfu,
            (const float *)io->dftd, (const float *)io->dftu, Y);
    else
        return EXOTX_BAD_ARG;
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_rad_surrogate(exotx_mlp net, const exotx_rad_params *p, int prec,
                                           const exotx_rad_io *io, int *nfallback, exotx_stream sv) {
    if (!net || !surr_io_ok(p, io)) return EXOTX_BAD_ARG;
    if (!io->dtdt || !io->dfd || !io->dfu || !io->dftd || !io->dftu || !io->dswfl || !io->dlwfl) return EXOTX_BAD_ARG;
    if (prec != EXOTX_FP64 && prec != EXOTX_FP32) return EXOTX_BAD_ARG;
    if (!net->prepared || !net->has_norm) return EXOTX_BAD_ARG;
    if (net->nin != surr_nin(p->nlev) || net->nout != surr_nout(p->nlev)) return EXOTX_BAD_DIM;
    if (p->nsol != 0) return EXOTX_NOT_BUILT;  // the cosine of the zenith angle is an input (gmu0)
    // the network was trained on each column's own cos zenith; zonal-mean
    // insolation (ndcycle = 0) is a different input
    if (p->ndcycle != 1) return EXOTX_NOT_BUILT;
    cudaStream_t s = (cudaStream_t)sv;
    if (net->fb_cap < p->nhor) {
        cudaFree(net->fb);
        net->fb = nullptr;
        net->fb_cap = 0;
        EXOTX_CUDA(cudaMalloc(&net->fb, sizeof(int) * (p->nhor + 1)));
        net->fb_cap = p->nhor;
    }
    EXOTX_CUDA(cudaMemsetAsync(net->fb, 0, sizeof(int), s));
    if (prec == EXOTX_FP64) EXOTX_TRY(surr_launch<double>(net, p, prec, io, s));
    else EXOTX_TRY(surr_launch<float>(net, p, prec, io, s));
    // columns outside the training ranges: the plain radstep kernel
    EXOTX_TRY(radstep_columns(p, prec, io, net->fb + 1, net->fb, p->nhor, s));
    if (nfallback) {
        int err = 0;
        EXOTX_CUDA(cudaMemcpyAsync(nfallback, net->fb, sizeof(int), cudaMemcpyDeviceToHost, s));
        EXOTX_CUDA(cudaMemcpyFromSymbolAsync(&err, g_surr_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
        EXOTX_CUDA(cudaStreamSynchronize(s));
        if (err) {
            const int zero = 0;
            EXOTX_CUDA(cudaMemcpyToSymbol(g_surr_error, &zero, sizeof(int)));
            return EXOTX_TIMEOUT;
        }
    }
    return EXOTX_OK;
}
