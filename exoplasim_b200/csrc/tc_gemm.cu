// FP32-accurate GEMM on the tensor cores, for the radiation surrogate's
// training (surrogate.cu): C[m][n] = sum_k A(m,k) B(k,n) (+ bias[n]) with
// A(m,k) = A[m*am + k*ak] and B(k,n) = B[k*bk + n*bn] in FP32.
//
// Both operands are split into three BF16 terms (x ~= h + m + l to 2^-24
// relative) as they are staged in shared memory, and the six split products
// of order <= 2 accumulate in FP32 in tensor memory: the hi*hi product in one
// accumulator, the five corrections in another (the tensor-core adder
// truncates; keeping the large term's chain apart bounds that error), summed
// in the epilogue.  The result agrees with an FP32 SIMT GEMM to about 1e-6.
//
// A CTA (8 warps) computes a 128 x 128 tile of C over a range of K: all
// threads stage K-chunks of 32 into one of two buffers while thread 0 issues
// the MMAs of the previous chunk (tcgen05.mma, kind::f16, M = 128); a commit
// per chunk frees its buffer.  Long K (the weight gradient's sum over the
// batch) is split over CTAs (grid z) into a workspace that a second kernel
// sums in a fixed order.  Every wait is bounded and reports through an error
// word that exotx_mlp_check reads.
#include <algorithm>
#include "exotx_internal.cuh"
#include "tc_prims.cuh"

namespace exotx {

constexpr int TG_M = 128, TG_N = 128, TG_KC = 32, TG_THREADS = 256;
constexpr int TG_NGK = TG_KC / 8;                                    // K core matrices per row group
constexpr uint32_t TG_TERM = (TG_M / 8) * TG_NGK * tc::kPadLbo;     // bytes of one split term of a tile
constexpr size_t TG_SMEM = 2 * 6 * (size_t)TG_TERM + 64;             // 2 stages x (3 A + 3 B terms) + barriers
constexpr int TG_KSPLIT = 256;                                       // K per CTA when K is split

__device__ int g_tg_error;   // nonzero: a bounded wait in k_tc_sgemm gave up

__device__ __forceinline__ void tg_st4(unsigned char *p, uint32_t v) { *reinterpret_cast<uint32_t *>(p) = v; }

// stage K-chunk [k0, k0 + 32) of the A tile (rows m0..) and the B tile (rows n0..) as split terms
__device__ __forceinline__ void tg_stage(int M, int N, int kend, int m0, int n0, int k0, const float *A, long long am,
                                         long long ak, const float *B, long long bk, long long bn, unsigned char *sa,
                                         unsigned char *sb) {
    constexpr int NP = TG_M * TG_KC / 2;   // (row, K-pair) slots of a tile
    for (int i = threadIdx.x; i < NP; i += TG_THREADS) {
        // K-contiguous operands: consecutive threads along K; otherwise along the rows
        int r, kp;
        if (ak == 1) { r = i / (TG_KC / 2); kp = i % (TG_KC / 2); }
        else { r = i % TG_M; kp = i / TG_M; }
        const int k = k0 + 2 * kp, m = m0 + r;
        const float a0 = (m < M && k < kend) ? A[m * am + k * ak] : 0.f;
        const float a1 = (m < M && k + 1 < kend) ? A[m * am + (k + 1) * ak] : 0.f;
        uint32_t h, md, l;
        tc::split3x2(a0, a1, h, md, l);
        const uint32_t o = tc::kpad_off(r, 2 * kp, TG_NGK);
        tg_st4(sa + o, h);
        tg_st4(sa + TG_TERM + o, md);
        tg_st4(sa + 2 * TG_TERM + o, l);
    }
    for (int i = threadIdx.x; i < NP; i += TG_THREADS) {
        int r, kp;
        if (bk == 1) { r = i / (TG_KC / 2); kp = i % (TG_KC / 2); }
        else { r = i % TG_N; kp = i / TG_N; }
        const int k = k0 + 2 * kp, n = n0 + r;
        const float b0 = (n < N && k < kend) ? B[k * bk + n * bn] : 0.f;
        const float b1 = (n < N && k + 1 < kend) ? B[(k + 1) * bk + n * bn] : 0.f;
        uint32_t h, md, l;
        tc::split3x2(b0, b1, h, md, l);
        const uint32_t o = tc::kpad_off(r, 2 * kp, TG_NGK);
        tg_st4(sb + o, h);
        tg_st4(sb + TG_TERM + o, md);
        tg_st4(sb + 2 * TG_TERM + o, l);
    }
}

// part == nullptr: C = A B (+ bias); otherwise part[z][M][N] = this K-range's A B
__global__ void __launch_bounds__(TG_THREADS) k_tc_sgemm(int M, int N, int K, const float *__restrict__ A, long long am,
                                                          long long ak, const float *__restrict__ B, long long bk,
                                                          long long bn, float *__restrict__ C, long long ldc,
                                                          const float *__restrict__ bias, int klen,
                                                          float *__restrict__ part) {
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char *st[2] = {sm, sm + 6 * (size_t)TG_TERM};   // stage: A terms, then B terms
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 12 * (size_t)TG_TERM);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TG_M, n0 = blockIdx.y * TG_N;
    const int kbeg = blockIdx.z * klen, kend = min(K, kbeg + klen);
    const int NT = min(TG_N, (N - n0 + 15) & ~15);   // MMA N
    const int nchunk = (kend - kbeg + TG_KC - 1) / TG_KC;
    if (warp == 0) tc::tmem_alloc(slot, 256);        // accumulators: hi*hi at column 0, corrections at 128
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar + 1, 1);
        tc::mbar_fence_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    bool ok = true;
    if (nchunk > 0) tg_stage(M, N, kend, m0, n0, kbeg, A, am, ak, B, bk, bn, st[0], st[0] + 3 * TG_TERM);
    tc::fence_proxy_async();
    __syncthreads();
    const uint32_t idesc = tc::idesc_bf16(TG_M, NT);
    for (int c = 0; c < nchunk && ok; c++) {
        const int b = c & 1;
        if (tid == 0) {
            tc::fence_after_sync();
            const uint64_t da = tc::smem_desc(st[b], tc::kPadLbo, TG_NGK * tc::kPadLbo);
            const uint64_t db = tc::smem_desc(st[b] + 3 * TG_TERM, tc::kPadLbo, TG_NGK * tc::kPadLbo);
#pragma unroll
            for (int ks = 0; ks < TG_KC / 16; ks++) {
#pragma unroll
                for (int pr = 0; pr < 6; pr++) {
                    const bool first = c == 0 && ks == 0 && pr <= 1;
                    tc::mma_bf16(tmem + (pr == 0 ? 0u : 128u),
                                 tc::desc_add(da, tc::pair_a(pr) * TG_TERM + ks * 2 * tc::kPadLbo),
                                 tc::desc_add(db, tc::pair_b(pr) * TG_TERM + ks * 2 * tc::kPadLbo), idesc, !first);
                }
            }
            tc::mma_commit(bar + b);
        }
        if (c + 1 < nchunk) {
            const int nb = (c + 1) & 1;
            // the buffer's previous chunk (c - 1) must have been read by its MMAs
            if (c >= 1) ok = tc::mbar_wait(bar + nb, ((c - 1) >> 1) & 1);
            ok = __syncthreads_and(ok) != 0;
            if (!ok) break;
            tg_stage(M, N, kend, m0, n0, kbeg + (c + 1) * TG_KC, A, am, ak, B, bk, bn, st[nb], st[nb] + 3 * TG_TERM);
            tc::fence_proxy_async();
        }
        __syncthreads();
    }
    // every MMA has completed once the last chunk's commit has arrived
    if (ok && nchunk > 0) ok = tc::mbar_wait(bar + ((nchunk - 1) & 1), ((nchunk - 1) >> 1) & 1);
    ok = __syncthreads_and(ok) != 0;
    if (!ok && tid == 0) atomicExch(&g_tg_error, 1);
    tc::fence_after_sync();
    if (ok) {
        // epilogue: warp w drains TMEM lane quarter w % 4 (32 rows), columns half w / 4
        const int q = warp & 3, half = warp >> 2, row = m0 + 32 * q + lane;
        const uint32_t lane_addr = (uint32_t)(32 * q) << 16;
        const int nh = NT / 2, cend = (half + 1) * nh;
        for (int c0 = half * nh; c0 < cend; c0 += 16) {
            uint32_t ra[16], rb[16];
            if (nchunk > 0) {
                tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)c0, ra);
                tc::tmem_ld16_nw(tmem + lane_addr + 128u + (uint32_t)c0, rb);
                tc::tmem_wait_ld();
            } else {
#pragma unroll
                for (int i = 0; i < 16; i++) ra[i] = rb[i] = 0u;
            }
            if (row >= M) continue;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int n = n0 + c0 + i;
                if (c0 + i >= cend || n >= N) break;
                const float v = __uint_as_float(ra[i]) + __uint_as_float(rb[i]);
                if (part) part[((size_t)blockIdx.z * M + row) * N + n] = v;
                else C[(size_t)row * ldc + n] = v + (bias ? bias[n] : 0.f);
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

// C[m][n] = sum over z in order of part[z][m][n] (+ bias[n])
__global__ void k_tg_reduce(const float *part, int nz, int M, int N, float *C, long long ldc, const float *bias) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)M * N;
         i += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(i / N), n = (int)(i - (long long)m * N);
        float v = 0.f;
        for (int z = 0; z < nz; z++) v += part[(size_t)z * M * N + i];
        C[(size_t)m * ldc + n] = v + (bias ? bias[n] : 0.f);
    }
}

// workspace floats the split-K form needs for an M x N product over K
size_t tc_sgemm_work(int M, int N, int K) {
    const int nz = (K + TG_KSPLIT - 1) / TG_KSPLIT;
    return nz > 1 ? (size_t)nz * M * N : 0;
}

exotx_status tc_sgemm(int M, int N, int K, const float *A, long long am, long long ak, const float *B, long long bk,
                      long long bn, float *C, long long ldc, const float *bias, float *work, size_t work_elems,
                      cudaStream_t s) {
    if (M <= 0 || N <= 0 || K < 0) return EXOTX_BAD_ARG;
    const int nz = K > TG_KSPLIT ? (K + TG_KSPLIT - 1) / TG_KSPLIT : 1;
    const bool split = nz > 1;
    if (split && (!work || work_elems < (size_t)nz * M * N)) return EXOTX_BAD_ARG;
    EXOTX_CUDA(cudaFuncSetAttribute(k_tc_sgemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TG_SMEM));
    const dim3 grid((unsigned)((M + TG_M - 1) / TG_M), (unsigned)((N + TG_N - 1) / TG_N), (unsigned)nz);
    k_tc_sgemm<<<grid, TG_THREADS, TG_SMEM, s>>>(M, N, K, A, am, ak, B, bk, bn, C, ldc, bias, split ? TG_KSPLIT : K,
                                                  split ? work : nullptr);
    EXOTX_CHECK_LAUNCH();
    if (split) {
        const long long n = (long long)M * N;
        k_tg_reduce<<<(unsigned)std::min<long long>((n + 255) / 256, 1184), 256, 0, s>>>(work, nz, M, N, C, ldc, bias);
        EXOTX_CHECK_LAUNCH();
    }
    return EXOTX_OK;
}

exotx_status tc_sgemm_error(int *err, cudaStream_t s) {
    EXOTX_CUDA(cudaMemcpyFromSymbolAsync(err, g_tg_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    EXOTX_CUDA(cudaStreamSynchronize(s));
    return EXOTX_OK;
}

}  // namespace exotx
