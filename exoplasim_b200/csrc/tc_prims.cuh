// Blackwell (sm_100a) tensor-core primitives in inline PTX: TMEM allocation,
// tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulate), commit/mbarrier
// completion, TMEM loads, and 1-D bulk (TMA) copies into shared memory.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout:
// 8-row x 16-byte "core matrices" (8 rows x 8 bf16), with
//   LBO = byte distance between K-adjacent core matrices,
//   SBO = byte distance between 8-row groups.
// Every wait is bounded: after kSpinLimit polls a wait gives up and reports
// failure, so no kernel can hang the GPU.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace exotx {
namespace tc {

constexpr uint32_t kSpinLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// true when the phase with parity `phase` completed; false after kSpinLimit polls
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase) {
    uint32_t addr = smem_u32(bar);
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ------------------------------------------------------------ bulk copies
// global -> shared, completion counted on `bar` (bytes % 16 == 0, 16-B aligned)
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst_smem)),
                 "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// make generic-proxy shared-memory writes visible to the async proxy (MMA operands)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// -------------------------------------------------------------------- TMEM
// whole warp: allocate ncols (power of two >= 32) columns; address written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// loads without the wait: issue several, then one tmem_wait_ld() before use
__device__ __forceinline__ void tmem_ld8_nw(uint32_t taddr, uint32_t *r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16_nw(uint32_t taddr, uint32_t *r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld32_nw(uint32_t taddr, uint32_t *r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// -------------------------------------------------------------------- MMA
// shared-memory matrix descriptor, K-major, no swizzle
__device__ __forceinline__ uint64_t smem_desc(const void *p, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_u32(p) >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}
// descriptor of (p + bytes) from the descriptor of p (16-byte aligned offsets;
// the 14-bit start-address field cannot carry below 256 KB of shared memory)
__device__ __forceinline__ uint64_t desc_add(uint64_t d, uint32_t bytes) { return d + (uint64_t)(bytes >> 4); }
// split-product schedule: term pairs (a, b) with a + b <= 2; product 0 is hi*hi
__host__ __device__ constexpr int pair_a(int pr) { return pr == 2 || pr == 4 ? 1 : (pr == 5 ? 2 : 0); }
__host__ __device__ constexpr int pair_b(int pr) { return pr == 1 || pr == 4 ? 1 : (pr == 3 ? 2 : 0); }
// instruction descriptor: D=F32, A=B=BF16, both K-major, shape M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, bool acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"((uint32_t)acc)
        : "memory");
}
// arrive on `bar` once all previously issued MMAs of this thread completed
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// byte offset of element (row r, k) in a K-major no-swizzle tile with kt
// K-elements per row (kt multiple of 8); core matrices K-fastest in a row group
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int kt) {
    return (uint32_t)(((r >> 3) * (kt >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// The same layout with the K-adjacent core matrices 144 bytes apart (16 bytes
// of padding after each): a warp storing one 4-byte word (2 K-elements) per
// lane for 32 consecutive K-pairs of one row then touches 32 distinct banks.
// ngk = K-groups of 8 in a row group; the row-group stride (SBO) is ngk * 144.
constexpr uint32_t kPadLbo = 144;
__host__ __device__ __forceinline__ uint32_t kpad_off(int r, int k, int ngk) {
    return (uint32_t)(((r >> 3) * ngk + (k >> 3)) * kPadLbo + (r & 7) * 16 + (k & 7) * 2);
}

// three-term BF16 split of two values into BF16x2 words (a in the low half)
__device__ __forceinline__ void split3x2(float a, float b, uint32_t &h, uint32_t &m, uint32_t &l) {
    const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
    const float2 hf = __bfloat1622float2(h2);
    const float r0 = a - hf.x, r1 = b - hf.y;
    const __nv_bfloat162 m2 = __floats2bfloat162_rn(r0, r1);
    const float2 mf = __bfloat1622float2(m2);
    const __nv_bfloat162 l2 = __floats2bfloat162_rn(r0 - mf.x, r1 - mf.y);
    h = *reinterpret_cast<const uint32_t *>(&h2);
    m = *reinterpret_cast<const uint32_t *>(&m2);
    l = *reinterpret_cast<const uint32_t *>(&l2);
}

// three-term BF16 split: x ~= h + m + l with |x - (h+m+l)| <= 2^-24 |x| (normal range)
__device__ __forceinline__ void split3(float x, __nv_bfloat16 &h, __nv_bfloat16 &m, __nv_bfloat16 &l) {
    h = __float2bfloat16_rn(x);
    float r1 = x - __bfloat162float(h);
    m = __float2bfloat16_rn(r1);
    float r2 = r1 - __bfloat162float(m);
    l = __float2bfloat16_rn(r2);
}

// split3 of 8 values into three rows of 8 packed BF16 (one 16-byte core-matrix row each)
__device__ __forceinline__ void split3x8(const float *x, uint4 &h, uint4 &m, uint4 &l) {
    uint32_t hw[4], mw[4], lw[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
        const float2 hf = __bfloat1622float2(h2);
        const float r0 = x[2 * i] - hf.x, r1 = x[2 * i + 1] - hf.y;
        const __nv_bfloat162 m2 = __floats2bfloat162_rn(r0, r1);
        const float2 mf = __bfloat1622float2(m2);
        const __nv_bfloat162 l2 = __floats2bfloat162_rn(r0 - mf.x, r1 - mf.y);
        hw[i] = *reinterpret_cast<const uint32_t *>(&h2);
        mw[i] = *reinterpret_cast<const uint32_t *>(&m2);
        lw[i] = *reinterpret_cast<const uint32_t *>(&l2);
    }
    h = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    m = make_uint4(mw[0], mw[1], mw[2], mw[3]);
    l = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

}  // namespace tc
}  // namespace exotx
