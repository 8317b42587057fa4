// Tensor-core Legendre kernels (included by legendre_tc.cu).
//
// One CTA per job.  Thread 0 issues the TMA table copies and the MMAs; the
// other threads stage operands and drain accumulators.  Warps w, w+4, ...
// share TMEM lane quarter w % 4.
#pragma once

constexpr int TCT2 = 256;

__device__ __forceinline__ void st_shared16(unsigned char *p, uint4 v) { *reinterpret_cast<uint4 *>(p) = v; }

// ------------------------------------------------------------ inverse
struct TcInvArgs {
    const unsigned char *tab;
    const long long *off;
    const int *woff;
    const float *spin;      // [inst][4L+1][NRSP]
    const float *filt;      // skspgp
    float2 *W;              // [m][row], row = (inst*(6L+3) + field)*nlat + lat
    long long nrows;
    int L, nlat, nlath, nj8, ntp1, nrsp;
    float plavor;
};

// One launch covers up to TC_MAXSEG segments (a resolution, a level count and
// a run of instances each); a job names its segment.  nprod = 6 keeps every
// split product of order <= 2 (3-term split); nprod = 3 keeps a0b0, a0b1, a1b0.
struct TcInvLaunch {
    TcInvArgs seg[TC_MAXSEG];
    const int4 *jobs;       // (m, group | seg << 2, first column, columns)
    int nprod;
};

// spectral row (complex, filter not applied) feeding column pair gq, and
// whether it is the vorticity of a dv2uv pair (planetary vorticity removed)
__device__ __forceinline__ const float2 *inv_row(const TcInvArgs &A, int group, int gq, bool *zvort) {
    const int L = A.L, nf = 4 * L + 1;
    int inst, f;
    *zvort = false;
    if (group == 0) { inst = gq / nf; f = gq % nf; }
    else if (group == 1) { inst = gq; f = 4 * L; }
    else {
        // columns per level: Dr, Di, Zr, Zi -> pairs 2l (D), 2l+1 (Z)
        inst = gq / (2 * L);
        const int l = (gq % (2 * L)) >> 1;
        *zvort = gq & 1;
        f = *zvort ? 2 * L + l : l;
    }
    return reinterpret_cast<const float2 *>(A.spin + ((size_t)inst * nf + f) * A.nrsp);
}

// 16 warps: all stage operands; thread 0 issues the table copies and MMAs;
// in the epilogue warp w drains TMEM lane quarter w % 4 for column chunk w / 4
constexpr int TCI = 512;

__global__ void __launch_bounds__(TCI) k_tc_inverse(const __grid_constant__ TcInvLaunch P) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int4 jb = P.jobs[blockIdx.x];
    const TcInvArgs &A = P.seg[jb.y >> 2];
    const int nprod = P.nprod;
    const int m = jb.x, group = jb.y & 3, c0 = jb.z, nc = jb.w;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, quarter = warp & 3, sub = warp >> 2;
    const int K = A.ntp1 - m;
    const int Kq[2] = {kpar(K, 0), kpar(K, 1)};
    const int Kp[2] = {pad16(Kq[0]), pad16(Kq[1])};
    const int ncp = pad16(nc);
    const int ntab = group == 2 ? 2 : 1;
    const int nj8 = A.nj8;
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
        // first table copy goes out before the staging so the two overlap
        const int t0 = group == 0 ? 0 : (group == 1 ? 1 : 2);
        tc::mbar_arrive_expect_tx(bar_tma, (uint32_t)tbytes);
        tc::bulk_g2s(tab, A.tab + A.off[m * 4 + t0], (uint32_t)tbytes, bar_tma);
    }
    // stage the spectral columns of both parities.  A unit is one column pair
    // (re, im) and 8 modes of one parity: one 16-byte core-matrix row per
    // column and split term.  The units of both parities form one index space;
    // each thread first loads INV_SLOTS units, then splits and stores them, so
    // the global loads of all its units are in flight together.
    {
        const int npair = ncp >> 1;
        const int U0 = npair * (Kp[0] >> 3), U = U0 + (Kq[1] ? npair * (Kp[1] >> 3) : 0);
        const int w0 = A.woff[m];
        constexpr int INV_SLOTS = 2;
        for (int base = 0; base < U; base += INV_SLOTS * TCI) {
            float2 x[INV_SLOTS][8];
            float fl[INV_SLOTS][8];
#pragma unroll
            for (int s = 0; s < INV_SLOTS; s++) {
                const int u = base + s * TCI + tid;
                const int p = u >= U0, uu = u - (p ? U0 : 0);
                const int q = uu % npair, g = uu / npair;
                const int c = 2 * q;
                bool zv = false;
                const float2 *row = (u < U && c < nc) ? inv_row(A, group, (c0 + c) >> 1, &zv) : nullptr;
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int k = 8 * g + e, nm = 2 * k + p;  // nm = n - m
                    const bool in = row != nullptr && k < Kq[p];
                    x[s][e] = in ? __ldg(row + w0 + nm) : make_float2(0.f, 0.f);
                    fl[s][e] = in ? __ldg(A.filt + m + nm) : 0.f;
                    if (in && zv && m == 0 && nm == 1) x[s][e].x -= A.plavor;  // dv2uv, legmod.f90:332
                }
            }
#pragma unroll
            for (int s = 0; s < INV_SLOTS; s++) {
                const int u = base + s * TCI + tid;
                if (u >= U) break;
                const int p = u >= U0, uu = u - (p ? U0 : 0);
                const int q = uu % npair, g = uu / npair;
                float xr[8], xi[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    xr[e] = x[s][e].x * fl[s][e];
                    xi[e] = x[s][e].y * fl[s][e];
                }
                const uint32_t o = tc::kmajor_off(2 * q, 8 * g, Kp[p]);  // re row; the im row follows at +16
                unsigned char *d0 = dat + (p ? 3 * dtile[0] : 0);
                const size_t dtp = dtile[p];
                uint4 h, mm, l;
                tc::split3x8(xr, h, mm, l);
                st_shared16(d0 + o, h); st_shared16(d0 + dtp + o, mm); st_shared16(d0 + 2 * dtp + o, l);
                tc::split3x8(xi, h, mm, l);
                st_shared16(d0 + o + 16, h); st_shared16(d0 + dtp + o + 16, mm);
                st_shared16(d0 + 2 * dtp + o + 16, l);
            }
        }
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
            if (ti > 0) {
                ok = tc::mbar_wait(bar_mma, (ti - 1) & 1);  // table buffer free again
                if (!ok) break;
                const int t = 2 + ti;
                tc::mbar_arrive_expect_tx(bar_tma, (uint32_t)tbytes);
                tc::bulk_g2s(tab, A.tab + A.off[m * 4 + t], (uint32_t)tbytes, bar_tma);
            }
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
                const uint64_t da0 = tc::smem_desc(tab + to, 128, sbo), db0 = tc::smem_desc(dat + dd, 128, sbo);
                const uint32_t tt = (uint32_t)ttile[p], dt = (uint32_t)dtile[p];
                for (int kc = 0; kc < Kp[p] / 16; kc++) {
#pragma unroll
                    for (int pr = 0; pr < 6; pr++)
                        if (pr < nprod)
                            tc::mma_bf16(pr == 0 ? dm : dc, tc::desc_add(da0, tc::pair_a(pr) * tt + kc * 256),
                                         tc::desc_add(db0, tc::pair_b(pr) * dt + kc * 256), idesc,
                                         kc > 0 || pr > 1);
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
    ok = __all_sync(0xffffffffu, tc::mbar_wait(bar_done, 0));  // warp-uniform for the .sync.aligned TMEM loads
    if (!ok && lane == 0) atomicExch(&g_tc_error, 2);
    tc::fence_after_sync();
    // epilogue: TMEM lane = latitude pair j; quarters past the last pair hold
    // nothing (a warp-uniform test, as the TMEM loads need whole warps)
    if (ok && quarter * 32 < A.nlath) {
        const int j = quarter * 32 + lane;
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        const int L = A.L, nfo = 6 * L + 3, nf = 4 * L + 1;
        const bool has1 = Kq[1] > 0;
        const bool row_ok = j < A.nlath;
        const int latN = j, latS = A.nlat - 1 - j;
        float2 *Wm = A.W + (size_t)m * A.nrows;
        if (group < 2) {
            // P-type qi: N = D0 + D1, S = D0 - D1; Q-type qj: S = D1 - D0
            const float ss = group == 0 ? 1.f : -1.f;
            for (int cc = sub * 16; cc < ncp; cc += 64) {
                uint32_t rm0[16], rc0[16], rm1[16], rc1[16];
                tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(0 * ncp + cc), rm0);
                tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(1 * ncp + cc), rc0);
                if (has1) {
                    tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(2 * ncp + cc), rm1);
                    tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(3 * ncp + cc), rc1);
                }
                tc::tmem_wait_ld();
                // column pair gq = (c0 + cc)/2 + i/2: instance and field without a
                // division per pair (a chunk holds 8 pairs, fewer than nf)
                const int gq0 = (c0 + cc) >> 1;
                const int inst0 = group == 0 ? gq0 / nf : gq0, f0 = group == 0 ? gq0 - inst0 * nf : 4 * L;
#pragma unroll
                for (int i = 0; i < 16; i += 2) {
                    const float d0r = __uint_as_float(rm0[i]) + __uint_as_float(rc0[i]);
                    const float d0i = __uint_as_float(rm0[i + 1]) + __uint_as_float(rc0[i + 1]);
                    const float d1r = has1 ? __uint_as_float(rm1[i]) + __uint_as_float(rc1[i]) : 0.f;
                    const float d1i = has1 ? __uint_as_float(rm1[i + 1]) + __uint_as_float(rc1[i + 1]) : 0.f;
                    if (!row_ok || cc + i >= nc) continue;
                    int inst = inst0, f = f0;
                    if (group == 0) {
                        f += i >> 1;
                        if (f >= nf) { f -= nf; inst++; }
                    } else {
                        inst += i >> 1;
                    }
                    const float2 vn = make_float2(d0r + d1r, d0i + d1i);
                    const float2 vs = make_float2(ss * (d0r - d1r), ss * (d0i - d1i));
                    int F;
                    if (group == 1) F = 6 * L;                    // gpj
                    else if (f < L) F = 3 * L + f;                // sd -> gd
                    else if (f < 2 * L) F = f + L;                // st -> gt
                    else if (f < 4 * L) F = f + 2 * L;            // sz -> gz, sq -> gq
                    else F = 6 * L + 2;                           // sp -> gp
                    float2 *wr = Wm + (size_t)(inst * nfo + F) * A.nlat;
                    wr[latN] = vn;
                    wr[latS] = vs;
                    if (group == 0 && f == 4 * L) {               // gpmt = i*m*gp
                        const float fm = (float)m;
                        float2 *wt = Wm + (size_t)(inst * nfo + 6 * L + 1) * A.nlat;
                        wt[latN] = make_float2(-fm * vn.y, fm * vn.x);
                        wt[latS] = make_float2(-fm * vs.y, fm * vs.x);
                    }
                }
            }
        } else {
            // dv2uv: u = qv*Z - i*qu*D, v = -i*qu*Z - qv*D; qu P-type, qv Q-type.
            // accumulators r = (table, parity): 0 qu p0, 1 qu p1, 2 qv p0, 3 qv p1;
            // columns Dr, Di, Zr, Zi per level; a chunk of 8 columns is 2 levels
            for (int cc = sub * 8; cc < ncp; cc += 32) {
                uint32_t rm[4][8], rc[4][8];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    if ((r & 1) && !has1) continue;
                    tc::tmem_ld8_nw(tmem + lane_addr + (uint32_t)((r * 2 + 0) * ncp + cc), rm[r]);
                    tc::tmem_ld8_nw(tmem + lane_addr + (uint32_t)((r * 2 + 1) * ncp + cc), rc[r]);
                }
                tc::tmem_wait_ld();
                float d[4][8];
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int i = 0; i < 8; i++)
                        d[r][i] = ((r & 1) && !has1) ? 0.f : __uint_as_float(rm[r][i]) + __uint_as_float(rc[r][i]);
                const int q0 = (c0 + cc) >> 2;                    // (instance, level) of the chunk's first level
                const int inst0 = q0 / L, l0 = q0 - inst0 * L;
#pragma unroll
                for (int i = 0; i < 8; i += 4) {
                    if (!row_ok || cc + i >= nc) continue;
                    int inst = inst0, l = l0 + (i >> 2);
                    if (l >= L) { l -= L; inst++; }
                    const int Dr = i, Di = i + 1, Zr = i + 2, Zi = i + 3;
                    const float urs = d[0][Di] + d[3][Zr], ura = d[1][Di] + d[2][Zr];
                    const float uis = -d[0][Dr] + d[3][Zi], uia = -d[1][Dr] + d[2][Zi];
                    const float vrs = d[0][Zi] - d[3][Dr], vra = d[1][Zi] - d[2][Dr];
                    const float vis = -d[0][Zr] - d[3][Di], via = -d[1][Zr] - d[2][Di];
                    float2 *wu = Wm + (size_t)(inst * nfo + l) * A.nlat;
                    float2 *wv = Wm + (size_t)(inst * nfo + L + l) * A.nlat;
                    wu[latN] = make_float2(urs + ura, uis + uia);
                    wu[latS] = make_float2(urs - ura, uis - uia);
                    wv[latN] = make_float2(vrs + vra, vis + via);
                    wv[latS] = make_float2(vrs - vra, vis - via);
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
    int L, nlat, nlath, njc, ntp1, nrsp;
};

struct TcFwdLaunch {
    TcFwdArgs seg[TC_MAXSEG];
    const int4 *jobs;       // (m, inst | seg << 16, first level, levels)
    int nprod;
    int onebuf;             // 1: both parity halves of a table share one buffer (large grids)
};

// Columns of one forward job (levels l0..l0+nl-1 of one instance), per table,
// laid out as if the slab always had NLT levels (fixed positions):
//   column (fi, li, ri) = (fi*NLT + li)*2 + ri
//   qc: tn, qn [+ gvpp at 2*2*NLT]   qe: fv, vt, fu, vq   qm: fu, ut, fv, uq   qq: ke
// gpin field kinds: gtn 0, gqn 1, gut 2, gvt 3, guz 4, gvz 5, gke 6, gvpp 7, guq 8, gvq 9;
// mktend call: tn=gtn, fu=gvz, fv=guz, ke=gke, ut=gut, vt=gvt; qtend: qn=gqn, uq=guq, vq=gvq
__device__ __constant__ int c_fwd_nf[4] = {2, 4, 4, 1};
__device__ __constant__ int c_fwd_fields[4][4] = {{0, 1, -1, -1}, {4, 3, 5, 9}, {5, 2, 4, 8}, {6, -1, -1, -1}};
template <int NLT> __host__ __device__ constexpr int fwd_ncol(int t) {
    return t == 0 ? 2 * NLT * 2 + 2 : (t == 3 ? NLT * 2 : 4 * NLT * 2);
}
template <int NLT> __host__ __device__ constexpr int fwd_ncp(int t) { return (fwd_ncol<NLT>(t) + 15) & ~15; }
template <int NLT> __host__ __device__ constexpr int fwd_colbase(int t) {
    return t == 0 ? 0 : fwd_colbase<NLT>(t - 1) + 4 * fwd_ncp<NLT>(t - 1);  // 2 parities x (main, correction)
}
// TMEM loads of 16 or 32 columns without the wait
template <int NC> __device__ __forceinline__ void tmem_ld_nw(uint32_t taddr, uint32_t *r) {
    if constexpr (NC >= 32) tc::tmem_ld32_nw(taddr, r);
    else tc::tmem_ld16_nw(taddr, r);
}

__device__ __forceinline__ long long fwd_row(int L, int inst, int kind, int l) {
    const int nfi = 9 * L + 1;
    int F;
    if (kind == 7) F = 7 * L;
    else if (kind < 7) F = kind * L + l;
    else F = 7 * L + 1 + (kind - 8) * L + l;
    return (long long)inst * nfi + F;
}

template <int NLT>
__global__ void __launch_bounds__(TCT2) k_tc_forward(const __grid_constant__ TcFwdLaunch P) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int4 jb = P.jobs[blockIdx.x];
    const TcFwdArgs &A = P.seg[jb.y >> 16];
    const int nprod = P.nprod;
    const int m = jb.x, inst = jb.y & 0xffff, l0 = jb.z, nl = jb.w;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, quarter = warp & 3, half = warp >> 2;
    const int K = A.ntp1 - m;
    const int Kq[2] = {kpar(K, 0), kpar(K, 1)};
    const int R[2] = {pad8(Kq[0]), pad8(Kq[1])};
    const int njc = A.njc, L = A.L, nlat = A.nlat;
    const bool with_vpp = (l0 == 0);
    const bool onebuf = P.onebuf != 0;
    // a table block is [parity 0: 3 splits x R0 rows][parity 1: 3 splits x R1 rows];
    // the halves travel separately, into two buffers so the next table's half 0
    // lands while half 1 computes, or (large grids) one after the other into one
    const uint32_t hbytes[2] = {(uint32_t)(3 * R[0] * njc * 2), (uint32_t)(3 * R[1] * njc * 2)};
    const uint32_t hoff[2] = {0u, hbytes[0]};                 // in the global block
    const uint32_t soff[2] = {0u, onebuf ? 0u : hbytes[0]};   // in shared memory
    const size_t tregion = onebuf ? hbytes[0] : (size_t)hbytes[0] + hbytes[1];
    // rows >= R of the M=128 table tiles read past the block: keep a margin
    // before the data so those reads (whose TMEM lanes are never used) stay in bounds
    unsigned char *tab = sm;
    unsigned char *dat = sm + tregion + 128 * 32 * 2;
    size_t doffs[4], dbytes = 0;
    for (int t = 0; t < 4; t++) { doffs[t] = dbytes; dbytes += 2 * 3 * (size_t)fwd_ncp<NLT>(t) * njc * 2; }
    unsigned char *tail = dat + dbytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>((reinterpret_cast<uintptr_t>(tail) + 15) & ~(uintptr_t)15);
    uint64_t *bar_tma = bars;       // [2] table half of parity p landed
    uint64_t *bar_mma = bars + 2;   // [2] MMAs reading table half p completed
    uint64_t *bar_done = bars + 4;  // every MMA completed
    uint32_t *slot = reinterpret_cast<uint32_t *>(bars + 5);
    if (warp == 0) tc::tmem_alloc(slot, 512);
    if (tid == 0) {
        for (int i = 0; i < 5; i++) tc::mbar_init(bars + i, 1);
        tc::mbar_fence_init();
        for (int p = 0; p < 2; p++)
            if (Kq[p] && (p == 0 || !onebuf)) {
                tc::mbar_arrive_expect_tx(bar_tma + p, hbytes[p]);
                tc::bulk_g2s(tab + soff[p], A.tab + A.off[m * 4 + 0] + hoff[p], hbytes[p], bar_tma + p);
            }
    }
    // stage folded Fourier columns: for each table, S (= N+S) and D (= N-S)
    // versions.  A unit is one column pair (re, im of one field-level) and 8
    // latitude pairs: 16-byte loads of the north and south rows, and one
    // 16-byte core-matrix row per column, split term and version.
    const int ng = njc >> 3;
    for (int t = 0; t < 4; t++) {
        const int nf = c_fwd_nf[t];
        const int ncp = fwd_ncp<NLT>(t), npair = ncp >> 1;
        const int nreal = nf * NLT + ((t == 0) ? 1 : 0);  // column pairs in use (incl. padding levels)
        const uint32_t dt = (uint32_t)ncp * njc * 2;       // one split tile
        unsigned char *bS = dat + doffs[t], *bD = bS + 3 * dt;
        const int nunit = npair * ng;
        for (int u = tid; u < nunit; u += TCT2) {
            const int q = u % npair, g = u / npair;
            long long rb = -1;
            if (q < nreal) {
                if (t == 0 && q == nf * NLT) { if (with_vpp) rb = fwd_row(L, inst, 7, 0); }
                else {
                    const int fi = q / NLT, li = q - fi * NLT;
                    if (li < nl) rb = fwd_row(L, inst, c_fwd_fields[t][fi], l0 + li);
                }
            }
            const int j0 = 8 * g;
            float sr[8], si[8], dr[8], di[8];
            float2 vn[8], vs[8];
#pragma unroll
            for (int e = 0; e < 8; e++) vn[e] = vs[e] = make_float2(0.f, 0.f);
            if (rb >= 0) {
                const float2 *wr = A.W + (size_t)m * A.nrows + (size_t)rb * nlat;
                if (j0 + 8 <= A.nlath) {
                    // rows j0..j0+7 north, and nlat-8-j0..nlat-1-j0 south (reversed)
                    const float4 *pn = reinterpret_cast<const float4 *>(wr + j0);
                    const float4 *ps = reinterpret_cast<const float4 *>(wr + nlat - 8 - j0);
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float4 x = __ldg(pn + i), y = __ldg(ps + i);
                        vn[2 * i] = make_float2(x.x, x.y);
                        vn[2 * i + 1] = make_float2(x.z, x.w);
                        vs[7 - 2 * i] = make_float2(y.x, y.y);
                        vs[6 - 2 * i] = make_float2(y.z, y.w);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 8; e++)
                        if (j0 + e < A.nlath) {
                            vn[e] = __ldg(wr + j0 + e);
                            vs[e] = __ldg(wr + nlat - 1 - j0 - e);
                        }
                }
            }
#pragma unroll
            for (int e = 0; e < 8; e++) {
                sr[e] = vn[e].x + vs[e].x;
                si[e] = vn[e].y + vs[e].y;
                dr[e] = vn[e].x - vs[e].x;
                di[e] = vn[e].y - vs[e].y;
            }
            const uint32_t o = tc::kmajor_off(2 * q, j0, njc);  // re row; the im row follows at +16
            uint4 h, mm, l;
            tc::split3x8(sr, h, mm, l);
            st_shared16(bS + o, h); st_shared16(bS + dt + o, mm); st_shared16(bS + 2 * dt + o, l);
            tc::split3x8(si, h, mm, l);
            st_shared16(bS + o + 16, h); st_shared16(bS + dt + o + 16, mm); st_shared16(bS + 2 * dt + o + 16, l);
            tc::split3x8(dr, h, mm, l);
            st_shared16(bD + o, h); st_shared16(bD + dt + o, mm); st_shared16(bD + 2 * dt + o, l);
            tc::split3x8(di, h, mm, l);
            st_shared16(bD + o + 16, h); st_shared16(bD + dt + o + 16, mm); st_shared16(bD + 2 * dt + o + 16, l);
        }
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    bool ok = true;
    if (tid == 0) {
        const uint32_t sbo_b = (uint32_t)(njc / 8) * 128;
        int u = 0;  // table-half units issued (one-buffer mode)
        for (int t = 0; t < 4 && ok; t++) {
            const int ncp = fwd_ncp<NLT>(t);
            const uint32_t idesc = tc::idesc_bf16(128, ncp);
            const uint32_t dt = (uint32_t)ncp * njc * 2;
            // P-type (qc, qm, qq) use N+S on even n-m and N-S on odd; Q-type (qe) the reverse
            const bool ptype = (t != 1);
            for (int p = 0; p < 2 && ok; p++) {
                if (!Kq[p]) break;
                ok = onebuf ? tc::mbar_wait(bar_tma, u & 1) : tc::mbar_wait(bar_tma + p, t & 1);
                if (!ok) break;
                tc::fence_after_sync();
                const int sel = ptype ? p : 1 - p;  // 0 -> S, 1 -> D
                const uint64_t db0 = tc::smem_desc(dat + doffs[t] + (size_t)sel * 3 * dt, 128, sbo_b);
                const uint32_t dm = tmem + (uint32_t)(fwd_colbase<NLT>(t) + (2 * p + 0) * ncp);
                const uint32_t dc = tmem + (uint32_t)(fwd_colbase<NLT>(t) + (2 * p + 1) * ncp);
                uint32_t jo = 0;
                for (int j0 = 0; j0 < njc; j0 += 32) {
                    const int jw = njc - j0 < 32 ? njc - j0 : 32;
                    const uint32_t tt = (uint32_t)R[p] * jw * 2;
                    const uint64_t da0 = tc::smem_desc(tab + soff[p] + jo, 128, (uint32_t)(jw / 8) * 128);
                    for (int kc = 0; kc < jw / 16; kc++) {
#pragma unroll
                        for (int pr = 0; pr < 6; pr++)
                            if (pr < nprod)
                                tc::mma_bf16(pr == 0 ? dm : dc, tc::desc_add(da0, tc::pair_a(pr) * tt + kc * 256),
                                             tc::desc_add(db0, tc::pair_b(pr) * dt + (j0 / 8) * 128 + kc * 256),
                                             idesc, j0 > 0 || kc > 0 || pr > 1);
                    }
                    jo += 3 * tt;
                }
                if (onebuf) {
                    // the next half may overwrite the buffer once these MMAs have read it
                    const bool last = t == 3 && (p == 1 || !Kq[1]);
                    if (!last) {
                        tc::mma_commit(bar_mma);
                        ok = tc::mbar_wait(bar_mma, u & 1);
                        if (ok) {
                            const int tn = (p == 0 && Kq[1]) ? t : t + 1, pn = (p == 0 && Kq[1]) ? 1 : 0;
                            tc::mbar_arrive_expect_tx(bar_tma, hbytes[pn]);
                            tc::bulk_g2s(tab, A.tab + A.off[m * 4 + tn] + hoff[pn], hbytes[pn], bar_tma);
                        }
                    }
                    u++;
                } else if (t < 3) {
                    tc::mma_commit(bar_mma + p);
                }
            }
            // refill each half with the next table once its MMAs have drained
            for (int p = 0; p < 2 && ok && t < 3 && !onebuf; p++) {
                if (!Kq[p]) break;
                ok = tc::mbar_wait(bar_mma + p, t & 1);
                if (!ok) break;
                tc::mbar_arrive_expect_tx(bar_tma + p, hbytes[p]);
                tc::bulk_g2s(tab + hoff[p], A.tab + A.off[m * 4 + t + 1] + hoff[p], hbytes[p], bar_tma + p);
            }
        }
        if (ok) tc::mma_commit(bar_done);  // arrives once every MMA issued above has completed
        if (!ok) atomicExch(&g_tc_error, 3);
    }
    __syncthreads();
    ok = __all_sync(0xffffffffu, tc::mbar_wait(bar_done, 0));  // warp-uniform for the .sync.aligned TMEM loads
    if (!ok && lane == 0) atomicExch(&g_tc_error, 4);
    tc::fence_after_sync();
    // epilogue: warp half h drains parity h; TMEM lane = mode index k'
    const int p = half;
    if (ok && Kq[p]) {
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        const int kk = quarter * 32 + lane;
        const bool valid = kk < Kq[p];
        // outputs per level: d, t, z, q (re, im)
        float od[NLT][2], ot[NLT][2], oz[NLT][2], oq[NLT][2], ov[2] = {0.f, 0.f};
#pragma unroll
        for (int li = 0; li < NLT; li++)
            for (int ri = 0; ri < 2; ri++) od[li][ri] = ot[li][ri] = oz[li][ri] = oq[li][ri] = 0.f;
        uint32_t rm[32], rc[32];
        float v[32];
        // table qc (t=0): tn -> t, qn -> q, gvpp -> spf
        tmem_ld_nw<fwd_ncp<NLT>(0)>(tmem + lane_addr + (uint32_t)(fwd_colbase<NLT>(0) + (2 * p) * fwd_ncp<NLT>(0)), rm);
        tmem_ld_nw<fwd_ncp<NLT>(0)>(tmem + lane_addr + (uint32_t)(fwd_colbase<NLT>(0) + (2 * p + 1) * fwd_ncp<NLT>(0)), rc);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 32; i++) v[i] = i < fwd_ncp<NLT>(0) ? __uint_as_float(rm[i]) + __uint_as_float(rc[i]) : 0.f;
#pragma unroll
        for (int li = 0; li < NLT; li++) {
            ot[li][0] += v[(0 * NLT + li) * 2]; ot[li][1] += v[(0 * NLT + li) * 2 + 1];
            oq[li][0] += v[(1 * NLT + li) * 2]; oq[li][1] += v[(1 * NLT + li) * 2 + 1];
        }
        ov[0] = v[2 * NLT * 2]; ov[1] = v[2 * NLT * 2 + 1];
        // table qe (t=1): fv -> d (-), vt -> t, fu -> z, vq -> q
        tmem_ld_nw<fwd_ncp<NLT>(1)>(tmem + lane_addr + (uint32_t)(fwd_colbase<NLT>(1) + (2 * p) * fwd_ncp<NLT>(1)), rm);
        tmem_ld_nw<fwd_ncp<NLT>(1)>(tmem + lane_addr + (uint32_t)(fwd_colbase<NLT>(1) + (2 * p + 1) * fwd_ncp<NLT>(1)), rc);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 32; i++) v[i] = i < fwd_ncp<NLT>(1) ? __uint_as_float(rm[i]) + __uint_as_float(rc[i]) : 0.f;
#pragma unroll
        for (int li = 0; li < NLT; li++)
#pragma unroll
            for (int ri = 0; ri < 2; ri++) {
                od[li][ri] -= v[(0 * NLT + li) * 2 + ri];
                ot[li][ri] += v[(1 * NLT + li) * 2 + ri];
                oz[li][ri] += v[(2 * NLT + li) * 2 + ri];
                oq[li][ri] += v[(3 * NLT + li) * 2 + ri];
            }
        // table qm (t=2): i*fu -> d, -i*ut -> t, i*fv -> z, -i*uq -> q  (i*(a+ib) = -b + ia)
        tmem_ld_nw<fwd_ncp<NLT>(2)>(tmem + lane_addr + (uint32_t)(fwd_colbase<NLT>(2) + (2 * p) * fwd_ncp<NLT>(2)), rm);
        tmem_ld_nw<fwd_ncp<NLT>(2)>(tmem + lane_addr + (uint32_t)(fwd_colbase<NLT>(2) + (2 * p + 1) * fwd_ncp<NLT>(2)), rc);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 32; i++) v[i] = i < fwd_ncp<NLT>(2) ? __uint_as_float(rm[i]) + __uint_as_float(rc[i]) : 0.f;
#pragma unroll
        for (int li = 0; li < NLT; li++) {
            const float fur = v[(0 * NLT + li) * 2], fui = v[(0 * NLT + li) * 2 + 1];
            const float utr = v[(1 * NLT + li) * 2], uti = v[(1 * NLT + li) * 2 + 1];
            const float fvr = v[(2 * NLT + li) * 2], fvi = v[(2 * NLT + li) * 2 + 1];
            const float uqr = v[(3 * NLT + li) * 2], uqi = v[(3 * NLT + li) * 2 + 1];
            od[li][0] -= fui; od[li][1] += fur;
            ot[li][0] += uti; ot[li][1] -= utr;
            oz[li][0] -= fvi; oz[li][1] += fvr;
            oq[li][0] += uqi; oq[li][1] -= uqr;
        }
        // table qq (t=3): ke -> d
        tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(fwd_colbase<NLT>(3) + (2 * p) * fwd_ncp<NLT>(3)), rm);
        tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(fwd_colbase<NLT>(3) + (2 * p + 1) * fwd_ncp<NLT>(3)), rc);
        tc::tmem_wait_ld();
#pragma unroll
        for (int li = 0; li < NLT; li++) {
            od[li][0] += __uint_as_float(rm[2 * li]) + __uint_as_float(rc[2 * li]);
            od[li][1] += __uint_as_float(rm[2 * li + 1]) + __uint_as_float(rc[2 * li + 1]);
        }
        if (valid) {
            const int k = 2 * kk + p;  // n - m
            const float fl = A.filt[m + k];
            const size_t wo = 2 * (size_t)(A.woff[m] + k);
            const int nfo = 4 * L + 1;
#pragma unroll
            for (int li = 0; li < NLT; li++) {
                if (li >= nl) break;
                const int l = l0 + li;
                float2 *sd = reinterpret_cast<float2 *>(A.spout + ((size_t)inst * nfo + l) * A.nrsp + wo);
                float2 *st = reinterpret_cast<float2 *>(A.spout + ((size_t)inst * nfo + L + l) * A.nrsp + wo);
                float2 *sz = reinterpret_cast<float2 *>(A.spout + ((size_t)inst * nfo + 2 * L + l) * A.nrsp + wo);
                float2 *sq = reinterpret_cast<float2 *>(A.spout + ((size_t)inst * nfo + 3 * L + l) * A.nrsp + wo);
                *sd = make_float2(od[li][0] * fl, od[li][1] * fl);
                *st = make_float2(ot[li][0] * fl, ot[li][1] * fl);
                *sz = make_float2(oz[li][0] * fl, oz[li][1] * fl);
                *sq = make_float2(oq[li][0] * fl, oq[li][1] * fl);
            }
            if (with_vpp) {
                float2 *sp = reinterpret_cast<float2 *>(A.spout + ((size_t)inst * nfo + 4 * L) * A.nrsp + wo);
                *sp = make_float2(ov[0] * fl, ov[1] * fl);
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

static int fwd_ncp_rt(int nlt, int t) {
    const int c = t == 0 ? 4 * nlt + 2 : (t == 3 ? 2 * nlt : 8 * nlt);
    return (c + 15) & ~15;
}
// shared memory of a forward job at the widest m (K = NTP1 modes)
static size_t fwd_smem(int K, int njc, int nlt, bool onebuf) {
    size_t h[2] = {0, 0};
    for (int p = 0; p < 2; p++) {
        const int Kq = kpar(K, p);
        if (Kq) h[p] = 3 * (size_t)pad8(Kq) * njc * 2;
    }
    const size_t tblk = onebuf ? std::max(h[0], h[1]) : h[0] + h[1];
    size_t d = 0;
    for (int t = 0; t < 4; t++) d += 2 * 3 * (size_t)fwd_ncp_rt(nlt, t) * njc * 2;
    return tblk + 128 * 32 * 2 + d + 80;
}

// ------------------------------------------------------------ forward, stacked splits
// Variant for NTRU+1 <= 128 (every parity has at most 64 modes): one parity per
// job, and the table's split terms stacked in the M=128 tile so that two MMAs
// per K-chunk cover all six split products.  Per (m, table, parity) and
// latitude chunk the table holds two 2R-row K-major tiles:
//   S01 = [a0 of modes 0..R-1 ; a1 of modes 0..R-1],   S2 = [0 ; a2]
// and the data of the table's columns is staged as [b0 | b1 | b2] (N-adjacent):
//   MMA1  [X0|X1|X2] (+)= S01 x [b0|b1|b2]   (N = 3 ncp)
//   MMA2   X0        +=  S2  x  b0           (N = ncp)
// Row k' < R of X0 is the hi*hi chain alone; every other entry of rows k' and
// R+k' is a correction product.  The mode's value is the sum of both rows'
// three blocks; the rows meet in shared memory in the epilogue.
struct TcFwd3Args {
    const unsigned char *tab;
    const long long *off;   // [(m*4 + t)*2 + p]
    const int *woff;
    const float2 *W;
    long long nrows;
    const float *filt;
    float *spout;
    int L, nlat, nlath, njc, ntp1, nrsp;
};
struct TcFwd3Launch {
    TcFwd3Args seg[TC_MAXSEG];
    const int4 *jobs;       // (m, inst | seg << 16, first level, levels | parity << 8)
    int nprod;              // 6: all six products; 3: a0b0, a0b1, a1b0 (and a1b1)
};
template <int NLT> __host__ __device__ constexpr int f3_colbase(int t) {
    return t == 0 ? 0 : f3_colbase<NLT>(t - 1) + 3 * fwd_ncp<NLT>(t - 1);
}
constexpr int F3_NLT = 5;   // levels per job: 3 x (32 + 48 + 48 + 16) = 432 TMEM columns

// partial outputs of one table's columns: d, t, z, q per level (re, im) and spf
template <int NLT>
__device__ __forceinline__ void f3_combine(int t, int c, float v, float (*o)[4][2], float *ov) {
    const int q = c >> 1, ri = c & 1;
    if (t == 0) {
        if (q == 2 * NLT) { ov[ri] += v; return; }
        if (q >= 2 * NLT) return;
        const int fi = q / NLT, li = q - fi * NLT;
        o[li][fi == 0 ? 1 : 3][ri] += v;             // tn -> t, qn -> q
    } else if (t == 1) {
        if (q >= 4 * NLT) return;
        const int fi = q / NLT, li = q - fi * NLT;
        if (fi == 0) o[li][0][ri] -= v;              // fv -> d (-)
        else if (fi == 1) o[li][1][ri] += v;         // vt -> t
        else if (fi == 2) o[li][2][ri] += v;         // fu -> z
        else o[li][3][ri] += v;                      // vq -> q
    } else if (t == 2) {
        if (q >= 4 * NLT) return;
        const int fi = q / NLT, li = q - fi * NLT;
        // i*(a + ib) = -b + ia: the real column feeds im, the imaginary feeds re
        const float sgn = (fi == 0 || fi == 2) ? 1.f : -1.f;   // +i for fu, fv; -i for ut, uq
        const int out = fi == 0 ? 0 : fi == 1 ? 1 : fi == 2 ? 2 : 3;
        if (ri == 0) o[li][out][1] += sgn * v;
        else o[li][out][0] -= sgn * v;
    } else {
        if (q >= NLT) return;
        o[q][0][ri] += v;                            // ke -> d
    }
}

// load the north and south rows of one staging unit (column pair u % npair of
// table t, latitude pairs 8 (u / npair) ..+7); zeros outside the job
template <int NLT>
__device__ __forceinline__ void f3_load(const TcFwd3Args &A, int m, int inst, int l0, int nl, bool with_vpp, int t,
                                        int u, float2 *vn, float2 *vs) {
    const int nf = c_fwd_nf[t];
    const int npair = fwd_ncp<NLT>(t) >> 1, ng = A.njc >> 3;
    const int nreal = nf * NLT + ((t == 0) ? 1 : 0);
    const int q = u % npair, g = u / npair;
    long long rb = -1;
    if (g < ng && q < nreal) {
        if (t == 0 && q == nf * NLT) { if (with_vpp) rb = fwd_row(A.L, inst, 7, 0); }
        else {
            const int fi = q / NLT, li = q - fi * NLT;
            if (li < nl) rb = fwd_row(A.L, inst, c_fwd_fields[t][fi], l0 + li);
        }
    }
#pragma unroll
    for (int e = 0; e < 8; e++) vn[e] = vs[e] = make_float2(0.f, 0.f);
    if (rb < 0) return;
    const int nlat = A.nlat, j0 = 8 * g;
    const float2 *wr = A.W + (size_t)m * A.nrows + (size_t)rb * nlat;
    if (j0 + 8 <= A.nlath) {
        // rows j0..j0+7 north, and nlat-8-j0..nlat-1-j0 south (reversed)
        const float4 *pn = reinterpret_cast<const float4 *>(wr + j0);
        const float4 *ps = reinterpret_cast<const float4 *>(wr + nlat - 8 - j0);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float4 x = __ldg(pn + i), y = __ldg(ps + i);
            vn[2 * i] = make_float2(x.x, x.y);
            vn[2 * i + 1] = make_float2(x.z, x.w);
            vs[7 - 2 * i] = make_float2(y.x, y.y);
            vs[6 - 2 * i] = make_float2(y.z, y.w);
        }
    } else {
#pragma unroll
        for (int e = 0; e < 8; e++)
            if (j0 + e < A.nlath) {
                vn[e] = __ldg(wr + j0 + e);
                vs[e] = __ldg(wr + nlat - 1 - j0 - e);
            }
    }
}

// fold a loaded unit for parity p, split it into three BF16 terms and store
// the re and im core-matrix rows of every term
template <int NLT>
__device__ __forceinline__ void f3_store(int t, int p, int u, int njc, unsigned char *bt, const float2 *vn,
                                         const float2 *vs) {
    const int ncp = fwd_ncp<NLT>(t), npair = ncp >> 1;
    const int q = u % npair, g = u / npair;
    const bool diff = (t != 1) ? (p == 1) : (p == 0);
    float xr[8], xi[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
        xr[e] = diff ? vn[e].x - vs[e].x : vn[e].x + vs[e].x;
        xi[e] = diff ? vn[e].y - vs[e].y : vn[e].y + vs[e].y;
    }
    const uint32_t dt = (uint32_t)ncp * njc * 2;
    const uint32_t o = tc::kmajor_off(2 * q, 8 * g, njc);
    uint4 h, mm, l;
    tc::split3x8(xr, h, mm, l);
    st_shared16(bt + o, h); st_shared16(bt + dt + o, mm); st_shared16(bt + 2 * dt + o, l);
    tc::split3x8(xi, h, mm, l);
    st_shared16(bt + o + 16, h); st_shared16(bt + dt + o + 16, mm); st_shared16(bt + 2 * dt + o + 16, l);
}

// sum the split blocks of table T's accumulator columns for this thread's TMEM
// row and fold them into the partial outputs
template <int NLT, int T>
__device__ __forceinline__ void f3_drain(uint32_t taddr, int nprod, float (*o)[4][2], float *ov) {
    constexpr int ncp = fwd_ncp<NLT>(T);
    const uint32_t X = taddr + (uint32_t)f3_colbase<NLT>(T);
#pragma unroll
    for (int c0 = 0; c0 < ncp; c0 += 16) {
        uint32_t x0[16], x1[16], x2[16];
        tc::tmem_ld16_nw(X + c0, x0);
        tc::tmem_ld16_nw(X + ncp + c0, x1);
        if (nprod == 6) tc::tmem_ld16_nw(X + 2 * ncp + c0, x2);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; i++) {
            float v = __uint_as_float(x0[i]) + __uint_as_float(x1[i]);
            if (nprod == 6) v += __uint_as_float(x2[i]);
            f3_combine<NLT>(T, c0 + i, v, o, ov);
        }
    }
}

// 16 warps: warp 0 issues copies and MMAs, warps 1-15 stage operands (the
// staging loads are latency-bound, so more warps keep more of them in flight),
// warps 0-3 drain TMEM
constexpr int TCT3 = 512;

template <int NLT>
__global__ void __launch_bounds__(TCT3) k_tc_forward3(const __grid_constant__ TcFwd3Launch P) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int4 jb = P.jobs[blockIdx.x];
    const TcFwd3Args &A = P.seg[jb.y >> 16];
    const int nprod = P.nprod;
    const int m = jb.x, inst = jb.y & 0xffff, l0 = jb.z, nl = jb.w & 0xff, p = jb.w >> 8;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, quarter = warp & 3;
    const int K = A.ntp1 - m;
    const int Kq = kpar(K, p), R = pad8(Kq);
    const int njc = A.njc, L = A.L;
    const bool with_vpp = (l0 == 0);
    const uint32_t tbytes = (uint32_t)8 * R * njc;   // one (m, table, parity) block
    const uint32_t tbuf = (uint32_t)8 * 64 * njc;    // buffer for the widest block
    unsigned char *tabb[2] = {sm, sm + tbuf};
    // rows >= 2R of the M=128 tiles read past a block (their TMEM lanes are unused)
    unsigned char *dat = sm + 2 * tbuf + 128 * 32 * 2;
    size_t doffs[4], dbytes = 0;
    for (int t = 0; t < 4; t++) { doffs[t] = dbytes; dbytes += 3 * (size_t)fwd_ncp<NLT>(t) * njc * 2; }
    // the epilogue's partial outputs reuse the table and operand space; the
    // barriers lie past both
    constexpr int NO = NLT * 8 + 2;
    constexpr size_t ebytes = 4 * 128 * NO * sizeof(float);
    unsigned char *tail = (size_t)(dat + dbytes - sm) > ebytes ? dat + dbytes : sm + ebytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>((reinterpret_cast<uintptr_t>(tail) + 15) & ~(uintptr_t)15);
    uint64_t *bar_tma = bars;       // [2] table buffer b landed
    uint64_t *bar_mma = bars + 2;   // [2] MMAs reading table buffer b completed
    uint64_t *bar_done = bars + 4;
    uint64_t *bar_stage = bars + 5; // [4] operands of table t staged (warps 1-15 arrive)
    uint32_t *slot = reinterpret_cast<uint32_t *>(bars + 9);
    if (warp == 0) tc::tmem_alloc(slot, 512);
    if (tid == 0) {
        for (int i = 0; i < 5; i++) tc::mbar_init(bars + i, 1);
        for (int t = 0; t < 4; t++) tc::mbar_init(bar_stage + t, TCT3 - 32);
        tc::mbar_fence_init();
        for (int t = 0; t < 2; t++) {
            tc::mbar_arrive_expect_tx(bar_tma + t, tbytes);
            tc::bulk_g2s(tabb[t], A.tab + A.off[(m * 4 + t) * 2 + p], tbytes, bar_tma + t);
        }
    }
    tc::fence_before_sync();
    __syncthreads();  // barriers initialised, TMEM address published
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    bool ok = true;
    // warps 1-15 stage the folded columns each table needs for this parity,
    // table by table, while warp 0 issues the MMAs of every table already
    // staged.  P-type tables (qc, qm, qq) take N+S on even n-m and N-S on odd,
    // Q-type (qe) the reverse.  A unit (column pair, 8 latitude pairs) of the
    // next table is loaded before the current one is split and stored, so the
    // loads of successive tables overlap.
    if (warp != 0) {
        const int stid = tid - 32;
        float2 vn[8], vs[8];
        f3_load<NLT>(A, m, inst, l0, nl, with_vpp, 0, stid, vn, vs);
        for (int t = 0; t < 4; t++) {
            const int nunit = (fwd_ncp<NLT>(t) >> 1) * (njc >> 3);
            float2 wn[8], ws[8];
            if (t + 1 < 4) f3_load<NLT>(A, m, inst, l0, nl, with_vpp, t + 1, stid, wn, ws);
            if (stid < nunit) f3_store<NLT>(t, p, stid, njc, dat + doffs[t], vn, vs);
            // more units than staging threads (not at NLAT <= 192, where every table has fewer)
            for (int u = stid + (TCT3 - 32); u < nunit; u += TCT3 - 32) {
                f3_load<NLT>(A, m, inst, l0, nl, with_vpp, t, u, vn, vs);
                f3_store<NLT>(t, p, u, njc, dat + doffs[t], vn, vs);
            }
            tc::fence_proxy_async();  // these stores feed the tensor cores
            tc::mbar_arrive(bar_stage + t);
#pragma unroll
            for (int e = 0; e < 8; e++) { vn[e] = wn[e]; vs[e] = ws[e]; }
        }
    }
    if (tid == 0) {
        const uint32_t sbo_b = (uint32_t)(njc / 8) * 128;
        for (int t = 0; t < 4 && ok; t++) {
            const int b = t & 1;
            ok = tc::mbar_wait(bar_stage + t, 0) && tc::mbar_wait(bar_tma + b, (t >> 1) & 1);
            if (!ok) break;
            tc::fence_after_sync();
            const int ncp = fwd_ncp<NLT>(t);
            const uint32_t idesc1 = tc::idesc_bf16(128, (nprod == 6 ? 3 : 2) * ncp);
            const uint32_t idesc2 = tc::idesc_bf16(128, ncp);
            const uint32_t X = tmem + (uint32_t)f3_colbase<NLT>(t);
            const uint64_t db = tc::smem_desc(dat + doffs[t], 128, sbo_b);
            uint32_t jo = 0;
            for (int j0 = 0; j0 < njc; j0 += 32) {
                const int jw = njc - j0 < 32 ? njc - j0 : 32;
                const uint32_t tt = (uint32_t)2 * R * jw * 2;   // one stacked tile
                const uint64_t da1 = tc::smem_desc(tabb[b] + jo, 128, (uint32_t)(jw / 8) * 128);
                const uint64_t da2 = tc::desc_add(da1, tt);
                for (int kc = 0; kc < jw / 16; kc++) {
                    const uint64_t dbk = tc::desc_add(db, (j0 / 8) * 128 + kc * 256);
                    tc::mma_bf16(X, tc::desc_add(da1, kc * 256), dbk, idesc1, j0 > 0 || kc > 0);
                    if (nprod == 6) tc::mma_bf16(X, tc::desc_add(da2, kc * 256), dbk, idesc2, true);
                }
                jo += 2 * tt;
            }
            if (t <= 1) tc::mma_commit(bar_mma + b);
            // refill the other buffer with table t+1 once table t-1's MMAs have read it
            if (t >= 1 && t + 1 < 4) {
                const int bn = (t + 1) & 1;
                ok = tc::mbar_wait(bar_mma + bn, 0);
                if (!ok) break;
                tc::mbar_arrive_expect_tx(bar_tma + bn, tbytes);
                tc::bulk_g2s(tabb[bn], A.tab + A.off[(m * 4 + t + 1) * 2 + p], tbytes, bar_tma + bn);
            }
        }
        if (ok) tc::mma_commit(bar_done);
        if (!ok) atomicExch(&g_tc_error, 5);
    }
    __syncthreads();
    ok = __all_sync(0xffffffffu, tc::mbar_wait(bar_done, 0));  // warp-uniform for the .sync.aligned TMEM loads
    if (!ok && lane == 0) atomicExch(&g_tc_error, 6);
    tc::fence_after_sync();
    // epilogue: warp w drains table w / 4 for TMEM lane quarter w % 4.  Row r
    // holds mode r (r < R) or corrections of mode r - R (R <= r < 2R); every
    // (table, row) hands its partial outputs to shared memory, and the sums
    // over tables and both rows of a mode are formed there.
    float *E = reinterpret_cast<float *>(sm);   // [4][128][NO]; tables and operands are dead now
    const int r = quarter * 32 + lane;
    const int gw = warp >> 2;
    if (ok && quarter * 32 < 2 * R) {           // warp-uniform (ok is)
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        float o[NLT][4][2], ov[2] = {0.f, 0.f};
#pragma unroll
        for (int li = 0; li < NLT; li++)
#pragma unroll
            for (int k = 0; k < 4; k++) o[li][k][0] = o[li][k][1] = 0.f;
        if (gw == 0) f3_drain<NLT, 0>(tmem + lane_addr, nprod, o, ov);
        else if (gw == 1) f3_drain<NLT, 1>(tmem + lane_addr, nprod, o, ov);
        else if (gw == 2) f3_drain<NLT, 2>(tmem + lane_addr, nprod, o, ov);
        else f3_drain<NLT, 3>(tmem + lane_addr, nprod, o, ov);
        if (r < 2 * R) {
            float *e = E + (size_t)(gw * 128 + r) * NO;
#pragma unroll
            for (int li = 0; li < NLT; li++)
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    e[(li * 4 + k) * 2] = o[li][k][0];
                    e[(li * 4 + k) * 2 + 1] = o[li][k][1];
                }
            e[NLT * 8] = ov[0];
            e[NLT * 8 + 1] = ov[1];
        }
    }
    __syncthreads();
    if (ok) {
        // outputs: Kq modes x (4 fields x NLT levels + spf); consecutive threads take consecutive modes
        const int nout = 4 * NLT + 1, nfo = 4 * L + 1;
        const size_t wb = (size_t)A.woff[m];
        for (int idx = tid; idx < Kq * nout; idx += TCT3) {
            const int oi = idx / Kq, rr = idx - oi * Kq;
            size_t fr;                                   // output field row
            if (oi < 4 * NLT) {
                const int li = oi >> 2, kk = oi & 3;
                if (li >= nl) continue;
                fr = (size_t)inst * nfo + kk * L + l0 + li;
            } else {
                if (!with_vpp) continue;
                fr = (size_t)inst * nfo + 4 * L;
            }
            float sr = 0.f, si = 0.f;
#pragma unroll
            for (int g = 0; g < 4; g++) {
                const float *e0 = E + (size_t)(g * 128 + rr) * NO + 2 * oi;
                const float *e1 = E + (size_t)(g * 128 + R + rr) * NO + 2 * oi;
                sr += e0[0] + e1[0];
                si += e0[1] + e1[1];
            }
            const int k = 2 * rr + p;                    // n - m
            const float fl = A.filt[m + k];
            reinterpret_cast<float2 *>(A.spout + fr * A.nrsp)[wb + k] = make_float2(sr * fl, si * fl);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

static size_t fwd3_smem(int njc, int nlt) {
    size_t d = 0;
    for (int t = 0; t < 4; t++) d += 3 * (size_t)fwd_ncp_rt(nlt, t) * njc * 2;
    const size_t ops = 2 * (size_t)8 * 64 * njc + 128 * 32 * 2 + d;
    const size_t ebytes = 4 * 128 * (size_t)(nlt * 8 + 2) * sizeof(float);
    return std::max(ops, ebytes) + 128;
}
