// Tensor-core Legendre kernels (included by legendre_tc.cu).
//
// One CTA per job.  Thread 0 issues the TMA table copies and the MMAs; the
// other threads stage operands and drain accumulators.  Warps w, w+4, ...
// share TMEM lane quarter w % 4.
#pragma once

constexpr int TCT2 = 256;

__device__ __forceinline__ void st_shared16(unsigned char *p, uint4 v) { *reinterpret_cast<uint4 *>(p) = v; }
__device__ __forceinline__ void st_shared4(unsigned char *p, uint32_t v) { *reinterpret_cast<uint32_t *>(p) = v; }
__device__ __forceinline__ void st_shared8(unsigned char *p, uint2 v) { *reinterpret_cast<uint2 *>(p) = v; }

// ------------------------------------------------------------ inverse
struct TcInvArgs {
    const unsigned char *tab;
    const long long *off;
    const int *woff;
    const float *spin;      // [inst][4L+1][NRSP]
    const float *filt;      // skspgp (unused: folded into the tables)
    float2 *W;              // [m][row], row = (inst*(6L+3) + field)*nlat + lat
    long long nrows;
    int L, nlat, nlath, nj8, ntp1, nrsp;
    float plavor;
    int dset = 0;           // 0: gridpointa set (invlega), 1: gridpointd set (invlegd)
};

// One launch covers up to TC_MAXSEG segments (a resolution, a level count and
// a run of instances each); a job names its segment.  nprod = 6 keeps every
// split product of order <= 2 (3-term split); nprod = 3 keeps a0b0, a0b1, a1b0.
struct TcInvLaunch {
    TcInvArgs seg[TC_MAXSEG];
    const int4 *jobs;       // (m, group | seg << 2, first column, columns)
    int nprod;
    // 0: one CTA of 512 threads per SM, a table's two parity halves staged
    // together, 512 TMEM columns.  1: two CTAs of 256 threads per SM, one
    // parity half of a table in shared memory at a time and 256 TMEM columns,
    // so one CTA's copies, staging and epilogue overlap the other's MMAs.
    int half = 0;
};

// spectral row (complex, filter not applied) feeding column pair gq, and
// whether it is the vorticity of a dv2uv pair (planetary vorticity removed).
// Group 0 takes every field of an instance in the gridpointa set (sd, st, sz,
// sq, sp) and, in the gridpointd set, st, sq and sp only (invlegd,
// legmod.f90:661-677): column pair j of an instance reads st (j < L), sq
// (j < 2L) or sp (j = 2L), fields L + j for j < L and 2L + j after.
__device__ __forceinline__ const float2 *inv_row(const TcInvArgs &A, int group, int gq, bool *zvort) {
    const int L = A.L, nf = 4 * L + 1;
    int inst, f;
    *zvort = false;
    if (group == 0 && A.dset) {
        const int nf0 = 2 * L + 1;
        inst = gq / nf0;
        const int j = gq - inst * nf0;
        f = j < L ? L + j : 2 * L + j;
    } else if (group == 0) { inst = gq / nf; f = gq % nf; }
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

// 16 warps (8 in the half-table mode): all stage operands; thread 0 issues
// the table copies and MMAs; in the epilogue warp w drains TMEM lane quarter
// w % 4 for column chunks w / 4, w / 4 + nwarps / 4, ...
constexpr int TCI = 512;
constexpr int TCI_HALF = 256;

// Per-job geometry of the inverse kernel: job (m, group, first column,
// columns); the table buffer at `tab`, the staged data tiles right after it.
struct InvJob {
    int m, group, c0, nc, K, ncp, ntab, nj8, t0;
    int Kq[2], Kp[2];
    size_t ttile[2], tbytes, dtile[2];
    unsigned char *tab, *dat;
};
__device__ __forceinline__ InvJob inv_job(const TcInvArgs &A, int4 jb, unsigned char *tab, bool half) {
    InvJob J;
    J.m = jb.x;
    J.group = jb.y & 3;
    J.c0 = jb.z;
    J.nc = jb.w;
    J.K = A.ntp1 - J.m;
    J.Kq[0] = kpar(J.K, 0);
    J.Kq[1] = kpar(J.K, 1);
    J.Kp[0] = pad16(J.Kq[0]);
    J.Kp[1] = pad16(J.Kq[1]);
    J.ncp = pad16(J.nc);
    J.ntab = J.group == 2 ? 2 : 1;
    J.nj8 = A.nj8;
    J.ttile[0] = (size_t)J.nj8 * J.Kp[0] * 2;
    J.ttile[1] = (size_t)J.nj8 * J.Kp[1] * 2;
    // the table buffer: both parity halves, or (half mode) the larger one
    J.tbytes = half ? 3 * J.ttile[0] : 3 * (J.ttile[0] + J.ttile[1]);
    // data tiles use the padded operand layout (core matrices 144 bytes apart along K)
    J.dtile[0] = (size_t)(J.ncp / 8) * (J.Kp[0] / 8) * tc::kPadLbo;
    J.dtile[1] = (size_t)(J.ncp / 8) * (J.Kp[1] / 8) * tc::kPadLbo;
    J.t0 = J.group == 0 ? 0 : (J.group == 1 ? 1 : 2);
    J.tab = tab;
    J.dat = tab + J.tbytes;
    return J;
}
// bytes from the table buffer's start to the end of the job's data tiles and
// the padding the MMAs read past them (table rows nj8..127 of the M=128 tile)
__device__ __forceinline__ size_t inv_job_bytes(const InvJob &J) {
    return J.tbytes + 3 * (J.dtile[0] + J.dtile[1]) + (size_t)(128 - J.nj8) * 64 * 2 + 128;
}

// thread 0: the job's first table copy (half mode: parity 0 of the first table)
__device__ __forceinline__ void inv_first_copy(const TcInvArgs &A, const InvJob &J, uint64_t *bar_tma) {
    tc::mbar_arrive_expect_tx(bar_tma, (uint32_t)J.tbytes);
    tc::bulk_g2s(J.tab, A.tab + A.off[J.m * 4 + J.t0], (uint32_t)J.tbytes, bar_tma);
}

// all threads: stage the job's spectral columns (both parities) as split BF16 operands
__device__ __forceinline__ void inv_stage(const TcInvArgs &A, const InvJob &J, int tid, int nthr) {
    const int m = J.m, group = J.group, c0 = J.c0, nc = J.nc, ncp = J.ncp;
    const int Kq[2] = {J.Kq[0], J.Kq[1]}, Kp[2] = {J.Kp[0], J.Kp[1]};
    const size_t dtile[2] = {J.dtile[0], J.dtile[1]};
    unsigned char *dat = J.dat;
    // stage the spectral columns of both parities.  A slot is one column pair
    // q (re, im) and the modes k = 2l, 2l+1 of both parities, i.e. the four
    // consecutive spectral entries n - m = 4l .. 4l+3: consecutive threads
    // read consecutive 32-byte pieces of a row, and each stores 4-byte words
    // (two K-elements) into the padded operand layout, where a warp's stores
    // for one pair fall in 32 distinct banks.  The filter is in the tables.
    // Each thread has the loads of INV_SLOTS slots in flight before it splits
    // and stores them.
    {
        constexpr int INV_SLOTS = 4;
        const int npair = ncp >> 1, hk = Kp[0] >> 1;   // Kp[0] >= Kp[1]
        const int nslot = npair * hk;
        const int w0 = A.woff[m];
        for (int s0 = tid; s0 < nslot; s0 += INV_SLOTS * nthr) {
            float2 x[INV_SLOTS][2][2];   // [slot][parity][k - 2l]
#pragma unroll
            for (int i = 0; i < INV_SLOTS; i++) {
                const int s = s0 + i * nthr, q = s / hk, l = s - q * hk;
                bool zv = false;
                const float2 *row = (s < nslot && 2 * q < nc) ? inv_row(A, group, (c0 + 2 * q) >> 1, &zv) : nullptr;
#pragma unroll
                for (int p = 0; p < 2; p++)
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const int k = 2 * l + e, nm = 2 * k + p;  // nm = n - m
                        const bool in = row != nullptr && k < Kq[p];
                        x[i][p][e] = in ? __ldg(row + w0 + nm) : make_float2(0.f, 0.f);
                        if (in && zv && m == 0 && nm == 1) x[i][p][e].x -= A.plavor;  // dv2uv, legmod.f90:332
                    }
            }
#pragma unroll
            for (int i = 0; i < INV_SLOTS; i++) {
                const int s = s0 + i * nthr, q = s / hk, l = s - q * hk;
                if (s >= nslot) break;
#pragma unroll
                for (int p = 0; p < 2; p++) {
                    if (2 * l >= Kp[p]) continue;   // past this parity's (padded) modes
                    uint32_t hr, mr, lr, hi, mi, li;
                    tc::split3x2(x[i][p][0].x, x[i][p][1].x, hr, mr, lr);
                    tc::split3x2(x[i][p][0].y, x[i][p][1].y, hi, mi, li);
                    unsigned char *d0 = dat + (p ? 3 * dtile[0] : 0);
                    const size_t dtp = dtile[p];
                    const uint32_t o = tc::kpad_off(2 * q, 2 * l, Kp[p] >> 3);  // re row; the im row follows at +16
                    st_shared4(d0 + o, hr); st_shared4(d0 + dtp + o, mr); st_shared4(d0 + 2 * dtp + o, lr);
                    st_shared4(d0 + o + 16, hi); st_shared4(d0 + dtp + o + 16, mi); st_shared4(d0 + 2 * dtp + o + 16, li);
                }
            }
        }
    }
}

// thread 0, full mode: the job's MMAs, table by table (the first table's copy
// is already issued); ntma / nmma count the completed phases of bar_tma /
// bar_mma, ncopy the copies issued on bar_tma; the last table's commit
// arrives on bar_done
__device__ __forceinline__ bool inv_mma_full(const TcInvArgs &A, const InvJob &J, uint32_t tmem, int nprod,
                                             uint64_t *bar_tma, uint64_t *bar_mma, uint64_t *bar_done,
                                             uint32_t &ntma, uint32_t &nmma, uint32_t &ncopy) {
    const int m = J.m, ncp = J.ncp, ntab = J.ntab;
    const int Kq[2] = {J.Kq[0], J.Kq[1]}, Kp[2] = {J.Kp[0], J.Kp[1]};
    const size_t ttile[2] = {J.ttile[0], J.ttile[1]}, dtile[2] = {J.dtile[0], J.dtile[1]}, tbytes = J.tbytes;
    unsigned char *tab = J.tab, *dat = J.dat;
    bool ok = true;
    const uint32_t idesc = tc::idesc_bf16(128, ncp);
    for (int ti = 0; ti < ntab && ok; ti++) {
        if (ti > 0) {
            ok = tc::mbar_wait(bar_mma, nmma & 1);  // table buffer free again
            nmma++;
            if (!ok) break;
            const int t = 2 + ti;
            tc::mbar_arrive_expect_tx(bar_tma, (uint32_t)tbytes);
            tc::bulk_g2s(tab, A.tab + A.off[m * 4 + t], (uint32_t)tbytes, bar_tma);
            ncopy++;
        }
        ok = tc::mbar_wait(bar_tma, ntma & 1);
        if (!ok) break;   // the copy is still counted as outstanding (ntma < ncopy)
        ntma++;
        tc::fence_after_sync();
        size_t to = 0, dd = 0;
        for (int p = 0; p < 2; p++) {
            if (!Kq[p]) break;
            // hi*hi products and the five smaller correction products go to
            // separate accumulators (the tensor-core adder truncates; keeping the
            // large term's chain short bounds that error), summed in the epilogue
            const uint32_t dm = tmem + (uint32_t)(((ti * 2 + p) * 2 + 0) * ncp);
            const uint32_t dc = tmem + (uint32_t)(((ti * 2 + p) * 2 + 1) * ncp);
            const uint32_t sbo = (uint32_t)(Kp[p] / 8) * 128, sbo_b = (uint32_t)(Kp[p] / 8) * tc::kPadLbo;
            const uint64_t da0 = tc::smem_desc(tab + to, 128, sbo);
            const uint64_t db0 = tc::smem_desc(dat + dd, tc::kPadLbo, sbo_b);
            const uint32_t tt = (uint32_t)ttile[p], dt = (uint32_t)dtile[p];
            for (int kc = 0; kc < Kp[p] / 16; kc++) {
#pragma unroll
                for (int pr = 0; pr < 6; pr++)
                    if (pr < nprod)
                        tc::mma_bf16(pr == 0 ? dm : dc, tc::desc_add(da0, tc::pair_a(pr) * tt + kc * 256),
                                     tc::desc_add(db0, tc::pair_b(pr) * dt + kc * 2 * tc::kPadLbo), idesc,
                                     kc > 0 || pr > 1);
            }
            to += 3 * ttile[p];
            dd += 3 * dtile[p];
        }
        // intermediate batches recycle the table buffer; the last one releases the epilogue
        tc::mma_commit(ti == ntab - 1 ? bar_done : bar_mma);
    }
    if (!ok) atomicExch(&g_tc_error, 1);
    return ok;
}

// thread 0, half mode: one parity half of one table at a time through one
// buffer: copy, MMAs, and the next copy once those MMAs have read the buffer
__device__ __forceinline__ bool inv_mma_half(const TcInvArgs &A, const InvJob &J, uint32_t tmem, int nprod,
                                             uint64_t *bar_tma, uint64_t *bar_mma, uint64_t *bar_done) {
    const int m = J.m, ncp = J.ncp, ntab = J.ntab, t0 = J.t0;
    const int Kq[2] = {J.Kq[0], J.Kq[1]}, Kp[2] = {J.Kp[0], J.Kp[1]};
    const size_t ttile[2] = {J.ttile[0], J.ttile[1]}, dtile[2] = {J.dtile[0], J.dtile[1]};
    unsigned char *tab = J.tab, *dat = J.dat;
    bool ok = true;
    // one parity half of one table at a time through one buffer: copy,
    // MMAs, and the next copy once those MMAs have read the buffer
    const uint32_t idesc = tc::idesc_bf16(128, ncp);
    const int np = Kq[1] ? 2 : 1, nh = ntab * np;
    for (int hix = 0; hix < nh && ok; hix++) {
        const int ti = hix / np, p = hix - ti * np;
        if (hix > 0) {
            ok = tc::mbar_wait(bar_mma, (hix - 1) & 1);
            if (!ok) break;
            const uint32_t hb = (uint32_t)(3 * ttile[p]);
            tc::mbar_arrive_expect_tx(bar_tma, hb);
            tc::bulk_g2s(tab, A.tab + A.off[m * 4 + t0 + ti] + (p ? 3 * ttile[0] : 0), hb, bar_tma);
        }
        ok = tc::mbar_wait(bar_tma, hix & 1);
        if (!ok) break;
        tc::fence_after_sync();
        const uint32_t dm = tmem + (uint32_t)(((ti * 2 + p) * 2 + 0) * ncp);
        const uint32_t dc = tmem + (uint32_t)(((ti * 2 + p) * 2 + 1) * ncp);
        const uint32_t sbo = (uint32_t)(Kp[p] / 8) * 128, sbo_b = (uint32_t)(Kp[p] / 8) * tc::kPadLbo;
        const uint64_t da0 = tc::smem_desc(tab, 128, sbo);
        const uint64_t db0 = tc::smem_desc(dat + (p ? 3 * dtile[0] : 0), tc::kPadLbo, sbo_b);
        const uint32_t tt = (uint32_t)ttile[p], dt = (uint32_t)dtile[p];
        for (int kc = 0; kc < Kp[p] / 16; kc++) {
#pragma unroll
            for (int pr = 0; pr < 6; pr++)
                if (pr < nprod)
                    tc::mma_bf16(pr == 0 ? dm : dc, tc::desc_add(da0, tc::pair_a(pr) * tt + kc * 256),
                                 tc::desc_add(db0, tc::pair_b(pr) * dt + kc * 2 * tc::kPadLbo), idesc,
                                 kc > 0 || pr > 1);
        }
        tc::mma_commit(hix == nh - 1 ? bar_done : bar_mma);
    }
    if (!ok) atomicExch(&g_tc_error, 1);
    return ok;
}

// all threads (a warp-uniform test, as the TMEM loads need whole warps): TMEM
// lane = latitude pair j, quarters past the last pair hold nothing; drain
// the accumulators and write the job's m-major Fourier rows
__device__ __forceinline__ void inv_epilogue(const TcInvArgs &A, const InvJob &J, uint32_t tmem, int warp, int lane,
                                             int nsub) {
    const int quarter = warp & 3, sub = warp >> 2;
    if (quarter * 32 >= A.nlath) return;
    const int m = J.m, group = J.group, c0 = J.c0, nc = J.nc, ncp = J.ncp;
    const int Kq[2] = {J.Kq[0], J.Kq[1]};
    const int j = quarter * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    // gridpointa writes gu gv gt gd gz gq gpj gpmt gp (6L+3 fields),
    // gridpointd gu gv gt gq gp (4L+1)
    const int L = A.L, nfo = A.dset ? 4 * L + 1 : 6 * L + 3, nf = A.dset ? 2 * L + 1 : 4 * L + 1;
    const bool has1 = Kq[1] > 0;
    const bool row_ok = j < A.nlath;
    const int latN = j, latS = A.nlat - 1 - j;
    float2 *Wm = A.W + (size_t)m * A.nrows;
    if (group < 2) {
        // P-type qi: N = D0 + D1, S = D0 - D1; Q-type qj: S = D1 - D0
        const float ss = group == 0 ? 1.f : -1.f;
        for (int cc = sub * 16; cc < ncp; cc += 16 * nsub) {
            // parity 0's main and correction accumulators, summed, then parity 1's
            // (two loads in flight at a time: fewer live registers)
            float d0[16], d1[16];
            {
                uint32_t ra[16], rb[16];
                tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(0 * ncp + cc), ra);
                tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(1 * ncp + cc), rb);
                tc::tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; i++) d0[i] = __uint_as_float(ra[i]) + __uint_as_float(rb[i]);
                if (has1) {
                    tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(2 * ncp + cc), ra);
                    tc::tmem_ld16_nw(tmem + lane_addr + (uint32_t)(3 * ncp + cc), rb);
                    tc::tmem_wait_ld();
                }
#pragma unroll
                for (int i = 0; i < 16; i++) d1[i] = has1 ? __uint_as_float(ra[i]) + __uint_as_float(rb[i]) : 0.f;
            }
            // column pair gq = (c0 + cc)/2 + i/2: instance and field without a
            // division per pair (a chunk holds 8 pairs, fewer than nf)
            const int gq0 = (c0 + cc) >> 1;
            const int inst0 = group == 0 ? gq0 / nf : gq0, f0 = group == 0 ? gq0 - inst0 * nf : 4 * L;
#pragma unroll
            for (int i = 0; i < 16; i += 2) {
                const float d0r = d0[i], d0i = d0[i + 1], d1r = d1[i], d1i = d1[i + 1];
                if (!row_ok || cc + i >= nc) continue;
                int inst = inst0, f = f0;
                if (group == 0) {
                    f += i >> 1;
                    while (f >= nf) { f -= nf; inst++; }
                } else {
                    inst += i >> 1;
                }
                const float2 vn = make_float2(d0r + d1r, d0i + d1i);
                const float2 vs = make_float2(ss * (d0r - d1r), ss * (d0i - d1i));
                int F;
                if (A.dset) F = 2 * L + f;                    // st -> gt, sq -> gq, sp -> gp
                else if (group == 1) F = 6 * L;               // gpj
                else if (f < L) F = 3 * L + f;                // sd -> gd
                else if (f < 2 * L) F = f + L;                // st -> gt
                else if (f < 4 * L) F = f + 2 * L;            // sz -> gz, sq -> gq
                else F = 6 * L + 2;                           // sp -> gp
                float2 *wr = Wm + (size_t)(inst * nfo + F) * A.nlat;
                wr[latN] = vn;
                wr[latS] = vs;
                if (group == 0 && !A.dset && f == 4 * L) {    // gpmt = i*m*gp
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
        for (int cc = sub * 8; cc < ncp; cc += 8 * nsub) {
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

// One job per CTA (half mode: two CTAs of 256 threads per SM)
__global__ void __launch_bounds__(TCI) k_tc_inverse(const __grid_constant__ TcInvLaunch P) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int4 jb = P.jobs[blockIdx.x];
    const TcInvArgs &A = P.seg[jb.y >> 2];
    const int nprod = P.nprod;
    const bool half = P.half != 0;
    const int nthr = blockDim.x, nsub = nthr >> 7;   // column-chunk groups of 4 warps
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const InvJob J = inv_job(A, jb, sm, half);
    unsigned char *tail = sm + inv_job_bytes(J);
    uint64_t *bar_tma = reinterpret_cast<uint64_t *>((reinterpret_cast<uintptr_t>(tail) + 15) & ~(uintptr_t)15);
    uint64_t *bar_mma = bar_tma + 1;
    uint64_t *bar_done = bar_tma + 2;
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar_tma + 3);
    const uint32_t tcols = half ? 256 : 512;
    pdl_trigger();
    if (warp == 0) tc::tmem_alloc(slot, tcols);
    if (tid == 0) {
        tc::mbar_init(bar_tma, 1);
        tc::mbar_init(bar_mma, 1);
        tc::mbar_init(bar_done, 1);
        tc::mbar_fence_init();
        // the first table copy goes out before the staging so the two overlap
        inv_first_copy(A, J, bar_tma);
    }
    pdl_wait();   // the spectral input and the intermediate are shared with earlier kernels
    inv_stage(A, J, tid, nthr);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    bool ok = true;
    uint32_t ntma = 0, nmma = 0, ncopy = 1;   // thread 0's bar_tma accounting (full mode)
    if (tid == 0)
        ok = half ? inv_mma_half(A, J, tmem, nprod, bar_tma, bar_mma, bar_done)
                  : inv_mma_full(A, J, tmem, nprod, bar_tma, bar_mma, bar_done, ntma, nmma, ncopy);
    __syncthreads();
    ok = __all_sync(0xffffffffu, tc::mbar_wait(bar_done, 0));  // warp-uniform for the .sync.aligned TMEM loads
    if (!ok && lane == 0) atomicExch(&g_tc_error, 2);
    tc::fence_after_sync();
    if (ok) inv_epilogue(A, J, tmem, warp, lane, nsub);
    // after a timeout, copies issued but never waited for land before the block exits
    if (tid == 0 && !ok && !half)
        while (ntma < ncopy) tc::mbar_wait(bar_tma, ntma++ & 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, tcols);
}

// Persistent form (full mode): one CTA of 512 threads per SM walks the jobs
// blockIdx.x, + gridDim.x, ...  The barriers sit at the start of shared memory
// and the table buffer after them.  Once a job's MMAs have completed, thread 0
// issues the next job's first table copy, which lands while this job's
// epilogue drains TMEM; the next job's staging follows the epilogue.
constexpr int TCI_BARS = 128;   // bytes in front of the table buffer
__global__ void __launch_bounds__(TCI) k_tc_inverse_p(const __grid_constant__ TcInvLaunch P, int njobs) {
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t *bar_tma = reinterpret_cast<uint64_t *>(sm);
    uint64_t *bar_mma = bar_tma + 1;
    uint64_t *bar_done = bar_tma + 2;
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar_tma + 3);
    unsigned char *tabbuf = sm + TCI_BARS;
    const int nprod = P.nprod;
    const int nthr = blockDim.x, nsub = nthr >> 7;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    pdl_trigger();
    if (warp == 0) tc::tmem_alloc(slot, 512);
    int j = blockIdx.x;
    uint32_t ncopy = 0;   // table copies issued on bar_tma (thread 0)
    if (tid == 0) {
        tc::mbar_init(bar_tma, 1);
        tc::mbar_init(bar_mma, 1);
        tc::mbar_init(bar_done, 1);
        tc::mbar_fence_init();
        if (j < njobs) {   // job descriptors and tables are host-built: before the dependent-launch wait
            const int4 jb = P.jobs[j];
            inv_first_copy(P.seg[jb.y >> 2], inv_job(P.seg[jb.y >> 2], jb, tabbuf, false), bar_tma);
            ncopy++;
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    pdl_wait();   // the spectral input and the intermediate are shared with earlier kernels
    uint32_t ntma = 0, nmma = 0, ndone = 0;
    bool ok = true;
    for (; j < njobs; j += gridDim.x) {
        const int4 jb = P.jobs[j];
        const TcInvArgs &A = P.seg[jb.y >> 2];
        const InvJob J = inv_job(A, jb, tabbuf, false);
        inv_stage(A, J, tid, nthr);
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();   // staged; the previous job's TMEM loads have completed
        tc::fence_after_sync();
        if (tid == 0) inv_mma_full(A, J, tmem, nprod, bar_tma, bar_mma, bar_done, ntma, nmma, ncopy);
        ok = __all_sync(0xffffffffu, tc::mbar_wait(bar_done, ndone & 1));   // warp-uniform
        ndone++;
        ok = __syncthreads_and(ok) != 0;   // block-uniform, so every thread leaves the loop together
        if (!ok) {
            if (tid == 0) atomicExch(&g_tc_error, 2);
            break;
        }
        tc::fence_after_sync();
        // the MMAs have read the table buffer and the data tiles: the next job's
        // first table lands while this job's epilogue runs
        if (tid == 0 && j + (int)gridDim.x < njobs) {
            const int4 jn = P.jobs[j + gridDim.x];
            inv_first_copy(P.seg[jn.y >> 2], inv_job(P.seg[jn.y >> 2], jn, tabbuf, false), bar_tma);
            ncopy++;
        }
        inv_epilogue(A, inv_job(A, jb, tabbuf, false), tmem, warp, lane, nsub);   // recomputed: fewer live registers
        tc::fence_before_sync();
    }
    // after a timeout, copies issued but never waited for land before the block exits
    if (tid == 0 && !ok)
        while (ntma < ncopy) tc::mbar_wait(bar_tma, ntma++ & 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 512);
}

static size_t inv_smem(int nj8, int K, int ncp) {
    const int Kp0 = pad16(kpar(K, 0)), Kp1 = pad16(kpar(K, 1));
    return 3 * (size_t)nj8 * (Kp0 + Kp1) * 2 + 3 * (size_t)(ncp / 8) * ((Kp0 + Kp1) / 8) * tc::kPadLbo +
           (size_t)(128 - nj8) * 64 * 2 + 128 + 80;
}
// the same in the half-table mode: one parity half (the larger) of a table
static size_t inv_smem_half(int nj8, int K, int ncp) {
    const int Kp0 = pad16(kpar(K, 0)), Kp1 = pad16(kpar(K, 1));
    return 3 * (size_t)nj8 * Kp0 * 2 + 3 * (size_t)(ncp / 8) * ((Kp0 + Kp1) / 8) * tc::kPadLbo +
           (size_t)(128 - nj8) * 64 * 2 + 128 + 80;
}

// ------------------------------------------------------------ forward
struct TcFwdArgs {
    const unsigned char *tab;
    const long long *off;
    const int *woff;
    const float2 *W;        // [m][row], row = (inst*(9L+1) + field)*nlat + lat
    long long nrows;
    const float *filt;      // skgpsp
    float *spout;           // [inst][4L+1][NRSP] (gridpointd: [inst][4L][NRSP])
    int L, nlat, nlath, njc, ntp1, nrsp;
    int dset = 0;           // 0: gridpointa forward set, 1: gridpointd
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

// Fourier row of field kind `kind`, level l of an instance, or -1 for a kind
// the set does not have.  gridpointa (9L+1 fields) has every kind; gridpointd
// (4L fields gtdt, gudt, gvdt, gqdt, plasim.f90:3415-3428) feeds fc2sp of
// gtdt and gqdt through the tn and qn columns and uv2dv(gudt, gvdt) through
// the fu and fv columns: mktend's d and z with ke = 0 are uv2dv's
// (legmod.f90:356-426, :555-602), its t with vt = ut = 0 and qtend's q with
// vq = uq = 0 are fc2sp's.
__device__ __forceinline__ long long fwd_row(int L, int inst, int kind, int l, int dset = 0) {
    if (dset) {
        int F;
        if (kind == 0) F = l;               // tn <- gtdt
        else if (kind == 5) F = L + l;      // fu <- gudt
        else if (kind == 4) F = 2 * L + l;  // fv <- gvdt
        else if (kind == 1) F = 3 * L + l;  // qn <- gqdt
        else return -1;
        return (long long)inst * (4 * L) + F;
    }
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
    const bool with_vpp = (l0 == 0) && !A.dset;
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
                    if (li < nl) rb = fwd_row(L, inst, c_fwd_fields[t][fi], l0 + li, A.dset);
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
            const int nfo = A.dset ? 4 * L : 4 * L + 1;
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
    int dset = 0;           // 0: gridpointa forward set, 1: gridpointd (no gvpp; 4L outputs)
};
struct TcFwd3Launch {
    TcFwd3Args seg[TC_MAXSEG];
    const int4 *jobs;       // (m, inst | seg << 16, first level, levels | parity << 8)
    int nprod;              // 6: all six products; 3: a0b0, a0b1, a1b0 (and a1b1)
    int njobs;              // jobs in the list (the persistent kernel walks them)
    int njmax;              // largest njc over the segments (sizes the persistent kernel's rings)
};
constexpr int F3_NLT = 5;   // levels per job; the widest table then has 48 columns (3 x 48 TMEM columns)

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

// Fourier row of column pair q of table t in a job, or -1 for a padding pair
template <int NLT>
__device__ __forceinline__ long long f3_row(const TcFwd3Args &A, int inst, int l0, int nl, bool with_vpp, int t,
                                            int q) {
    const int nf = c_fwd_nf[t];
    if (q >= nf * NLT + ((t == 0) ? 1 : 0)) return -1;
    if (t == 0 && q == nf * NLT) return (with_vpp && !A.dset) ? fwd_row(A.L, inst, 7, 0) : -1;
    const int fi = q / NLT, li = q - fi * NLT;
    return li < nl ? fwd_row(A.L, inst, c_fwd_fields[t][fi], l0 + li, A.dset) : -1;
}

// Operand staging works on slots: a slot is one column pair q (a field level,
// re and im) and the four latitude pairs j = 4jq .. 4jq+3.  Consecutive threads
// take consecutive jq of a pair, so a warp's loads read 1 KB of a Fourier row's
// northern half and of its mirrored southern half, and its 8-byte stores fall
// in distinct banks of the padded operand layout (one half-warp per wavefront).
struct F3Slot {
    float2 n[4], s[4];  // north and south values at latitude pairs j .. j+3
};

template <int NLT>
__device__ __forceinline__ void f3_load(const TcFwd3Args &A, int m, int inst, int l0, int nl, bool with_vpp, int t,
                                        int sl, F3Slot &v) {
    const int hj = A.njc >> 2;
    const int q = sl / hj, jq = sl - q * hj;
#pragma unroll
    for (int e = 0; e < 4; e++) v.n[e] = v.s[e] = make_float2(0.f, 0.f);
    if (q >= (fwd_ncp<NLT>(t) >> 1)) return;
    const long long rb = f3_row<NLT>(A, inst, l0, nl, with_vpp, t, q);
    if (rb < 0) return;
    const int j = 4 * jq, nlat = A.nlat, nlath = A.nlath;
    const float2 *wr = A.W + (size_t)m * A.nrows + (size_t)rb * nlat;
    if (j + 4 <= nlath) {
        // north rows j .. j+3; south rows nlat-4-j .. nlat-1-j (pairs j+3 .. j)
        const float4 x0 = __ldg(reinterpret_cast<const float4 *>(wr + j));
        const float4 x1 = __ldg(reinterpret_cast<const float4 *>(wr + j + 2));
        const float4 y0 = __ldg(reinterpret_cast<const float4 *>(wr + nlat - 4 - j));
        const float4 y1 = __ldg(reinterpret_cast<const float4 *>(wr + nlat - 2 - j));
        v.n[0] = make_float2(x0.x, x0.y); v.n[1] = make_float2(x0.z, x0.w);
        v.n[2] = make_float2(x1.x, x1.y); v.n[3] = make_float2(x1.z, x1.w);
        v.s[3] = make_float2(y0.x, y0.y); v.s[2] = make_float2(y0.z, y0.w);
        v.s[1] = make_float2(y1.x, y1.y); v.s[0] = make_float2(y1.z, y1.w);
    } else {
#pragma unroll
        for (int e = 0; e < 4; e++)
            if (j + e < nlath) {
                v.n[e] = __ldg(wr + j + e);
                v.s[e] = __ldg(wr + nlat - 1 - j - e);
            }
    }
}

// fold a slot for parity p, split it into three BF16 terms and store the re
// and im words of every term
template <int NLT>
__device__ __forceinline__ void f3_store(int t, int p, int sl, int njc, unsigned char *bt, const F3Slot &v) {
    const int hj = njc >> 2, ngk = njc >> 3;
    const int q = sl / hj, jq = sl - q * hj;
    const int ncp = fwd_ncp<NLT>(t);
    if (q >= (ncp >> 1)) return;
    const bool diff = (t != 1) ? (p == 1) : (p == 0);
    float xr[4], xi[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        xr[e] = diff ? v.n[e].x - v.s[e].x : v.n[e].x + v.s[e].x;
        xi[e] = diff ? v.n[e].y - v.s[e].y : v.n[e].y + v.s[e].y;
    }
    uint2 hr, mr, lr, hi, mi, li;
    tc::split3x2(xr[0], xr[1], hr.x, mr.x, lr.x);
    tc::split3x2(xr[2], xr[3], hr.y, mr.y, lr.y);
    tc::split3x2(xi[0], xi[1], hi.x, mi.x, li.x);
    tc::split3x2(xi[2], xi[3], hi.y, mi.y, li.y);
    const uint32_t dt = (uint32_t)(ncp >> 3) * ngk * tc::kPadLbo;  // one split term
    const uint32_t o = tc::kpad_off(2 * q, 4 * jq, ngk);            // re row; the im row follows at +16
    st_shared8(bt + o, hr); st_shared8(bt + dt + o, mr); st_shared8(bt + 2 * dt + o, lr);
    st_shared8(bt + o + 16, hi); st_shared8(bt + dt + o + 16, mi); st_shared8(bt + 2 * dt + o + 16, li);
}

// The same staging from the equator-folded intermediate (rfft_fwd_fold_body):
// each field row holds E = N + S for the latitude pairs, then O = N - S, so a
// parity reads only the half it needs and a slot covers eight latitude pairs
// j = 8jg .. 8jg+7 of one row (n[] the first four, s[] the next four), stored
// as one 16-byte core-matrix row per split term.
template <int NLT>
__device__ __forceinline__ void f3_load_fold(const TcFwd3Args &A, int m, int inst, int l0, int nl, bool with_vpp,
                                             int t, int p, int sl, F3Slot &v) {
    const int hj = A.njc >> 3;
    const int q = sl / hj, jg = sl - q * hj;
#pragma unroll
    for (int e = 0; e < 4; e++) v.n[e] = v.s[e] = make_float2(0.f, 0.f);
    if (q >= (fwd_ncp<NLT>(t) >> 1)) return;
    const long long rb = f3_row<NLT>(A, inst, l0, nl, with_vpp, t, q);
    if (rb < 0) return;
    const int j = 8 * jg, nlath = A.nlath;
    const bool diff = (t != 1) ? (p == 1) : (p == 0);
    const float2 *wf = A.W + (size_t)m * A.nrows + (size_t)rb * A.nlat + (diff ? nlath : 0);
    if (j + 8 <= nlath && !(nlath & 1)) {
        const float4 *w4 = reinterpret_cast<const float4 *>(wf + j);
        const float4 x0 = __ldg(w4), x1 = __ldg(w4 + 1), x2 = __ldg(w4 + 2), x3 = __ldg(w4 + 3);
        v.n[0] = make_float2(x0.x, x0.y); v.n[1] = make_float2(x0.z, x0.w);
        v.n[2] = make_float2(x1.x, x1.y); v.n[3] = make_float2(x1.z, x1.w);
        v.s[0] = make_float2(x2.x, x2.y); v.s[1] = make_float2(x2.z, x2.w);
        v.s[2] = make_float2(x3.x, x3.y); v.s[3] = make_float2(x3.z, x3.w);
    } else {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            if (j + e < nlath) v.n[e] = __ldg(wf + j + e);
            if (j + 4 + e < nlath) v.s[e] = __ldg(wf + j + 4 + e);
        }
    }
}
template <int NLT>
__device__ __forceinline__ void f3_store_fold(int t, int sl, int njc, unsigned char *bt, const F3Slot &v) {
    const int hj = njc >> 3, ngk = njc >> 3;
    const int q = sl / hj, jg = sl - q * hj;
    const int ncp = fwd_ncp<NLT>(t);
    if (q >= (ncp >> 1)) return;
    float xr[8], xi[8];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        xr[e] = v.n[e].x; xi[e] = v.n[e].y;
        xr[e + 4] = v.s[e].x; xi[e + 4] = v.s[e].y;
    }
    uint4 h, mm, l;
    const uint32_t dt = (uint32_t)(ncp >> 3) * ngk * tc::kPadLbo;  // one split term
    const uint32_t o = tc::kpad_off(2 * q, 8 * jg, ngk);            // re row; the im row follows at +16
    tc::split3x8(xr, h, mm, l);
    st_shared16(bt + o, h); st_shared16(bt + dt + o, mm); st_shared16(bt + 2 * dt + o, l);
    tc::split3x8(xi, h, mm, l);
    st_shared16(bt + o + 16, h); st_shared16(bt + dt + o + 16, mm); st_shared16(bt + 2 * dt + o + 16, l);
}

// ------------------------------------------------------------ forward, pipelined
// Persistent form of the stacked-split forward kernel.  One CTA per SM walks
// the jobs blockIdx.x, blockIdx.x + gridDim.x, ... of the launch; a job's four
// tables are four tiles, and tiles flow through rings so that different
// warps work on different tiles at once:
//   warp 1 (one lane)       copies table blocks into a 2-slot ring
//   warps 2-3, 8-15         stage the folded, split operands into a 2-slot ring
//   warp 0 (one lane)       issues the MMAs of a tile into one of 3 TMEM slots
//   warps 4-7               drain TMEM (lane quarter = warp - 4), accumulate a
//                           job's outputs over its tiles and store them
// Each ring slot has a full and an empty mbarrier; every wait is bounded, and
// a wait that times out raises an abort flag that ends every role's loop.
constexpr int FP_THREADS = 512;
constexpr int FP_NST = 320;              // staging threads
constexpr int FP_ACC = 144;              // TMEM columns of a slot: 3 x the widest table's columns
constexpr int FP_SLOTS = 2;              // staging slots per thread kept in flight for one tile
constexpr int FP_FOLD_DEPTH = 2;         // tiles ahead whose folded-intermediate loads are in flight

struct FpLayout {
    uint32_t tb, ob;                     // bytes of a table slot and of an operand slot
    uint32_t op, e, bars;                // offsets of the operand ring, the exchange area, the barriers
};
__host__ __device__ inline FpLayout fp_layout(int njmax) {
    FpLayout L;
    L.tb = 8u * 64u * (uint32_t)njmax;
    L.ob = 3u * (48u / 8u) * (uint32_t)(njmax / 8) * tc::kPadLbo;
    L.op = 2 * L.tb + 128 * 32 * 2;       // rows >= 2R of a table tile read up to 8 KB past it
    L.e = L.op + 2 * L.ob;
    L.bars = L.e + 128 * (F3_NLT * 8 + 2) * 4;
    L.bars = (L.bars + 15) & ~15u;
    return L;
}
constexpr int FP_JOBS = 512;             // jobs of a CTA kept in shared memory (later ones are read from global)
static size_t fpipe_smem(int njmax) { return fp_layout(njmax).bars + 32 * 8 + FP_JOBS * 16; }

// bounded wait that also gives up as soon as another role has aborted
__device__ __forceinline__ bool fp_wait(uint64_t *bar, uint32_t parity, volatile int *abort) {
    const uint32_t addr = tc::smem_u32(bar);
    for (uint32_t i = 0; i < tc::kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255) == 255 && *abort) return false;
    }
    *abort = 1;
    return false;
}

// barrier of the 128 epilogue threads on an mbarrier (count 128), bounded like every wait
__device__ __forceinline__ bool fp_epi_sync(uint64_t *bar, uint32_t &phase, volatile int *abort) {
    tc::mbar_arrive(bar);
    const bool ok = fp_wait(bar, phase, abort);
    phase ^= 1;
    return ok;
}

// one TMEM slot holds table T's split blocks at columns 0, ncp, 2 ncp; drained
// 8 columns at a time (fewer live registers than the 16-wide loads)
template <int NLT, int T>
__device__ __forceinline__ void fp_drain_t(uint32_t X, int nprod, float (*o)[4][2], float *ov) {
    constexpr int ncp = fwd_ncp<NLT>(T);
#pragma unroll
    for (int c0 = 0; c0 < ncp; c0 += 8) {
        uint32_t x0[8], x1[8], x2[8];
        tc::tmem_ld8_nw(X + c0, x0);
        tc::tmem_ld8_nw(X + ncp + c0, x1);
        if (nprod == 6) tc::tmem_ld8_nw(X + 2 * ncp + c0, x2);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; i++) {
            float v = __uint_as_float(x0[i]) + __uint_as_float(x1[i]);
            if (nprod == 6) v += __uint_as_float(x2[i]);
            f3_combine<NLT>(T, c0 + i, v, o, ov);
        }
    }
}
template <int NLT>
__device__ __forceinline__ void fp_drain(int t, uint32_t X, int nprod, float (*o)[4][2], float *ov) {
    if (t == 0) fp_drain_t<NLT, 0>(X, nprod, o, ov);
    else if (t == 1) fp_drain_t<NLT, 1>(X, nprod, o, ov);
    else if (t == 2) fp_drain_t<NLT, 2>(X, nprod, o, ov);
    else fp_drain_t<NLT, 3>(X, nprod, o, ov);
}

// FOLD: the intermediate is folded about the equator (rfft_fwd_fold_body)
template <int NLT, bool FOLD>
__global__ void __launch_bounds__(FP_THREADS, 1) k_tc_forward_pipe(const __grid_constant__ TcFwd3Launch P) {
    extern __shared__ __align__(128) unsigned char sm[];
    const FpLayout LY = fp_layout(P.njmax);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char *tabr = sm, *opr = sm + LY.op;
    float *E = reinterpret_cast<float *>(sm + LY.e);
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + LY.bars);
    uint64_t *tab_full = bars, *tab_empty = bars + 2, *op_full = bars + 4, *op_empty = bars + 6;
    uint64_t *acc_full = bars + 8, *acc_empty = bars + 11, *ep_bar = bars + 14;
    uint32_t *slot = reinterpret_cast<uint32_t *>(bars + 15);
    volatile int *abort = reinterpret_cast<volatile int *>(bars + 16);
    int4 *jobs_s = reinterpret_cast<int4 *>(sm + LY.bars + 32 * 8);
    const int nprod = P.nprod;
    const int njobs = P.njobs;
    // tiles of this CTA: jobs blockIdx.x + k gridDim.x, four tables each
    const int mine = njobs > (int)blockIdx.x ? (njobs - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int ntile = 4 * mine;
    pdl_trigger();
    // this CTA's job descriptors, read once (host-written, so before the dependent-launch wait)
    for (int k = tid; k < mine && k < FP_JOBS; k += FP_THREADS) jobs_s[k] = P.jobs[blockIdx.x + k * gridDim.x];
    auto job = [&](int i) {
        const int k = i >> 2;
        return k < FP_JOBS ? jobs_s[k] : P.jobs[blockIdx.x + k * gridDim.x];
    };
    if (warp == 0) tc::tmem_alloc(slot, 512);
    if (tid == 0) {
        for (int i = 0; i < 2; i++) {
            tc::mbar_init(tab_full + i, 1);
            tc::mbar_init(tab_empty + i, 1);
            tc::mbar_init(op_full + i, FP_NST);
            tc::mbar_init(op_empty + i, 1);
        }
        for (int i = 0; i < 3; i++) {
            tc::mbar_init(acc_full + i, 1);
            tc::mbar_init(acc_empty + i, 4);
        }
        tc::mbar_init(ep_bar, 128);
        *abort = 0;
        tc::mbar_fence_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;

    if (warp == 1) {
        // ---------------------------------------------------------- table copies
        if (lane == 0) {
            int issued[2] = {0, 0};
            for (int i = 0; i < ntile; i++) {
                const int b = i & 1, u = i >> 1;
                if (!fp_wait(tab_empty + b, (u & 1) ^ 1, abort)) break;
                const int4 jb = job(i);
                const TcFwd3Args &A = P.seg[jb.y >> 16];
                const int m = jb.x, p = jb.w >> 8, t = i & 3;
                const uint32_t tbytes = 8u * (uint32_t)pad8(kpar(A.ntp1 - m, p)) * (uint32_t)A.njc;
                tc::mbar_arrive_expect_tx(tab_full + b, tbytes);
                tc::bulk_g2s(tabr + b * LY.tb, A.tab + A.off[(m * 4 + t) * 2 + p], tbytes, tab_full + b);
                issued[b] = u + 1;
            }
            if (*abort) {
                // copies still in flight land before the block exits
                for (int b = 0; b < 2; b++)
                    if (issued[b]) tc::mbar_wait(tab_full + b, (issued[b] - 1) & 1);
            }
        }
    } else if (warp == 0) {
        // ---------------------------------------------------------------- MMAs
        if (lane == 0) {
            for (int i = 0; i < ntile; i++) {
                const int b = i & 1, u = i >> 1, a = i % 3, ua = i / 3;
                if (!fp_wait(tab_full + b, u & 1, abort) || !fp_wait(op_full + b, u & 1, abort) ||
                    !fp_wait(acc_empty + a, (ua & 1) ^ 1, abort))
                    break;
                tc::fence_after_sync();
                const int4 jb = job(i);
                const TcFwd3Args &A = P.seg[jb.y >> 16];
                const int m = jb.x, p = jb.w >> 8, t = i & 3;
                const int R = pad8(kpar(A.ntp1 - m, p)), njc = A.njc;
                const int ncp = fwd_ncp<NLT>(t);
                const uint32_t idesc1 = tc::idesc_bf16(128, (nprod == 6 ? 3 : 2) * ncp);
                const uint32_t idesc2 = tc::idesc_bf16(128, ncp);
                const uint32_t X = tmem + (uint32_t)(a * FP_ACC);
                const uint64_t db = tc::smem_desc(opr + b * LY.ob, tc::kPadLbo, (uint32_t)(njc / 8) * tc::kPadLbo);
                unsigned char *tb = tabr + b * LY.tb;
                uint32_t jo = 0;
                for (int j0 = 0; j0 < njc; j0 += 32) {
                    const int jw = njc - j0 < 32 ? njc - j0 : 32;
                    const uint32_t tt = (uint32_t)2 * R * jw * 2;   // one stacked tile
                    const uint64_t da1 = tc::smem_desc(tb + jo, 128, (uint32_t)(jw / 8) * 128);
                    const uint64_t da2 = tc::desc_add(da1, tt);
                    for (int kc = 0; kc < jw / 16; kc++) {
                        const uint64_t dbk = tc::desc_add(db, (uint32_t)(j0 / 8 + 2 * kc) * tc::kPadLbo);
                        tc::mma_bf16(X, tc::desc_add(da1, kc * 256), dbk, idesc1, j0 > 0 || kc > 0);
                        if (nprod == 6) tc::mma_bf16(X, tc::desc_add(da2, kc * 256), dbk, idesc2, true);
                    }
                    jo += 2 * tt;
                }
                tc::mma_commit(tab_empty + b);
                tc::mma_commit(op_empty + b);
                tc::mma_commit(acc_full + a);
            }
        }
    } else if (warp >= 4 && warp < 8) {
        // ------------------------------------------------------------ epilogue
        const int quarter = warp - 4, r = quarter * 32 + lane;
        pdl_wait();   // the outputs may be read by earlier kernels
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        constexpr int NO = NLT * 8 + 2;
        float o[NLT][4][2], ov[2];
        float fl = 0.f;   // the job's filter factor and output offset, loaded when the job starts
        int wom = 0;
        bool ok = true;
        uint32_t ep_phase = 0;
        for (int i = 0; i < ntile && ok; i++) {
            const int a = i % 3, ua = i / 3, t = i & 3;
            const int4 jb = job(i);
            const TcFwd3Args &A = P.seg[jb.y >> 16];
            const int m = jb.x, inst = jb.y & 0xffff, l0 = jb.z, nl = jb.w & 0xff, p = jb.w >> 8;
            const int Kq = kpar(A.ntp1 - m, p), R = pad8(Kq);
            if (t == 0) {
#pragma unroll
                for (int li = 0; li < NLT; li++)
#pragma unroll
                    for (int k = 0; k < 4; k++) o[li][k][0] = o[li][k][1] = 0.f;
                ov[0] = ov[1] = 0.f;
                if (r < Kq) fl = A.filt[m + 2 * r + p];
                wom = A.woff[m];
            }
            ok = __all_sync(0xffffffffu, fp_wait(acc_full + a, ua & 1, abort));   // warp-uniform
            if (!ok) break;
            tc::fence_after_sync();
            if (quarter * 32 < 2 * R) fp_drain<NLT>(t, tmem + lane_addr + (uint32_t)(a * FP_ACC), nprod, o, ov);
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(acc_empty + a);
            if (t < 3) continue;
            // the job's four tables are in: rows R..2R-1 hand their corrections to rows 0..R-1
            if (r >= R && r < 2 * R) {
                float *e = E + (size_t)(r - R) * NO;
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
            ok = __all_sync(0xffffffffu, fp_epi_sync(ep_bar, ep_phase, abort));
            if (!ok) break;
            if (r < Kq) {
                const float *e = E + (size_t)r * NO;
                const int L = A.L, nfo = A.dset ? 4 * L : 4 * L + 1, k = 2 * r + p;   // k = n - m
                const size_t wo = (size_t)wom + k;
#pragma unroll
                for (int li = 0; li < NLT; li++) {
                    if (li >= nl) break;
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {
                        float2 *dst = reinterpret_cast<float2 *>(A.spout + ((size_t)inst * nfo + kk * L + l0 + li) * A.nrsp);
                        dst[wo] = make_float2((o[li][kk][0] + e[(li * 4 + kk) * 2]) * fl,
                                              (o[li][kk][1] + e[(li * 4 + kk) * 2 + 1]) * fl);
                    }
                }
                if (l0 == 0 && !A.dset) {
                    float2 *dst = reinterpret_cast<float2 *>(A.spout + ((size_t)inst * nfo + 4 * L) * A.nrsp);
                    dst[wo] = make_float2((ov[0] + e[NLT * 8]) * fl, (ov[1] + e[NLT * 8 + 1]) * fl);
                }
            }
            ok = __all_sync(0xffffffffu, fp_epi_sync(ep_bar, ep_phase, abort));   // E is free again
        }
    } else {
        // ------------------------------------------------------------- staging
        const int stid = (warp < 4 ? warp - 2 : warp - 6) * 32 + lane;
        pdl_wait();   // the intermediate comes from the previous kernel
        // slots per thread kept in flight for a tile, and how many tiles ahead
        // they are loaded: the folded intermediate needs one slot per thread
        // per tile (eight latitude pairs), so its loads run FP_FOLD_DEPTH tiles
        // ahead (a ring of registers: q[d] holds tile i + d)
        constexpr int SL = FOLD ? 1 : FP_SLOTS, DEPTH = FOLD ? FP_FOLD_DEPTH : 1;
        F3Slot q[DEPTH + 1][SL];
        auto load = [&](const TcFwd3Args &A, int4 jb, int t, int sl, F3Slot &v) {
            if constexpr (FOLD)
                f3_load_fold<NLT>(A, jb.x, jb.y & 0xffff, jb.z, jb.w & 0xff, jb.z == 0, t, jb.w >> 8, sl, v);
            else
                f3_load<NLT>(A, jb.x, jb.y & 0xffff, jb.z, jb.w & 0xff, jb.z == 0, t, sl, v);
        };
        auto store = [&](int t, int p, int sl, int njc, unsigned char *bt, const F3Slot &v) {
            if constexpr (FOLD) f3_store_fold<NLT>(t, sl, njc, bt, v);
            else f3_store<NLT>(t, p, sl, njc, bt, v);
        };
#pragma unroll
        for (int d = 0; d < DEPTH; d++) {
            if (d < ntile) {
                const int4 jb = job(d);
#pragma unroll
                for (int k = 0; k < SL; k++) load(P.seg[jb.y >> 16], jb, d & 3, stid + k * FP_NST, q[d][k]);
            }
        }
        for (int i = 0; i < ntile; i++) {
            const int b = i & 1, u = i >> 1, t = i & 3;
            const int4 jb = job(i);
            const TcFwd3Args &A = P.seg[jb.y >> 16];
            const int njc = A.njc, p = jb.w >> 8;
            if (i + DEPTH < ntile) {
                // later tiles' loads are in flight while this one is stored
                const int4 jn = job(i + DEPTH);
#pragma unroll
                for (int k = 0; k < SL; k++) load(P.seg[jn.y >> 16], jn, (i + DEPTH) & 3, stid + k * FP_NST, q[DEPTH][k]);
            }
            if (!fp_wait(op_empty + b, (u & 1) ^ 1, abort)) break;
            unsigned char *bt = opr + b * LY.ob;
            const int nslot = (fwd_ncp<NLT>(t) >> 1) * (FOLD ? (njc >> 3) : (njc >> 2));
#pragma unroll
            for (int k = 0; k < SL; k++)
                if (stid + k * FP_NST < nslot) store(t, p, stid + k * FP_NST, njc, bt, q[0][k]);
            for (int s = stid + SL * FP_NST; s < nslot; s += FP_NST) {   // beyond the slots in flight
                F3Slot v;
                load(A, jb, t, s, v);
                store(t, p, s, njc, bt, v);
            }
            tc::fence_proxy_async();   // these stores feed the tensor cores
            tc::mbar_arrive(op_full + b);
#pragma unroll
            for (int d = 0; d < DEPTH; d++)
#pragma unroll
                for (int k = 0; k < SL; k++) q[d][k] = q[d + 1][k];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (*abort && tid == 0) atomicExch(&g_tc_error, 7);
    if (warp == 0) tc::tmem_dealloc(tmem, 512);
}
