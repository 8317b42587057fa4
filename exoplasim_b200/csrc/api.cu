// C-ABI entry points of the transform core (see include/exotx.h).
#include <cstring>
#include "exotx_internal.cuh"

namespace exotx {

// reference layout fc(2,NLON/2,NLAT,nlev)
static FourierLayout ref_layout(exotx_plan p) {
    return FourierLayout{(long long)p->nlat * (p->nlon / 2), p->nlon / 2, 1, p->nlon / 2};
}
// m-major intermediate: complex (field f, lat l, m) at m*nrows + f*nlat + l
static FourierLayout mmajor_layout(exotx_plan p, long long nrows) {
    return FourierLayout{p->nlat, 1, nrows, p->ntp1};
}

static bool prec_ok(int prec) { return prec == EXOTX_FP64 || prec == EXOTX_FP32 || prec == EXOTX_MIXED; }

template <typename T>
static exotx_status inverse_set_simt(exotx_plan p, const T *spin, T *gpout, int L, cudaStream_t s) {
    const long long nrsp = 2LL * p->ncsp, nhor = (long long)p->nlat * p->nlon;
    const long long nfld = 6LL * L + 3, nrows = nfld * p->nlat;
    EXOTX_TRY(ensure_work(p, sizeof(T) * 2 * (size_t)nrows * p->ntp1));
    T *w = (T *)p->d_work;
    FourierLayout F = mmajor_layout(p, nrows);
    const T *sd = spin, *st = spin + L * nrsp, *sz = spin + 2 * L * nrsp, *sq = spin + 3 * L * nrsp,
            *sp = spin + 4 * L * nrsp;
    // intermediate field offsets (complex units): field f occupies rows f*nlat..
    auto fld = [&](long long f) { return w + 2 * f * p->nlat; };
    // gu[L] gv[L] gt[L] gd[L] gz[L] gq[L] gpj gpmt gp
    EXOTX_TRY(leg_inverse_l<T>(p, OP_DV2UV, sd, sz, fld(0), fld(L), L, nrsp, nrsp, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FC, st, nullptr, fld(2 * L), nullptr, L, nrsp, 0, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FC, sd, nullptr, fld(3 * L), nullptr, L, nrsp, 0, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FC, sz, nullptr, fld(4 * L), nullptr, L, nrsp, 0, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FC, sq, nullptr, fld(5 * L), nullptr, L, nrsp, 0, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FCDMU, sp, nullptr, fld(6 * L), nullptr, 1, nrsp, 0, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FC_GPMT, sp, nullptr, fld(6 * L + 2), fld(6 * L + 1), 1, nrsp, 0, F, s));
    (void)nhor;
    return fft_inverse_l<T>(w, gpout, p->nlon, nrows, p->ntp1, 1, nrows, s);
}

template <typename T>
static exotx_status forward_set_simt(exotx_plan p, const T *gpin, T *spout, int L, cudaStream_t s) {
    const long long nrsp = 2LL * p->ncsp;
    const long long nfld = 9LL * L + 1, nrows = nfld * p->nlat;
    EXOTX_TRY(ensure_work(p, sizeof(T) * 2 * (size_t)nrows * p->ntp1));
    T *w = (T *)p->d_work;
    EXOTX_TRY(fft_forward_l<T>(gpin, w, p->nlon, nrows, p->ntp1, 1, nrows, s));
    FourierLayout F = mmajor_layout(p, nrows);
    auto fld = [&](long long f) -> const T * { return w + 2 * f * p->nlat; };
    // gtn[L] gqn[L] gut[L] gvt[L] guz[L] gvz[L] gke[L] gvpp guq[L] gvq[L]
    const T *gtn = fld(0), *gqn = fld(L), *gut = fld(2 * L), *gvt = fld(3 * L), *guz = fld(4 * L),
            *gvz = fld(5 * L), *gke = fld(6 * L), *gvpp = fld(7 * L), *guq = fld(7 * L + 1),
            *gvq = fld(8 * L + 1);
    T *sdf = spout, *stf = spout + L * nrsp, *szf = spout + 2 * L * nrsp, *sqf = spout + 3 * L * nrsp,
      *spf = spout + 4 * L * nrsp;
    {
        const T *in[1] = {gvpp};
        T *out[1] = {spf};
        EXOTX_TRY(leg_forward_l<T>(p, OP_FC2SP, in, out, 1, F, nrsp, s));
    }
    {
        // mktend(sdf,stf,szf,gtn,gvz,guz,gke,gut,gvt)  (plasim.f90:2478)
        const T *in[6] = {gtn, gvz, guz, gke, gut, gvt};
        T *out[3] = {sdf, stf, szf};
        EXOTX_TRY(leg_forward_l<T>(p, OP_MKTEND, in, out, L, F, nrsp, s));
    }
    {
        const T *in[3] = {gqn, guq, gvq};
        T *out[1] = {sqf};
        EXOTX_TRY(leg_forward_l<T>(p, OP_QTEND, in, out, L, F, nrsp, s));
    }
    return EXOTX_OK;
}

// gridpointd (plasim.f90:3142-3149): invlegd (legmod.f90:661-677) and fc2gp.
// spin (4L+1 fields) sd, st, sz, sq, sp -> gpout (4L+1) gu, gv, gt, gq, gp
template <typename T>
static exotx_status inverse_set_d_simt(exotx_plan p, const T *spin, T *gpout, int L, cudaStream_t s) {
    const long long nrsp = 2LL * p->ncsp;
    const long long nfld = 4LL * L + 1, nrows = nfld * p->nlat;
    EXOTX_TRY(ensure_work(p, sizeof(T) * 2 * (size_t)nrows * p->ntp1));
    T *w = (T *)p->d_work;
    FourierLayout F = mmajor_layout(p, nrows);
    const T *sd = spin, *st = spin + L * nrsp, *sz = spin + 2 * L * nrsp, *sq = spin + 3 * L * nrsp,
            *sp = spin + 4 * L * nrsp;
    auto fld = [&](long long f) { return w + 2 * f * p->nlat; };
    EXOTX_TRY(leg_inverse_l<T>(p, OP_DV2UV, sd, sz, fld(0), fld(L), L, nrsp, nrsp, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FC, st, nullptr, fld(2 * L), nullptr, L, nrsp, 0, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FC, sq, nullptr, fld(3 * L), nullptr, L, nrsp, 0, F, s));
    EXOTX_TRY(leg_inverse_l<T>(p, OP_SP2FC, sp, nullptr, fld(4 * L), nullptr, 1, nrsp, 0, F, s));
    return fft_inverse_l<T>(w, gpout, p->nlon, nrows, p->ntp1, 1, nrows, s);
}

// gridpointd (plasim.f90:3415-3428): gp2fc, fc2sp of the temperature and
// humidity tendencies, uv2dv.  gpin (4L) gtdt, gudt, gvdt, gqdt -> spout (4L) sdf, stf, szf, sqf
template <typename T>
static exotx_status forward_set_d_simt(exotx_plan p, const T *gpin, T *spout, int L, cudaStream_t s) {
    const long long nrsp = 2LL * p->ncsp;
    const long long nfld = 4LL * L, nrows = nfld * p->nlat;
    EXOTX_TRY(ensure_work(p, sizeof(T) * 2 * (size_t)nrows * p->ntp1));
    T *w = (T *)p->d_work;
    EXOTX_TRY(fft_forward_l<T>(gpin, w, p->nlon, nrows, p->ntp1, 1, nrows, s));
    FourierLayout F = mmajor_layout(p, nrows);
    auto fld = [&](long long f) -> const T * { return w + 2 * f * p->nlat; };
    const T *gtdt = fld(0), *gudt = fld(L), *gvdt = fld(2 * L), *gqdt = fld(3 * L);
    T *sdf = spout, *stf = spout + L * nrsp, *szf = spout + 2 * L * nrsp, *sqf = spout + 3 * L * nrsp;
    {
        const T *in[1] = {gtdt};
        T *out[1] = {stf};
        EXOTX_TRY(leg_forward_l<T>(p, OP_FC2SP, in, out, L, F, nrsp, s));
    }
    {
        const T *in[1] = {gqdt};
        T *out[1] = {sqf};
        EXOTX_TRY(leg_forward_l<T>(p, OP_FC2SP, in, out, L, F, nrsp, s));
    }
    {
        const T *in[2] = {gudt, gvdt};
        T *out[2] = {sdf, szf};
        EXOTX_TRY(leg_forward_l<T>(p, OP_UV2DV, in, out, L, F, nrsp, s));
    }
    return EXOTX_OK;
}

}  // namespace exotx

using namespace exotx;

#define PLAN_PREC_CHECK(p, prec)                      \
    do {                                              \
        if (!(p) || !prec_ok(prec)) return EXOTX_BAD_ARG; \
    } while (0)

template <typename Fn>
static exotx_status by_prec(int prec, Fn fn) {
    if (prec == EXOTX_FP64) return fn((double *)nullptr);
    return fn((float *)nullptr);
}

static exotx_status inv_api(exotx_plan p, int prec, int op, const void *a, const void *b, void *oa, void *ob,
                            int nlev, exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (nlev == 0) return EXOTX_OK;
    if (!a || !oa || nlev < 0 || ((op == OP_DV2UV) && (!b || !ob))) return EXOTX_BAD_ARG;
    const long long nrsp = 2LL * p->ncsp;
    FourierLayout F = ref_layout(p);
    return by_prec(prec, [&](auto tag) {
        using T = std::remove_pointer_t<decltype(tag)>;
        return leg_inverse_l<T>(p, op, (const T *)a, (const T *)b, (T *)oa, (T *)ob, nlev, nrsp, nrsp, F,
                                (cudaStream_t)s);
    });
}

EXOTX_API exotx_status exotx_sp2fc(exotx_plan p, int prec, const void *sp, void *fc, int nlev, exotx_stream s) {
    return inv_api(p, prec, OP_SP2FC, sp, nullptr, fc, nullptr, nlev, s);
}
EXOTX_API exotx_status exotx_sp2fcdmu(exotx_plan p, int prec, const void *sp, void *fc, int nlev,
                                      exotx_stream s) {
    return inv_api(p, prec, OP_SP2FCDMU, sp, nullptr, fc, nullptr, nlev, s);
}
EXOTX_API exotx_status exotx_dv2uv(exotx_plan p, int prec, const void *pd, const void *pz, void *pu, void *pv,
                                   int nlev, exotx_stream s) {
    return inv_api(p, prec, OP_DV2UV, pd, pz, pu, pv, nlev, s);
}

static exotx_status fwd_api(exotx_plan p, int prec, int op, const void *const *in, int nin, void *const *out,
                            int nout, int nlev, exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (nlev < 0) return EXOTX_BAD_ARG;
    if (nlev == 0) return EXOTX_OK;
    for (int i = 0; i < nin; i++) if (!in[i]) return EXOTX_BAD_ARG;
    for (int i = 0; i < nout; i++) if (!out[i]) return EXOTX_BAD_ARG;
    const long long nrsp = 2LL * p->ncsp;
    FourierLayout F = ref_layout(p);
    return by_prec(prec, [&](auto tag) {
        using T = std::remove_pointer_t<decltype(tag)>;
        const T *ii[6] = {};
        T *oo[3] = {};
        for (int i = 0; i < nin; i++) ii[i] = (const T *)in[i];
        for (int i = 0; i < nout; i++) oo[i] = (T *)out[i];
        return leg_forward_l<T>(p, op, ii, oo, nlev, F, nrsp, (cudaStream_t)s);
    });
}

EXOTX_API exotx_status exotx_fc2sp(exotx_plan p, int prec, const void *fc, void *sp, int nlev, exotx_stream s) {
    const void *in[1] = {fc};
    void *out[1] = {sp};
    return fwd_api(p, prec, OP_FC2SP, in, 1, out, 1, nlev, s);
}
EXOTX_API exotx_status exotx_uv2dv(exotx_plan p, int prec, const void *pu, const void *pv, void *pd, void *pz,
                                   int nlev, exotx_stream s) {
    const void *in[2] = {pu, pv};
    void *out[2] = {pd, pz};
    return fwd_api(p, prec, OP_UV2DV, in, 2, out, 2, nlev, s);
}
EXOTX_API exotx_status exotx_mktend(exotx_plan p, int prec, void *d, void *t, void *z, const void *tn,
                                    const void *fu, const void *fv, const void *ke, const void *ut,
                                    const void *vt, int nlev, exotx_stream s) {
    const void *in[6] = {tn, fu, fv, ke, ut, vt};
    void *out[3] = {d, t, z};
    return fwd_api(p, prec, OP_MKTEND, in, 6, out, 3, nlev, s);
}
EXOTX_API exotx_status exotx_qtend(exotx_plan p, int prec, void *q, const void *qn, const void *uq,
                                   const void *vq, int nlev, exotx_stream s) {
    const void *in[3] = {qn, uq, vq};
    void *out[1] = {q};
    return fwd_api(p, prec, OP_QTEND, in, 3, out, 1, nlev, s);
}

EXOTX_API exotx_status exotx_gp2fc(int prec, void *a, int n, int lot, exotx_stream s) {
    if (lot == 0 && prec_ok(prec) && exotx_fft_supported(n)) return EXOTX_OK;
    if (!a || lot < 0 || !prec_ok(prec)) return EXOTX_BAD_ARG;
    if (!exotx_fft_supported(n)) return EXOTX_UNSUPPORTED_N;
    return by_prec(prec, [&](auto tag) {
        using T = std::remove_pointer_t<decltype(tag)>;
        return fft_forward_l<T>((const T *)a, (T *)a, n, lot, n / 2, n / 2, 1, (cudaStream_t)s);
    });
}
EXOTX_API exotx_status exotx_fc2gp(int prec, void *a, int n, int lot, exotx_stream s) {
    if (lot == 0 && prec_ok(prec) && exotx_fft_supported(n)) return EXOTX_OK;
    if (!a || lot < 0 || !prec_ok(prec)) return EXOTX_BAD_ARG;
    if (!exotx_fft_supported(n)) return EXOTX_UNSUPPORTED_N;
    return by_prec(prec, [&](auto tag) {
        using T = std::remove_pointer_t<decltype(tag)>;
        return fft_inverse_l<T>((const T *)a, (T *)a, n, lot, n / 2, n / 2, 1, (cudaStream_t)s);
    });
}

EXOTX_API exotx_status exotx_inverse_set(exotx_plan p, int prec, const void *spin, void *gpout, int nlev,
                                         exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (!spin || !gpout || nlev < 1) return EXOTX_BAD_ARG;
    if (prec == EXOTX_FP64)
        return inverse_set_simt<double>(p, (const double *)spin, (double *)gpout, nlev, (cudaStream_t)s);
    if (prec == EXOTX_FP32)
        return inverse_set_simt<float>(p, (const float *)spin, (float *)gpout, nlev, (cudaStream_t)s);
    return tc_inverse_set(p, (const float *)spin, (float *)gpout, nlev, (cudaStream_t)s);
}

EXOTX_API exotx_status exotx_inverse_set_batch(exotx_plan p, int prec, const void *spin, void *gpout, int nlev,
                                               int ninst, exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (ninst == 0) return EXOTX_OK;
    if (!spin || !gpout || nlev < 1 || ninst < 0) return EXOTX_BAD_ARG;
    if (prec == EXOTX_MIXED)
        return tc_inverse_batch(p, (const float *)spin, (float *)gpout, nlev, ninst, (cudaStream_t)s);
    const size_t esz = prec == EXOTX_FP64 ? 8 : 4;
    const size_t in_b = (size_t)(4 * nlev + 1) * 2 * p->ncsp * esz;
    const size_t out_b = (size_t)(6 * nlev + 3) * p->nlat * p->nlon * esz;
    for (int i = 0; i < ninst; i++)
        EXOTX_TRY(exotx_inverse_set(p, prec, (const char *)spin + i * in_b, (char *)gpout + i * out_b, nlev, s));
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_forward_set_batch(exotx_plan p, int prec, const void *gpin, void *spout, int nlev,
                                               int ninst, exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (ninst == 0) return EXOTX_OK;
    if (!gpin || !spout || nlev < 1 || ninst < 0) return EXOTX_BAD_ARG;
    if (prec == EXOTX_MIXED)
        return tc_forward_batch(p, (const float *)gpin, (float *)spout, nlev, ninst, (cudaStream_t)s);
    const size_t esz = prec == EXOTX_FP64 ? 8 : 4;
    const size_t in_b = (size_t)(9 * nlev + 1) * p->nlat * p->nlon * esz;
    const size_t out_b = (size_t)(4 * nlev + 1) * 2 * p->ncsp * esz;
    for (int i = 0; i < ninst; i++)
        EXOTX_TRY(exotx_forward_set(p, prec, (const char *)gpin + i * in_b, (char *)spout + i * out_b, nlev, s));
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_tc_error(int *code, exotx_stream s) {
    if (!code) return EXOTX_BAD_ARG;
    int fe = 0;
    EXOTX_TRY(tc_error_read(code, (cudaStream_t)s));
    EXOTX_TRY(fft_error_read(&fe, (cudaStream_t)s));
    *code |= fe;
    EXOTX_TRY(fft_error_reset((cudaStream_t)s));
    return tc_error_reset((cudaStream_t)s);
}

EXOTX_API exotx_status exotx_forward_set(exotx_plan p, int prec, const void *gpin, void *spout, int nlev,
                                         exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (!gpin || !spout || nlev < 1) return EXOTX_BAD_ARG;
    if (prec == EXOTX_FP64)
        return forward_set_simt<double>(p, (const double *)gpin, (double *)spout, nlev, (cudaStream_t)s);
    if (prec == EXOTX_FP32)
        return forward_set_simt<float>(p, (const float *)gpin, (float *)spout, nlev, (cudaStream_t)s);
    return tc_forward_set(p, (const float *)gpin, (float *)spout, nlev, (cudaStream_t)s);
}

// ---- gridpointd sets ----
EXOTX_API exotx_status exotx_inverse_set_d(exotx_plan p, int prec, const void *spin, void *gpout, int nlev,
                                           exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (!spin || !gpout || nlev < 1) return EXOTX_BAD_ARG;
    if (prec == EXOTX_FP64)
        return inverse_set_d_simt<double>(p, (const double *)spin, (double *)gpout, nlev, (cudaStream_t)s);
    if (prec == EXOTX_FP32)
        return inverse_set_d_simt<float>(p, (const float *)spin, (float *)gpout, nlev, (cudaStream_t)s);
    return tc_inverse_batch_d(p, (const float *)spin, (float *)gpout, nlev, 1, (cudaStream_t)s);
}

EXOTX_API exotx_status exotx_forward_set_d(exotx_plan p, int prec, const void *gpin, void *spout, int nlev,
                                           exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (!gpin || !spout || nlev < 1) return EXOTX_BAD_ARG;
    if (prec == EXOTX_FP64)
        return forward_set_d_simt<double>(p, (const double *)gpin, (double *)spout, nlev, (cudaStream_t)s);
    if (prec == EXOTX_FP32)
        return forward_set_d_simt<float>(p, (const float *)gpin, (float *)spout, nlev, (cudaStream_t)s);
    return tc_forward_batch_d(p, (const float *)gpin, (float *)spout, nlev, 1, (cudaStream_t)s);
}

EXOTX_API exotx_status exotx_inverse_set_d_batch(exotx_plan p, int prec, const void *spin, void *gpout, int nlev,
                                                 int ninst, exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (ninst == 0) return EXOTX_OK;
    if (!spin || !gpout || nlev < 1 || ninst < 0) return EXOTX_BAD_ARG;
    if (prec == EXOTX_MIXED)
        return tc_inverse_batch_d(p, (const float *)spin, (float *)gpout, nlev, ninst, (cudaStream_t)s);
    const size_t esz = prec == EXOTX_FP64 ? 8 : 4;
    const size_t in_b = (size_t)(4 * nlev + 1) * 2 * p->ncsp * esz;
    const size_t out_b = (size_t)(4 * nlev + 1) * p->nlat * p->nlon * esz;
    for (int i = 0; i < ninst; i++)
        EXOTX_TRY(exotx_inverse_set_d(p, prec, (const char *)spin + i * in_b, (char *)gpout + i * out_b, nlev, s));
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_forward_set_d_batch(exotx_plan p, int prec, const void *gpin, void *spout, int nlev,
                                                 int ninst, exotx_stream s) {
    PLAN_PREC_CHECK(p, prec);
    if (ninst == 0) return EXOTX_OK;
    if (!gpin || !spout || nlev < 1 || ninst < 0) return EXOTX_BAD_ARG;
    if (prec == EXOTX_MIXED)
        return tc_forward_batch_d(p, (const float *)gpin, (float *)spout, nlev, ninst, (cudaStream_t)s);
    const size_t esz = prec == EXOTX_FP64 ? 8 : 4;
    const size_t in_b = (size_t)(4 * nlev) * p->nlat * p->nlon * esz;
    const size_t out_b = (size_t)(4 * nlev) * 2 * p->ncsp * esz;
    for (int i = 0; i < ninst; i++)
        EXOTX_TRY(exotx_forward_set_d(p, prec, (const char *)gpin + i * in_b, (char *)spout + i * out_b, nlev, s));
    return EXOTX_OK;
}
