// By-reference entry points under the reference's gfortran names
// (include/exotx_fortran.h): host arrays of the model's real kind in, host
// arrays out, dimensions from one registration made by exotx_legini_.
//
// Each call stages its arrays through one device arena: host arrays of the
// compute precision are copied straight into their device slots; arrays of
// the other kind are copied into a staging slot and converted by a kernel.
// Everything runs on the registration's stream and the call returns after a
// stream synchronisation, since the Fortran caller reads its outputs next.
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <mutex>
#include <vector>
#include "exotx_internal.cuh"
#include "exotx_fortran.h"

namespace exotx {

template <typename Tin, typename Tout>
__global__ void k_convert(const Tin *__restrict__ in, Tout *__restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (Tout)in[i];
}

// element-wise FP64 <-> FP32 conversion of device arrays (round to nearest)
exotx_status convert_reals(const void *in, size_t in_esz, void *out, size_t out_esz, size_t n, cudaStream_t s) {
    if (n == 0) return EXOTX_OK;
    if (!((in_esz == 8 && out_esz == 4) || (in_esz == 4 && out_esz == 8))) return EXOTX_BAD_ARG;
    const int block = 256;
    const int grid = (int)std::min<size_t>((n + block - 1) / block, 148 * 16);
    if (in_esz == 8)
        k_convert<double, float><<<grid, block, 0, s>>>((const double *)in, (float *)out, n);
    else
        k_convert<float, double><<<grid, block, 0, s>>>((const float *)in, (double *)out, n);
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}

struct FortranCtx {
    exotx_plan plan = nullptr;
    int nlev = 0, real_bytes = 8, prec = EXOTX_FP64;
    cudaStream_t s = nullptr;
    unsigned char *arena = nullptr;
    size_t arena_bytes = 0, used = 0;
    int stop_on_error = 1;
    exotx_status last = EXOTX_OK;
};
static FortranCtx g_f;
static std::mutex g_f_mu;

static exotx_status ctx_stream() {
    if (!g_f.s) EXOTX_CUDA(cudaStreamCreateWithFlags(&g_f.s, cudaStreamNonBlocking));
    return EXOTX_OK;
}

// the arena holds every slot of one call; it only grows
static exotx_status arena_reserve(size_t bytes) {
    g_f.used = 0;
    if (g_f.arena_bytes >= bytes) return EXOTX_OK;
    if (g_f.arena) {
        EXOTX_CUDA(cudaStreamSynchronize(g_f.s));
        cudaFree(g_f.arena);
        g_f.arena = nullptr;
        g_f.arena_bytes = 0;
    }
    EXOTX_CUDA(cudaMalloc(&g_f.arena, bytes));
    g_f.arena_bytes = bytes;
    return EXOTX_OK;
}
static void *arena_take(size_t bytes) {
    void *p = g_f.arena + g_f.used;
    g_f.used += (bytes + 255) & ~(size_t)255;
    return p;
}
static size_t slot_bytes(size_t n, size_t esz) { return (n * esz + 255) & ~(size_t)255; }

// A host array of n reals of the registered kind, seen on the device as an
// array of the compute element size dev_esz.
struct Arr {
    void *host;
    size_t n;
    bool in, out;
    void *dev = nullptr;    // compute-kind slot
    void *stage = nullptr;  // host-kind slot when the kinds differ
};

static size_t arrs_bytes(const std::vector<Arr> &a, size_t dev_esz) {
    size_t b = 0;
    for (const Arr &x : a) {
        b += slot_bytes(x.n, dev_esz);
        if ((size_t)g_f.real_bytes != dev_esz) b += slot_bytes(x.n, (size_t)g_f.real_bytes);
    }
    return b;
}

static exotx_status convert(const void *in, size_t in_esz, void *out, size_t out_esz, size_t n) {
    return convert_reals(in, in_esz, out, out_esz, n, g_f.s);
}

// carve the slots and copy the inputs in
static exotx_status stage_in(std::vector<Arr> &a, size_t dev_esz) {
    EXOTX_TRY(arena_reserve(arrs_bytes(a, dev_esz)));
    const size_t hesz = (size_t)g_f.real_bytes;
    for (Arr &x : a) {
        x.dev = arena_take(x.n * dev_esz);
        if (hesz != dev_esz) x.stage = arena_take(x.n * hesz);
        if (!x.in || x.n == 0) continue;
        if (hesz == dev_esz) {
            EXOTX_CUDA(cudaMemcpyAsync(x.dev, x.host, x.n * hesz, cudaMemcpyHostToDevice, g_f.s));
        } else {
            EXOTX_CUDA(cudaMemcpyAsync(x.stage, x.host, x.n * hesz, cudaMemcpyHostToDevice, g_f.s));
            EXOTX_TRY(convert(x.stage, hesz, x.dev, dev_esz, x.n));
        }
    }
    return EXOTX_OK;
}

// copy the outputs back and wait for them
static exotx_status stage_out(std::vector<Arr> &a, size_t dev_esz) {
    const size_t hesz = (size_t)g_f.real_bytes;
    for (Arr &x : a) {
        if (!x.out || x.n == 0) continue;
        if (hesz == dev_esz) {
            EXOTX_CUDA(cudaMemcpyAsync(x.host, x.dev, x.n * hesz, cudaMemcpyDeviceToHost, g_f.s));
        } else {
            EXOTX_TRY(convert(x.dev, dev_esz, x.stage, hesz, x.n));
            EXOTX_CUDA(cudaMemcpyAsync(x.host, x.stage, x.n * hesz, cudaMemcpyDeviceToHost, g_f.s));
        }
    }
    EXOTX_CUDA(cudaStreamSynchronize(g_f.s));
    int err = 0;
    EXOTX_TRY(exotx_tc_error(&err, g_f.s));
    return err ? EXOTX_TIMEOUT : EXOTX_OK;
}

// record a call's status; with stop_on_error a failure ends the program as the
// reference's stop does
static void finish(const char *name, exotx_status st) {
    if (st == EXOTX_OK) return;
    g_f.last = st;
    if (g_f.stop_on_error) {
        fprintf(stderr, "exotx: %s failed: %s\n", name, exotx_status_string(st));
        fflush(stderr);
        exit(1);
    }
}

static size_t dev_esz_legendre() { return g_f.prec == EXOTX_FP64 ? 8 : 4; }

// one Legendre routine: arrays in/out, then fn(device pointers) on the stream
template <typename Fn>
static exotx_status legendre_call(std::vector<Arr> a, Fn fn) {
    if (!g_f.plan) return EXOTX_BAD_ARG;
    for (const Arr &x : a) if (!x.host) return EXOTX_BAD_ARG;
    EXOTX_TRY(ctx_stream());
    const size_t esz = dev_esz_legendre();
    EXOTX_TRY(stage_in(a, esz));
    std::vector<void *> d;
    for (Arr &x : a) d.push_back(x.dev);
    // a single routine under EXOTX_MIXED runs the FP32 kernels
    const int prec = g_f.prec == EXOTX_FP64 ? EXOTX_FP64 : EXOTX_FP32;
    EXOTX_TRY(fn(prec, d.data()));
    return stage_out(a, esz);
}

static size_t nrsp() { return 2 * (size_t)g_f.plan->ncsp; }
static size_t nfc() { return (size_t)g_f.plan->nlat * g_f.plan->nlon; }

}  // namespace exotx

using namespace exotx;

EXOTX_API void exotx_legini_(const int *nlat, const int *nlev, const int *real_bytes, const int *prec,
                             const int *nfilter, const int *ngptfilter, const int *nspvfilter,
                             const double *landhoskn0, const double *filterkappa, const int *nfilterexp,
                             const double *plavor, int *ierr) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    exotx_status st = EXOTX_OK;
    if (!nlat || !nlev || !real_bytes || !prec || !nfilter || !ngptfilter || !nspvfilter || !landhoskn0 ||
        !filterkappa || !nfilterexp || !plavor || *nlev < 1 || (*real_bytes != 4 && *real_bytes != 8) ||
        (*prec != EXOTX_FP64 && *prec != EXOTX_FP32 && *prec != EXOTX_MIXED)) {
        st = EXOTX_BAD_ARG;
    } else {
        exotx_grid_desc d;
        st = exotx_grid_desc_default(*nlat, &d);
        if (st == EXOTX_OK) {
            d.nfilter = *nfilter;
            d.ngptfilter = *ngptfilter;
            d.nspvfilter = *nspvfilter;
            d.landhoskn0 = *landhoskn0;
            d.filterkappa = *filterkappa;
            d.nfilterexp = *nfilterexp;
            d.plavor = *plavor;
            exotx_plan p = nullptr;
            st = exotx_plan_create(&d, &p);
            if (st == EXOTX_OK) {
                if (g_f.plan) exotx_plan_destroy(g_f.plan);
                g_f.plan = p;
                g_f.nlev = *nlev;
                g_f.real_bytes = *real_bytes;
                g_f.prec = *prec;
            }
        }
    }
    if (ierr) *ierr = (int)st;
    if (st != EXOTX_OK) g_f.last = st;
}

EXOTX_API void exotx_legfree_(void) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    if (g_f.s) cudaStreamSynchronize(g_f.s);
    if (g_f.plan) exotx_plan_destroy(g_f.plan);
    if (g_f.arena) cudaFree(g_f.arena);
    g_f.plan = nullptr;
    g_f.arena = nullptr;
    g_f.arena_bytes = 0;
    g_f.nlev = 0;
    g_f.real_bytes = 8;
    g_f.prec = EXOTX_FP64;
}

EXOTX_API void exotx_fortran_status_(int *ierr) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    if (ierr) *ierr = (int)g_f.last;
    g_f.last = EXOTX_OK;
}

EXOTX_API void exotx_stop_on_error_(const int *flag) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    g_f.stop_on_error = flag ? (*flag != 0) : 1;
}

EXOTX_API void inigau_(const int *klat, double *pz0, double *pzw) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    auto run = [&]() -> exotx_status {
        if (!klat || !pz0 || !pzw || *klat < 2) return EXOTX_BAD_ARG;
        EXOTX_TRY(ctx_stream());
        EXOTX_TRY(arena_reserve(2 * slot_bytes((size_t)*klat, 8)));
        double *d0 = (double *)arena_take(8 * (size_t)*klat), *dw = (double *)arena_take(8 * (size_t)*klat);
        EXOTX_TRY(exotx_inigau(*klat, d0, dw, g_f.s));
        EXOTX_CUDA(cudaMemcpyAsync(pz0, d0, 8 * (size_t)*klat, cudaMemcpyDeviceToHost, g_f.s));
        EXOTX_CUDA(cudaMemcpyAsync(pzw, dw, 8 * (size_t)*klat, cudaMemcpyDeviceToHost, g_f.s));
        EXOTX_CUDA(cudaStreamSynchronize(g_f.s));
        return EXOTX_OK;
    };
    finish("inigau", run());
}

EXOTX_API void sp2fc_(const void *sp, void *fc) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    exotx_status st = !g_f.plan ? EXOTX_BAD_ARG : legendre_call(
        {{(void *)sp, nrsp(), true, false}, {fc, nfc(), false, true}},
        [](int prec, void **d) { return exotx_sp2fc(g_f.plan, prec, d[0], d[1], 1, g_f.s); });
    finish("sp2fc", st);
}

EXOTX_API void sp2fcdmu_(const void *sp, void *fc) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    exotx_status st = !g_f.plan ? EXOTX_BAD_ARG : legendre_call(
        {{(void *)sp, nrsp(), true, false}, {fc, nfc(), false, true}},
        [](int prec, void **d) { return exotx_sp2fcdmu(g_f.plan, prec, d[0], d[1], 1, g_f.s); });
    finish("sp2fcdmu", st);
}

EXOTX_API void fc2sp_(const void *fc, void *sp) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    exotx_status st = !g_f.plan ? EXOTX_BAD_ARG : legendre_call(
        {{(void *)fc, nfc(), true, false}, {sp, nrsp(), false, true}},
        [](int prec, void **d) { return exotx_fc2sp(g_f.plan, prec, d[0], d[1], 1, g_f.s); });
    finish("fc2sp", st);
}

EXOTX_API void dv2uv_(const void *pd, const void *pz, void *pu, void *pv) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    exotx_status st = EXOTX_BAD_ARG;
    if (g_f.plan) {
        const size_t L = (size_t)g_f.nlev;
        st = legendre_call({{(void *)pd, L * nrsp(), true, false}, {(void *)pz, L * nrsp(), true, false},
                            {pu, L * nfc(), false, true}, {pv, L * nfc(), false, true}},
                           [](int prec, void **d) {
                               return exotx_dv2uv(g_f.plan, prec, d[0], d[1], d[2], d[3], g_f.nlev, g_f.s);
                           });
    }
    finish("dv2uv", st);
}

EXOTX_API void uv2dv_(const void *pu, const void *pv, void *pd, void *pz) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    exotx_status st = EXOTX_BAD_ARG;
    if (g_f.plan) {
        const size_t L = (size_t)g_f.nlev;
        st = legendre_call({{(void *)pu, L * nfc(), true, false}, {(void *)pv, L * nfc(), true, false},
                            {pd, L * nrsp(), false, true}, {pz, L * nrsp(), false, true}},
                           [](int prec, void **d) {
                               return exotx_uv2dv(g_f.plan, prec, d[0], d[1], d[2], d[3], g_f.nlev, g_f.s);
                           });
    }
    finish("uv2dv", st);
}

EXOTX_API void qtend_(void *q, const void *qn, const void *uq, const void *vq) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    exotx_status st = EXOTX_BAD_ARG;
    if (g_f.plan) {
        const size_t L = (size_t)g_f.nlev;
        st = legendre_call({{q, L * nrsp(), false, true}, {(void *)qn, L * nfc(), true, false},
                            {(void *)uq, L * nfc(), true, false}, {(void *)vq, L * nfc(), true, false}},
                           [](int prec, void **d) {
                               return exotx_qtend(g_f.plan, prec, d[0], d[1], d[2], d[3], g_f.nlev, g_f.s);
                           });
    }
    finish("qtend", st);
}

EXOTX_API void mktend_(void *d, void *t, void *z, const void *tn, const void *fu, const void *fv, const void *ke,
                       const void *ut, const void *vt) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    exotx_status st = EXOTX_BAD_ARG;
    if (g_f.plan) {
        const size_t L = (size_t)g_f.nlev, S = L * nrsp(), F = L * nfc();
        st = legendre_call({{d, S, false, true}, {t, S, false, true}, {z, S, false, true},
                            {(void *)tn, F, true, false}, {(void *)fu, F, true, false},
                            {(void *)fv, F, true, false}, {(void *)ke, F, true, false},
                            {(void *)ut, F, true, false}, {(void *)vt, F, true, false}},
                           [](int prec, void **a) {
                               return exotx_mktend(g_f.plan, prec, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7],
                                                   a[8], g_f.nlev, g_f.s);
                           });
    }
    finish("mktend", st);
}

// the FFTs need no registration: without one they run in the host's kind (8 bytes)
static exotx_status fft_call(void *a, const int *n, const int *lot, bool forward) {
    if (!a || !n || !lot || *lot < 0) return EXOTX_BAD_ARG;
    if (!exotx_fft_supported(*n)) return EXOTX_UNSUPPORTED_N;
    if (*lot == 0) return EXOTX_OK;
    EXOTX_TRY(ctx_stream());
    const size_t esz = g_f.prec == EXOTX_FP64 ? 8 : 4;
    const int prec = esz == 8 ? EXOTX_FP64 : EXOTX_FP32;
    std::vector<Arr> arr = {{a, (size_t)*n * (size_t)*lot, true, true}};
    EXOTX_TRY(stage_in(arr, esz));
    if (forward) EXOTX_TRY(exotx_gp2fc(prec, arr[0].dev, *n, *lot, g_f.s));
    else EXOTX_TRY(exotx_fc2gp(prec, arr[0].dev, *n, *lot, g_f.s));
    return stage_out(arr, esz);
}

EXOTX_API void gp2fc_(void *a, const int *n, const int *lot) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    finish("gp2fc", fft_call(a, n, lot, true));
}

EXOTX_API void fc2gp_(void *a, const int *n, const int *lot) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    finish("fc2gp", fft_call(a, n, lot, false));
}

EXOTX_API void radstep_(const exotx_rad_params *par, const exotx_rad_io *io) {
    std::lock_guard<std::mutex> lk(g_f_mu);
    auto run = [&]() -> exotx_status {
        if (!par || !io) return EXOTX_BAD_ARG;
        const size_t H = (size_t)par->nhor, L = (size_t)par->nlev, E = L + 1;
        if (par->nhor < 1 || par->nlev < 2 || par->nlon < 1) return EXOTX_BAD_DIM;
        const size_t rows = (size_t)(par->nhor / par->nlon);
        // (io field, length, read, written): the reference's array roles
        struct F { const void *const *h; void **d; size_t n; bool in, out; };
        exotx_rad_io dio = {};
        const F fields[] = {
            {&io->sid, (void **)&dio.sid, rows, true, false},
            {&io->cola, (void **)&dio.cola, rows, true, false},
            {&io->dt, (void **)&dio.dt, E * H, true, false},
            {&io->dq, (void **)&dio.dq, E * H, true, false},
            {&io->dcc, (void **)&dio.dcc, E * H, true, false},
            {&io->dql, (void **)&dio.dql, E * H, true, false},
            {&io->dqco2, (void **)&dio.dqco2, L * H, true, false},
            {&io->dp, (void **)&dio.dp, H, true, false},
            {&io->dls, (void **)&dio.dls, H, true, false},
            {&io->dicec, (void **)&dio.dicec, H, true, false},
            {(const void *const *)&io->dqo3, &dio.dqo3, L * H, true, true},
            {(const void *const *)&io->gmu0, &dio.gmu0, H, true, true},
            {(const void *const *)&io->dalb, &dio.dalb, H, true, true},
            {(const void *const *)&io->dsalb, &dio.dsalb, 2 * H, true, true},
            {(const void *const *)&io->dfu, &dio.dfu, E * H, false, true},
            {(const void *const *)&io->dfd, &dio.dfd, E * H, false, true},
            {(const void *const *)&io->dftu, &dio.dftu, E * H, false, true},
            {(const void *const *)&io->dftd, &dio.dftd, E * H, false, true},
            {(const void *const *)&io->dswfl, &dio.dswfl, E * H, false, true},
            {(const void *const *)&io->dlwfl, &dio.dlwfl, E * H, false, true},
            {(const void *const *)&io->dflux, &dio.dflux, E * H, false, true},
            {(const void *const *)&io->dtdt, &dio.dtdt, L * H, true, true},
            {(const void *const *)&io->dtdtswr, &dio.dtdtswr, L * H, false, true},
            {(const void *const *)&io->dtdtlwr, &dio.dtdtlwr, L * H, false, true},
            {(const void *const *)&io->dconv, &dio.dconv, L * H, false, true},
            {&io->zsol, (void **)&dio.zsol, 3 * H, true, false},
        };
        std::vector<Arr> arr;
        std::vector<void **> dst;
        for (const F &f : fields) {
            if (!*f.h) continue;  // absent optional arrays stay NULL (radstep checks the rest)
            arr.push_back({(void *)*f.h, f.n, f.in, f.out});
            dst.push_back(f.d);
        }
        EXOTX_TRY(ctx_stream());
        const size_t esz = g_f.prec == EXOTX_FP64 ? 8 : 4;
        EXOTX_TRY(stage_in(arr, esz));
        for (size_t i = 0; i < arr.size(); i++) *dst[i] = arr[i].dev;
        EXOTX_TRY(exotx_radstep(par, esz == 8 ? EXOTX_FP64 : EXOTX_FP32, &dio, g_f.s));
        return stage_out(arr, esz);
    };
    finish("radstep", run());
}
