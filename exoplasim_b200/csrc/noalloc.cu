// Forward transform set that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// transform.  A host model that hands all device memory to its own pool up
// front (so a later cudaMalloc fails or fragments that pool), and a timestep
// loop that must not stall on an allocation call (cudaMalloc and cudaFree may
// synchronise the device), cannot let exotx_forward_set grow the plan's
// Fourier work buffer or build its FFT twiddle tables on first use.  This
// variant keeps both in one fixed array of device memory that is part of the
// library: EXOTX_STATIC_WORK_BYTES bytes on each GPU, held from the library's
// first use on that GPU (module loading is lazy) until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents.  Each call reads only bytes that it, or an earlier call with the
// same grid length and precision, wrote: the twiddles are copied in by the
// first call on a device and again only when the grid length or precision
// changes (a per-device record says which twiddles the array holds), and the
// Fourier intermediate is written by the FFT kernel before the Legendre
// kernels read it, so nothing has to start at zero.  Calls whose work overlaps
// on the GPU (other streams, other host threads, without synchronisation
// between them) race on the array.
#include <cstring>
#include <mutex>
#include "exotx_internal.cuh"

namespace exotx {

// The scratch array.  In host code this name is only a stand-in for the
// device object; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_static_work[EXOTX_STATIC_WORK_BYTES];

constexpr int kMaxDevices = 64;
static std::mutex g_static_mu;
static void *g_static_addr[kMaxDevices];  // device address of the array, per device ordinal
// which twiddles the array of each device holds: grid length and element size
// (0 = none yet)
static int g_tw_nlon[kMaxDevices];
static int g_tw_esz[kMaxDevices];

// Set-up, once per device, with that device current.
static exotx_status static_work_addr(unsigned char **out) {
    int dev = -1;
    EXOTX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return EXOTX_BAD_ARG;
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_addr[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_static_work);
        if (e != cudaSuccess) return cuda_status(e);
        g_static_addr[dev] = ptr;
    }
    *out = static_cast<unsigned char *>(g_static_addr[dev]);
    return EXOTX_OK;
}

static size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// host staging for the twiddles (largest FFT length 4096: 2048 + 2049 complex)
static double g_tw64[2 * 2048 + 2 * 2049];
static float g_tw32[2 * 2048 + 2 * 2049];

template <typename T> static T *tw_host();
template <> double *tw_host<double>() { return g_tw64; }
template <> float *tw_host<float>() { return g_tw32; }

// bytes of the array one call needs: twiddles w (h complex), r (h+1 complex), then W
template <typename T>
static size_t static_need(exotx_plan p, int L, size_t *w_off, size_t *r_off, size_t *W_off) {
    const int h = p->nlon / 2;
    *w_off = 0;
    *r_off = round256(sizeof(T) * 2 * (size_t)h);
    *W_off = *r_off + round256(sizeof(T) * 2 * (size_t)(h + 1));
    const size_t nrows = (size_t)(9 * L + 1) * p->nlat;
    return *W_off + sizeof(T) * 2 * nrows * p->ntp1;
}

// forward set (plasim.f90 gridpointa :2462-2486): gp2fc of every field into the
// m-major Fourier intermediate, then fc2sp(gvpp), mktend and qtend
template <typename T>
static exotx_status forward_set_static(exotx_plan p, const T *gpin, T *spout, int L, cudaStream_t s) {
    size_t w_off, r_off, W_off;
    const size_t need = static_need<T>(p, L, &w_off, &r_off, &W_off);
    if (need > (size_t)EXOTX_STATIC_WORK_BYTES) return EXOTX_BAD_DIM;
    if (!exotx_fft_supported(p->nlon)) return EXOTX_UNSUPPORTED_N;
    unsigned char *base;
    EXOTX_TRY(static_work_addr(&base));
    T *dw = reinterpret_cast<T *>(base + w_off), *dr = reinterpret_cast<T *>(base + r_off);
    T *W = reinterpret_cast<T *>(base + W_off);
    const int h = p->nlon / 2;
    {
        // rewrite the twiddles only when the array holds another length's or
        // precision's; the pageable source is staged before cudaMemcpyAsync
        // returns, so the host buffer may be refilled by the next call
        int dev = -1;
        EXOTX_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (g_tw_nlon[dev] != p->nlon || g_tw_esz[dev] != (int)sizeof(T)) {
            T *hw = tw_host<T>(), *hr = hw + 2 * h;
            fft_twiddles_host<T>(p->nlon, hw, hr);
            g_tw_nlon[dev] = 0;  // unknown contents if a copy fails
            EXOTX_CUDA(cudaMemcpyAsync(dw, hw, sizeof(T) * 2 * (size_t)h, cudaMemcpyHostToDevice, s));
            EXOTX_CUDA(cudaMemcpyAsync(dr, hr, sizeof(T) * 2 * (size_t)(h + 1), cudaMemcpyHostToDevice, s));
            g_tw_nlon[dev] = p->nlon;
            g_tw_esz[dev] = (int)sizeof(T);
        }
    }
    const long long nrsp = 2LL * p->ncsp;
    const long long nrows = (9LL * L + 1) * p->nlat;
    EXOTX_TRY(fft_forward_tw<T>(gpin, W, p->nlon, nrows, p->ntp1, 1, nrows, dw, dr, s));
    const FourierLayout F{p->nlat, 1, nrows, p->ntp1};
    auto fld = [&](long long f) -> const T * { return W + 2 * f * p->nlat; };
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

}  // namespace exotx

using namespace exotx;

EXOTX_API exotx_status exotx_forward_set_noalloc(exotx_plan p, int prec, const void *gpin, void *spout, int nlev,
                                                 exotx_stream s) {
    if (!p || !gpin || !spout || nlev < 1) return EXOTX_BAD_ARG;
    if (prec == EXOTX_FP64)
        return forward_set_static<double>(p, (const double *)gpin, (double *)spout, nlev, (cudaStream_t)s);
    if (prec == EXOTX_FP32)
        return forward_set_static<float>(p, (const float *)gpin, (float *)spout, nlev, (cudaStream_t)s);
    return EXOTX_BAD_ARG;  // the mixed path builds its tensor-core tables on first use
}
