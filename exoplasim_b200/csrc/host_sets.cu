// Transform sets of many instances whose arrays live in host memory.
//
// A host model (the Fortran gridpointa, plasim.f90:2396-2486, or a driver of
// many planets) keeps its spectral and grid-point arrays in host memory.  Here
// the instances stream through three device slots on three streams: while the
// transforms of group k run, the inputs of group k+1 are copied in and the
// outputs of group k-1 are copied out, so the PCIe link carries data in both
// directions while the GPU computes.  Within a group the inverse half goes
// first: its spectral input is small and its grid output large, so the grid
// output of the inverse set leaves while the forward set's grid input is still
// arriving.  Every slot is reused only after the copy-out of its previous group
// has finished (events order the streams).
#include <algorithm>
#include "exotx_internal.cuh"

namespace exotx {

struct HostPipe {
    static constexpr int NSLOT = 3;
    int prec = -1, nlev = 0, group = 0, conv = 0;
    void *d_spin[NSLOT] = {}, *d_gout[NSLOT] = {}, *d_gin[NSLOT] = {}, *d_sout[NSLOT] = {};
    // FP64 staging of the host arrays when the transforms run in FP32 (conv)
    void *x_spin[NSLOT] = {}, *x_gout[NSLOT] = {}, *x_gin[NSLOT] = {}, *x_sout[NSLOT] = {};
    cudaStream_t s_in = nullptr, s_run = nullptr, s_out = nullptr;
    // per slot: inverse inputs in, forward inputs in, inverse done, forward done, outputs out
    cudaEvent_t ev_in[NSLOT] = {}, ev_in2[NSLOT] = {}, ev_run[NSLOT] = {}, ev_run2[NSLOT] = {}, ev_out[NSLOT] = {};
    cudaEvent_t ev_edge = nullptr;

    void free_buffers() {
        for (int i = 0; i < NSLOT; i++) {
            cudaFree(d_spin[i]); cudaFree(d_gout[i]); cudaFree(d_gin[i]); cudaFree(d_sout[i]);
            cudaFree(x_spin[i]); cudaFree(x_gout[i]); cudaFree(x_gin[i]); cudaFree(x_sout[i]);
            d_spin[i] = d_gout[i] = d_gin[i] = d_sout[i] = nullptr;
            x_spin[i] = x_gout[i] = x_gin[i] = x_sout[i] = nullptr;
        }
        prec = -1; nlev = 0; group = 0; conv = 0;
    }
    ~HostPipe() {
        if (s_in) cudaStreamSynchronize(s_in);
        if (s_run) cudaStreamSynchronize(s_run);
        if (s_out) cudaStreamSynchronize(s_out);
        free_buffers();
        for (int i = 0; i < NSLOT; i++) {
            if (ev_in[i]) cudaEventDestroy(ev_in[i]);
            if (ev_in2[i]) cudaEventDestroy(ev_in2[i]);
            if (ev_run[i]) cudaEventDestroy(ev_run[i]);
            if (ev_run2[i]) cudaEventDestroy(ev_run2[i]);
            if (ev_out[i]) cudaEventDestroy(ev_out[i]);
        }
        if (ev_edge) cudaEventDestroy(ev_edge);
        if (s_in) cudaStreamDestroy(s_in);
        if (s_run) cudaStreamDestroy(s_run);
        if (s_out) cudaStreamDestroy(s_out);
    }
};

void host_pipe_free(exotx_plan p) {
    delete p->hpipe;
    p->hpipe = nullptr;
}

// bytes of one instance's arrays: spectral in/out, grid out (6L+3 fields), grid in (9L+1)
static void inst_bytes(exotx_plan p, int prec, int L, size_t *sp, size_t *go, size_t *gi) {
    const size_t esz = prec == EXOTX_FP64 ? 8 : 4;
    const size_t nhor = (size_t)p->nlat * p->nlon;
    *sp = (size_t)(4 * L + 1) * 2 * p->ncsp * esz;
    *go = (size_t)(6 * L + 3) * nhor * esz;
    *gi = (size_t)(9 * L + 1) * nhor * esz;
}

static exotx_status pipe_setup(exotx_plan p, int prec, int L, int ninst, int conv, HostPipe **out) {
    if (!p->hpipe) p->hpipe = new HostPipe();
    HostPipe *h = p->hpipe;
    if (!h->s_in) {
        EXOTX_CUDA(cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking));
        EXOTX_CUDA(cudaStreamCreateWithFlags(&h->s_run, cudaStreamNonBlocking));
        EXOTX_CUDA(cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking));
        for (int i = 0; i < HostPipe::NSLOT; i++) {
            EXOTX_CUDA(cudaEventCreateWithFlags(&h->ev_in[i], cudaEventDisableTiming));
            EXOTX_CUDA(cudaEventCreateWithFlags(&h->ev_in2[i], cudaEventDisableTiming));
            EXOTX_CUDA(cudaEventCreateWithFlags(&h->ev_run[i], cudaEventDisableTiming));
            EXOTX_CUDA(cudaEventCreateWithFlags(&h->ev_run2[i], cudaEventDisableTiming));
            EXOTX_CUDA(cudaEventCreateWithFlags(&h->ev_out[i], cudaEventDisableTiming));
        }
        EXOTX_CUDA(cudaEventCreateWithFlags(&h->ev_edge, cudaEventDisableTiming));
    }
    size_t sp, go, gi;
    inst_bytes(p, prec, L, &sp, &go, &gi);
    // instances per slot: about 128 MB of arrays, so the transform launches
    // still cover several instances at small resolutions while the first
    // copy in and the last copy out (which nothing overlaps) stay short
    const size_t per = 2 * sp + go + gi;
    int g = (int)std::max<size_t>(1, (128u << 20) / per);
    g = std::min(g, std::max(ninst, 1));
    if (h->prec != prec || h->nlev != L || h->group < g || h->conv != conv) {
        EXOTX_CUDA(cudaStreamSynchronize(h->s_in));
        EXOTX_CUDA(cudaStreamSynchronize(h->s_run));
        EXOTX_CUDA(cudaStreamSynchronize(h->s_out));
        h->free_buffers();
        for (int i = 0; i < HostPipe::NSLOT; i++) {
            EXOTX_CUDA(cudaMalloc(&h->d_spin[i], sp * g));
            EXOTX_CUDA(cudaMalloc(&h->d_sout[i], sp * g));
            EXOTX_CUDA(cudaMalloc(&h->d_gout[i], go * g));
            EXOTX_CUDA(cudaMalloc(&h->d_gin[i], gi * g));
            if (conv) {  // FP64 twins of the FP32 slots
                EXOTX_CUDA(cudaMalloc(&h->x_spin[i], 2 * sp * g));
                EXOTX_CUDA(cudaMalloc(&h->x_sout[i], 2 * sp * g));
                EXOTX_CUDA(cudaMalloc(&h->x_gout[i], 2 * go * g));
                EXOTX_CUDA(cudaMalloc(&h->x_gin[i], 2 * gi * g));
            }
        }
        h->prec = prec; h->nlev = L; h->group = g; h->conv = conv;
    }
    *out = h;
    return EXOTX_OK;
}

// host arrays of host_esz bytes per real; the transforms run in prec and,
// when its element size differs (FP64 host arrays, FP32 or mixed transforms),
// the slots' FP64 twins take the copies and a conversion kernel on the run
// stream moves the data between the two
static exotx_status sets_host(exotx_plan p, int prec, size_t host_esz, const void *h_spin, void *h_gpout,
                              const void *h_gpin, void *h_spout, int nlev, int ninst, cudaStream_t cs) {
    if (!p || (prec != EXOTX_FP64 && prec != EXOTX_FP32 && prec != EXOTX_MIXED)) return EXOTX_BAD_ARG;
    if (nlev < 1 || ninst < 0) return EXOTX_BAD_ARG;
    const bool inv = h_spin || h_gpout, fwd = h_gpin || h_spout;
    if ((inv && !(h_spin && h_gpout)) || (fwd && !(h_gpin && h_spout)) || !(inv || fwd)) return EXOTX_BAD_ARG;
    if (ninst == 0) return EXOTX_OK;
    const size_t esz = prec == EXOTX_FP64 ? 8 : 4;
    const int conv = host_esz != esz;
    HostPipe *h;
    EXOTX_TRY(pipe_setup(p, prec, nlev, ninst, conv, &h));
    size_t sp, go, gi;
    inst_bytes(p, prec, nlev, &sp, &go, &gi);
    // host-side bytes per instance
    const size_t hsp = sp / esz * host_esz, hgo = go / esz * host_esz, hgi = gi / esz * host_esz;
    // the pipeline starts after the work already queued on the caller's stream
    EXOTX_CUDA(cudaEventRecord(h->ev_edge, cs));
    EXOTX_CUDA(cudaStreamWaitEvent(h->s_in, h->ev_edge, 0));
    const int g = h->group;
    for (int k = 0, i0 = 0; i0 < ninst; k++, i0 += g) {
        const int ni = std::min(g, ninst - i0), b = k % HostPipe::NSLOT;
        void *c_spin = conv ? h->x_spin[b] : h->d_spin[b], *c_gin = conv ? h->x_gin[b] : h->d_gin[b];
        void *c_gout = conv ? h->x_gout[b] : h->d_gout[b], *c_sout = conv ? h->x_sout[b] : h->d_sout[b];
        // copy in: the slot is free once its previous group's outputs are out
        // (in this call or an earlier one; a never-recorded event is no wait)
        EXOTX_CUDA(cudaStreamWaitEvent(h->s_in, h->ev_out[b], 0));
        if (inv)
            EXOTX_CUDA(cudaMemcpyAsync(c_spin, (const char *)h_spin + hsp * i0, hsp * ni, cudaMemcpyHostToDevice,
                                       h->s_in));
        EXOTX_CUDA(cudaEventRecord(h->ev_in[b], h->s_in));
        if (fwd)
            EXOTX_CUDA(cudaMemcpyAsync(c_gin, (const char *)h_gpin + hgi * i0, hgi * ni, cudaMemcpyHostToDevice,
                                       h->s_in));
        EXOTX_CUDA(cudaEventRecord(h->ev_in2[b], h->s_in));
        // transforms: the inverse set as soon as its spectral input is in
        EXOTX_CUDA(cudaStreamWaitEvent(h->s_run, h->ev_in[b], 0));
        if (inv) {
            if (conv) EXOTX_TRY(convert_reals(c_spin, host_esz, h->d_spin[b], esz, sp / esz * ni, h->s_run));
            EXOTX_TRY(exotx_inverse_set_batch(p, prec, h->d_spin[b], h->d_gout[b], nlev, ni, h->s_run));
            if (conv) EXOTX_TRY(convert_reals(h->d_gout[b], esz, c_gout, host_esz, go / esz * ni, h->s_run));
        }
        EXOTX_CUDA(cudaEventRecord(h->ev_run[b], h->s_run));
        EXOTX_CUDA(cudaStreamWaitEvent(h->s_run, h->ev_in2[b], 0));
        if (fwd) {
            if (conv) EXOTX_TRY(convert_reals(c_gin, host_esz, h->d_gin[b], esz, gi / esz * ni, h->s_run));
            EXOTX_TRY(exotx_forward_set_batch(p, prec, h->d_gin[b], h->d_sout[b], nlev, ni, h->s_run));
            if (conv) EXOTX_TRY(convert_reals(h->d_sout[b], esz, c_sout, host_esz, sp / esz * ni, h->s_run));
        }
        EXOTX_CUDA(cudaEventRecord(h->ev_run2[b], h->s_run));
        // copy out: the inverse set's grid rows while the forward input may still be arriving
        EXOTX_CUDA(cudaStreamWaitEvent(h->s_out, h->ev_run[b], 0));
        if (inv)
            EXOTX_CUDA(cudaMemcpyAsync((char *)h_gpout + hgo * i0, c_gout, hgo * ni, cudaMemcpyDeviceToHost,
                                       h->s_out));
        EXOTX_CUDA(cudaStreamWaitEvent(h->s_out, h->ev_run2[b], 0));
        if (fwd)
            EXOTX_CUDA(cudaMemcpyAsync((char *)h_spout + hsp * i0, c_sout, hsp * ni, cudaMemcpyDeviceToHost,
                                       h->s_out));
        EXOTX_CUDA(cudaEventRecord(h->ev_out[b], h->s_out));
    }
    // the caller's stream continues once every output is in host memory
    EXOTX_CUDA(cudaEventRecord(h->ev_edge, h->s_out));
    EXOTX_CUDA(cudaStreamWaitEvent(cs, h->ev_edge, 0));
    return EXOTX_OK;
}

}  // namespace exotx

using namespace exotx;

EXOTX_API exotx_status exotx_sets_host(exotx_plan p, int prec, const void *h_spin, void *h_gpout, const void *h_gpin,
                                       void *h_spout, int nlev, int ninst, exotx_stream s) {
    return sets_host(p, prec, prec == EXOTX_FP64 ? 8 : 4, h_spin, h_gpout, h_gpin, h_spout, nlev, ninst,
                     (cudaStream_t)s);
}

EXOTX_API exotx_status exotx_sets_host_f64(exotx_plan p, int prec, const double *h_spin, double *h_gpout,
                                           const double *h_gpin, double *h_spout, int nlev, int ninst,
                                           exotx_stream s) {
    return sets_host(p, prec, 8, h_spin, h_gpout, h_gpin, h_spout, nlev, ninst, (cudaStream_t)s);
}
