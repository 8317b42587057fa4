// Per-kernel device timing (diagnostics): while enabled, launches of the
// library's main kernels outside stream capture are bracketed by CUDA events
// on the launching stream.
#include <mutex>
#include <utility>
#include <vector>
#include "exotx_internal.cuh"

namespace exotx {

static std::mutex g_kt_mu;
static bool g_kt_on = false;
static std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_kt_rec[EXOTX_K_COUNT];

static bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) return true;
    return st != cudaStreamCaptureStatusNone;
}

cudaEvent_t ktimer_start(int k, cudaStream_t s) {
    {
        std::lock_guard<std::mutex> lk(g_kt_mu);
        if (!g_kt_on || k < 0 || k >= EXOTX_K_COUNT) return nullptr;
    }
    if (capturing(s)) return nullptr;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    if (cudaEventRecord(e, s) != cudaSuccess) { cudaEventDestroy(e); return nullptr; }
    return e;
}

void ktimer_stop(int k, cudaStream_t s, cudaEvent_t e0) {
    if (!e0) return;
    cudaEvent_t e1 = nullptr;
    if (cudaEventCreate(&e1) != cudaSuccess || cudaEventRecord(e1, s) != cudaSuccess) {
        cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        return;
    }
    std::lock_guard<std::mutex> lk(g_kt_mu);
    g_kt_rec[k].emplace_back(e0, e1);
}

static void clear_locked(int k) {
    for (auto &pr : g_kt_rec[k]) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    g_kt_rec[k].clear();
}

}  // namespace exotx

using namespace exotx;

EXOTX_API exotx_status exotx_kernel_timing(int enable) {
    std::lock_guard<std::mutex> lk(g_kt_mu);
    g_kt_on = enable != 0;
    if (!g_kt_on)
        for (int k = 0; k < EXOTX_K_COUNT; k++) clear_locked(k);
    return EXOTX_OK;
}

EXOTX_API exotx_status exotx_kernel_time(int kernel, double *ms, long long *launches) {
    if (kernel < 0 || kernel >= EXOTX_K_COUNT || !ms || !launches) return EXOTX_BAD_ARG;
    std::lock_guard<std::mutex> lk(g_kt_mu);
    double tot = 0.0;
    for (auto &pr : g_kt_rec[kernel]) {
        EXOTX_CUDA(cudaEventSynchronize(pr.second));
        float t = 0.f;
        EXOTX_CUDA(cudaEventElapsedTime(&t, pr.first, pr.second));
        tot += t;
    }
    *ms = tot;
    *launches = (long long)g_kt_rec[kernel].size();
    clear_locked(kernel);
    return EXOTX_OK;
}
