// FP64 instance of the spectral time step (plasim.f90 spectrala/spectrald),
// compiled with -fmad=false: every product and sum rounds separately, in the
// reference's order.
#include "spectral_kernel.cuh"

namespace exotx {
static int spec_threads64(int L) {
    int t = 128;
    while (t > 32 && 4 * (size_t)L * t * sizeof(double) > 160 * 1024) t -= 32;
    return t;
}
exotx_status launch_spectral_fp64(const SpecArgs<double> &A, bool d_part, cudaStream_t s) {
    if (d_part) {
        k_spectrald<double><<<(A.nrsp + 127) / 128, 128, 0, s>>>(A);
    } else {
        const int nt = spec_threads64(A.L);
        const size_t smem = 4 * (size_t)A.L * nt * sizeof(double);
        if (smem > 48 * 1024)
            EXOTX_CUDA(cudaFuncSetAttribute(k_spectrala<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_spectrala<double><<<(A.nrsp + nt - 1) / nt, nt, smem, s>>>(A);
    }
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}
}  // namespace exotx
