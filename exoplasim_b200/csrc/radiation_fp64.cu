// FP64 instantiation of the radiation column kernel.  Built with
// -fmad=false: products and sums round separately, in the reference's order.
#include "radiation_kernel.cuh"

namespace exotx {
exotx_status launch_radstep_fp64(const RadDev &D, int blocks, int warps, size_t smem, cudaStream_t st) {
    if (smem > 48 * 1024)
        EXOTX_CUDA(cudaFuncSetAttribute(k_radstep<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaEvent_t ev = ktimer_start(EXOTX_K_RADSTEP, st);
    k_radstep<double><<<blocks, warps * 32, smem, st>>>(D);
    EXOTX_CHECK_LAUNCH();
    ktimer_stop(EXOTX_K_RADSTEP, st, ev);
    return EXOTX_OK;
}
}  // namespace exotx
