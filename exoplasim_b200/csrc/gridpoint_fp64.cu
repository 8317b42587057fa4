// FP64 instance of the grid-point step (plasim.f90:2441-2455), compiled with
// -fmad=false: every product and sum rounds separately, in the reference's order.
#include "gridpoint_kernel.cuh"

namespace exotx {
exotx_status launch_gridpoint_fp64(const GpArgs<double> &A, cudaStream_t s) {
    const size_t smem = 3 * (size_t)A.L * GP_THREADS * sizeof(double);
    if (smem > 48 * 1024)
        EXOTX_CUDA(cudaFuncSetAttribute(k_gridpoint<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long nb = (A.ncol + GP_THREADS - 1) / GP_THREADS;
    k_gridpoint<double><<<(unsigned)nb, GP_THREADS, smem, s>>>(A);
    EXOTX_CHECK_LAUNCH();
    return EXOTX_OK;
}
}  // namespace exotx
