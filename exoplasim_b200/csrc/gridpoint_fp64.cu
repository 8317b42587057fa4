// FP64 instance of the grid-point step (plasim.f90:2441-2455), compiled with
// -fmad=false: every product and sum rounds separately, in the reference's order.
#include "gridpoint_kernel.cuh"

namespace exotx {
exotx_status launch_gridpoint_fp64(const GpArgs<double> &A, cudaStream_t s) { return gp_launch<double>(A, s); }
}  // namespace exotx
