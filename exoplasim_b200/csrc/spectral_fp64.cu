// FP64 instance of the spectral time step (plasim.f90 spectrala/spectrald),
// compiled with -fmad=false: every product and sum rounds separately, in the
// reference's order.
#include "spectral_kernel.cuh"

namespace exotx {
exotx_status launch_spectral_fp64(const SpecBatch<double> &P, int n, bool d_part, cudaStream_t s) {
    return spec_launch<double>(P, n, d_part, s);
}
}  // namespace exotx
