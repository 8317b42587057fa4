// Tensor-core (tcgen05) Legendre transforms with 3-term BF16 splits.
#include "exotx_internal.cuh"

namespace exotx {

exotx_status tc_available() { return EXOTX_NOT_BUILT; }
void tc_free(exotx_plan) {}
exotx_status tc_inverse_set(exotx_plan, const float *, float *, int, cudaStream_t) { return EXOTX_NOT_BUILT; }
exotx_status tc_forward_set(exotx_plan, const float *, float *, int, cudaStream_t) { return EXOTX_NOT_BUILT; }

}  // namespace exotx
