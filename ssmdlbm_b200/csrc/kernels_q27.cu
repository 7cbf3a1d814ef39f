// kernels_q27.cu — D3Q27 + D3Q7 instantiations of the step and init launchers.
#include "host.cuh"

namespace ssmd {
namespace host {
SSMD_INSTANTIATE(27, float)
SSMD_INSTANTIATE(27, __half)
SSMD_INSTANTIATE(27, half_g32)
SSMD_INSTANTIATE(27, __nv_bfloat16)
} // namespace host
} // namespace ssmd
