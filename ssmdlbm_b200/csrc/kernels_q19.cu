// kernels_q19.cu — D3Q19 + D3Q7 instantiations of the step and init launchers.
#include "host.cuh"

namespace ssmd {
namespace host {
SSMD_INSTANTIATE(19, float)
SSMD_INSTANTIATE(19, __half)
SSMD_INSTANTIATE(19, half_g32)
SSMD_INSTANTIATE(19, __nv_bfloat16)
} // namespace host
} // namespace ssmd
