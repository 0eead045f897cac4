// bf3w_rhs_f32_clo.cu -- instantiates the mixed-precision kernels with the CLOSURE face variant.
#include "bf3w_rhs_impl.cuh"

namespace ws {
template struct RhsSlice<float, true>;
}  // namespace ws
