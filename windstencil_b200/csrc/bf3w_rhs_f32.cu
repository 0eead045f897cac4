// bf3w_rhs_f32.cu -- instantiates the mixed-precision kernels (plain sweep only).
#include "bf3w_rhs_impl.cuh"

namespace ws {
template struct RhsSlice<float, false>;
}  // namespace ws
