// bf3w_rhs_f64.cu -- instantiates the FP64 kernels (plain sweep only).
#include "bf3w_rhs_impl.cuh"

namespace ws {
template struct RhsSlice<double, false>;
}  // namespace ws
