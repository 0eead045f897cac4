// bf3w_rhs_f64_clo.cu -- instantiates the FP64 kernels with the CLOSURE face variant.
#include "bf3w_rhs_impl.cuh"

namespace ws {
template struct RhsSlice<double, true>;
}  // namespace ws
