// pencil.cu -- host dispatch of the line-pass RHS (pencil_impl.cuh).
#include "pencil_impl.cuh"

namespace ws {

int pencil_default_warps(int precision) { return precision == WS_MIXED ? 16 : 8; }

// krk 0: plain RHS into a.du; krk 1..3: into a.du, then the stage update.
// add_x: a.du already holds terms to add to (the viscous terms).
int launch_rhs_pencil(const RhsArgs& a, int precision, bool uniform, int wpb, int krk,
                      bool add_x, cudaStream_t st) {
    if (wpb <= 0) wpb = pencil_default_warps(precision);
    if (precision == WS_MIXED) {
        if (wpb != 16) return fail(WS_ERR_UNSUPPORTED, "line passes: 16 warps per CTA (mixed)");
        if (krk) return PencilLauncher<16, float, true>::stage(a, add_x, krk, st);
        return uniform ? PencilLauncher<16, float, true>::rhs(a, add_x, st)
                       : PencilLauncher<16, float, false>::rhs(a, add_x, st);
    }
    if (wpb != 8) return fail(WS_ERR_UNSUPPORTED, "line passes: 8 warps per CTA (FP64)");
    if (krk) return PencilLauncher<8, double, true>::stage(a, add_x, krk, st);
    return uniform ? PencilLauncher<8, double, true>::rhs(a, add_x, st)
                   : PencilLauncher<8, double, false>::rhs(a, add_x, st);
}

}  // namespace ws
