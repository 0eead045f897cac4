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
    // FP64: 8 warps per CTA (measured: 10 warps, at 148-151 registers, 3% slower)
    if (wpb != 8) return fail(WS_ERR_UNSUPPORTED, "line passes: 8 warps per CTA (FP64)");
    if (krk) return PencilLauncher<8, double, true>::stage(a, add_x, krk, st);
    return uniform ? PencilLauncher<8, double, true>::rhs(a, add_x, st)
                   : PencilLauncher<8, double, false>::rhs(a, add_x, st);
}

// the batched form over the argument table g of n Cartesian grids (woff: the
// x, y, z passes' work prefix tables, n + 1 entries each; clo: some grid has
// a CLOSURE face)
int launch_rhs_pencil_batch(const RhsArgs* g, const long* woff, int n, int precision, int krk,
                            bool clo, cudaStream_t st) {
    if (precision == WS_MIXED)
        return PencilLauncher<12, float, true>::batch(g, woff, n, krk, clo, st);
    return PencilLauncher<8, double, true>::batch(g, woff, n, krk, clo, st);
}

// work of pass dir over the interior of grid g: line groups x march length
long pencil_pass_work(const ws_grid& g, int dir) {
    const long nx = g.nx, ny = g.ny, nz = g.nz;
    const long nl = dir == 0 ? ny * nz : (dir == 1 ? nx * nz : nx * ny);
    const long L = dir == 0 ? nx : (dir == 1 ? ny : nz);
    return (nl + 31) / 32 * L;
}

}  // namespace ws
