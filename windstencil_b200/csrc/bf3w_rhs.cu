// bf3w_rhs.cu -- host dispatch of the fused BF3W RHS kernels.
//
// The kernels (bf3w_rhs_impl.cuh) are compiled in four slices, one
// translation unit each: FP64 and mixed, each with and without the CLOSURE
// face variant.  A grid without CLOSURE faces runs kernels that hold only
// the plain sweep.
#include "bf3w_rhs_impl.cuh"

namespace ws {

int num_tile_cfgs() { return kNumCfgs; }
TileCfg tile_cfg(int i) { return kCfgs[i]; }
int find_tile_cfg(int bx, int by, int threads) {
    for (int i = 0; i < kNumCfgs; ++i)
        if (kCfgs[i].bx == bx && kCfgs[i].by == by && kCfgs[i].threads == threads) return i;
    return -1;
}

int launch_rhs(const RhsArgs& a, int precision, bool uniform, int cfg, int ctas, int krk,
               cudaStream_t st) {
    const bool clo = a.clo[0] | a.clo[1] | a.clo[2] | a.clo[3];
    if (precision == WS_MIXED)
        return clo ? RhsSlice<float, true>::launch(cfg, a, uniform, ctas, krk, st)
                   : RhsSlice<float, false>::launch(cfg, a, uniform, ctas, krk, st);
    return clo ? RhsSlice<double, true>::launch(cfg, a, uniform, ctas, krk, st)
               : RhsSlice<double, false>::launch(cfg, a, uniform, ctas, krk, st);
}

int launch_rhs_batch(const RhsArgs* grids, const BatchWork& w, int precision, bool uniform,
                     bool closure, int cfg, int ctas, int krk, cudaStream_t st) {
    if (precision == WS_MIXED)
        return closure ? RhsSlice<float, true>::launch_batch(cfg, grids, w, uniform, ctas, krk, st)
                       : RhsSlice<float, false>::launch_batch(cfg, grids, w, uniform, ctas, krk,
                                                              st);
    return closure ? RhsSlice<double, true>::launch_batch(cfg, grids, w, uniform, ctas, krk, st)
                   : RhsSlice<double, false>::launch_batch(cfg, grids, w, uniform, ctas, krk, st);
}

int rhs_max_ctas(int precision, bool uniform, bool closure, int cfg, bool stage) {
    if (precision == WS_MIXED)
        return closure ? RhsSlice<float, true>::max_ctas(cfg, uniform, stage)
                       : RhsSlice<float, false>::max_ctas(cfg, uniform, stage);
    return closure ? RhsSlice<double, true>::max_ctas(cfg, uniform, stage)
                   : RhsSlice<double, false>::max_ctas(cfg, uniform, stage);
}

}  // namespace ws
