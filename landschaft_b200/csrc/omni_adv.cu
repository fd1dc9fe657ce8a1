// omni_adv.cu -- the raster kernels of the advanced mode (512 threads per CTA): FP32 CG with FP64 refinement and
// multigrid, or FP64 CG with Jacobi; 4 or 8 neighbours; arrays in shared memory (hot) or placed at run time.
#include "omni_adv.cuh"

namespace lsb {

template <bool HOT>
KernelFn pick_rasters_hot(bool four, bool dbl) {
    if (four) return dbl ? k_rasters<512, double, true, false, false, HOT> : k_rasters<512, float, true, true, true, HOT>;
    return dbl ? k_rasters<512, double, false, false, false, HOT> : k_rasters<512, float, false, true, true, HOT>;
}

KernelFn pick_rasters(bool hot, bool four, bool dbl) {
    return hot ? pick_rasters_hot<true>(four, dbl) : pick_rasters_hot<false>(four, dbl);
}

}  // namespace lsb
