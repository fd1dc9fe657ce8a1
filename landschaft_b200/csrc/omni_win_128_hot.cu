// omni_win_128_hot.cu -- the window kernels with 128 threads per CTA and four CTAs per SM (small windows whose
// solver arrays fit a quarter of the SM's shared memory).
#include "omni_windows.cuh"

namespace lsb {
KernelFn pick_windows_128_hot(bool four, bool dbl, bool mg) { return pick_windows_nt<128, true>(four, dbl, mg); }
}  // namespace lsb
