// omni_win_256_hot.cu -- the window kernels with 256 threads per CTA, all solver arrays in shared memory.
#include "omni_windows.cuh"

namespace lsb {
KernelFn pick_windows_256_hot(bool four, bool dbl, bool mg) { return pick_windows_nt<256, true>(four, dbl, mg); }
}  // namespace lsb
