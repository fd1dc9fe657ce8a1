// omni_win_512_hot.cu -- the window kernels with 512 threads per CTA, all solver arrays in shared memory.
#include "omni_windows.cuh"

namespace lsb {
KernelFn pick_windows_512_hot(bool four, bool dbl, bool mg) { return pick_windows_nt<512, true>(four, dbl, mg); }
}  // namespace lsb
