// omni_win_256_gen.cu -- the window kernels with 256 threads per CTA, solver arrays placed at run time (large windows).
#include "omni_windows.cuh"

namespace lsb {
KernelFn pick_windows_256_gen(bool four, bool dbl, bool mg) { return pick_windows_nt<256, false>(four, dbl, mg); }
}  // namespace lsb
