// omni_win_512_gen.cu -- the window kernels with 512 threads per CTA, solver arrays placed at run time (large windows).
#include "omni_windows.cuh"

namespace lsb {
KernelFn pick_windows_512_gen(bool four, bool dbl, bool mg) { return pick_windows_nt<512, false>(four, dbl, mg); }
}  // namespace lsb
