// omni_win_256.cu -- the window kernels with 256 threads per CTA.
#include "omni_windows.cuh"

namespace lsb {
KernelFn pick_windows_256(bool four, bool dbl, bool mg) { return pick_windows_nt<256>(four, dbl, mg); }
}  // namespace lsb
