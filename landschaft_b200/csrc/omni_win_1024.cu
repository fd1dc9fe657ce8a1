// omni_win_1024.cu -- the window kernels with 1024 threads per CTA.
#include "omni_windows.cuh"

namespace lsb {
KernelFn pick_windows_1024(bool four, bool dbl, bool mg) { return pick_windows_nt<1024>(four, dbl, mg); }
}  // namespace lsb
