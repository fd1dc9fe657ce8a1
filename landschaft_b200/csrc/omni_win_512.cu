// omni_win_512.cu -- the window kernels with 512 threads per CTA.
#include "omni_windows.cuh"

namespace lsb {
KernelFn pick_windows_512(bool four, bool dbl, bool mg) { return pick_windows_nt<512>(four, dbl, mg); }
}  // namespace lsb
