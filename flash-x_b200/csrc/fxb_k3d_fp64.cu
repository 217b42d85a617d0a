// FP64 instantiation of the 3-D kernels (built with -fmad=false).
#include "fxb_launch.h"
namespace fxb {
cudaError_t setup_hydro3d_fp64() { return cudaSuccess; }
void launch_hydro3d_fp64(const Args3D &a, cudaStream_t s) { launch_hydro3d_t<double>(a, s); }
} // namespace fxb
