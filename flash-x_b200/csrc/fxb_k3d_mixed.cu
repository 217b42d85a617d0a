// Mixed-precision instantiation of the 3-D kernels: FP32 reconstruction, CTU
// terms and Riemann solve with FP32 intermediates; FP64 update, Eos and CFL rate.
#include "fxb_launch.h"
namespace fxb {
cudaError_t setup_hydro3d_mixed() { return cudaSuccess; }
void launch_hydro3d_mixed(const Args3D &a, cudaStream_t s) { launch_hydro3d_t<float>(a, s); }
} // namespace fxb
