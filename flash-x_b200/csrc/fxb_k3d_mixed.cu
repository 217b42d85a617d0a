// Mixed-precision instantiation of the 3-D fused kernel (placeholder until built).
#include "fxb_launch.h"
namespace fxb {
cudaError_t setup_hydro3d_mixed() { return cudaErrorNotSupported; }
void launch_hydro3d_mixed(const Args3D &, cudaStream_t) {}
} // namespace fxb
