// FP64 instantiation of the 3-D fused kernel (placeholder until built).
#include "fxb_launch.h"
namespace fxb {
cudaError_t setup_hydro3d_fp64() { return cudaErrorNotSupported; }
void launch_hydro3d_fp64(const Args3D &, cudaStream_t) {}
} // namespace fxb
