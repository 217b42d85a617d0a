// Mixed-precision instantiation of the 2-D fused kernel: FP32 reconstruction,
// characteristic projection and Riemann solve; FP64 conserved update,
// internal-energy recovery, Eos and CFL rate.
#include "fxb_launch.h"
namespace fxb {
cudaError_t setup_hydro2d_mixed()
{
    cudaError_t e = cudaFuncSetAttribute(hydro2d_kernel<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem2d_bytes<float>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(hydro2d_kernel<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem2d_bytes<float>());
}
void launch_hydro2d_mixed(const Args2D &a, dim3 grid, cudaStream_t s)
{
    if (a.prm.flattening) flat2d_kernel<float><<<148 * 8, 256, 0, s>>>(a, (float *)a.flat);
    if (extended_options(a.prm) || a.prm.use_gravity)   // Roe, contact steepening, MUSCL-Hancock, 2-D gravity: their own instantiation
        hydro2d_kernel<float, true><<<grid, Threads2D<float>::value, smem2d_bytes<float>(), s>>>(a);
    else
        hydro2d_kernel<float, false><<<grid, Threads2D<float>::value, smem2d_bytes<float>(), s>>>(a);
}
} // namespace fxb
