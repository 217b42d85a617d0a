// Mixed-precision instantiation of the 2-D fused kernel: FP32 reconstruction,
// characteristic projection and Riemann solve; FP64 conserved update,
// internal-energy recovery, Eos and CFL rate.
#include "fxb_launch.h"
namespace fxb {
cudaError_t setup_hydro2d_mixed()
{
    cudaError_t e = cudaFuncSetAttribute(hydro2d_kernel<float, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem2d_bytes<float>());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(hydro2d_kernel<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem2d_bytes<float>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(hydro2d_kernel<float, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem2d_bytes<float>());
}
void launch_hydro2d_mixed(const Args2D &a, dim3 grid, cudaStream_t s)
{
    if (a.prm.flattening) flat2d_kernel<float><<<148 * 8, 256, 0, s>>>(a, (float *)a.flat);
    if (marquina_solver(a.prm))                          // Marquina solvers (with any other option)
        hydro2d_kernel<float, 2><<<grid, Threads2D<float>::value, smem2d_bytes<float>(), s>>>(a);
    else if (extended_options(a.prm) || a.prm.use_gravity)   // Roe, contact steepening, MUSCL-Hancock, 2-D gravity: their own instantiation
        hydro2d_kernel<float, 1><<<grid, Threads2D<float>::value, smem2d_bytes<float>(), s>>>(a);
    else
        hydro2d_kernel<float, 0><<<grid, Threads2D<float>::value, smem2d_bytes<float>(), s>>>(a);
}
} // namespace fxb
