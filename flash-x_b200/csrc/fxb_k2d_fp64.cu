// FP64 instantiation of the 2-D fused kernel (built with -fmad=false).
#include "fxb_launch.h"
namespace fxb {
cudaError_t setup_hydro2d_fp64()
{
    cudaError_t e = cudaFuncSetAttribute(hydro2d_kernel<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem2d_bytes<double>());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(hydro2d_kernel<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem2d_bytes<double>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(hydro2d_kernel<double, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem2d_bytes<double>());
}
void launch_hydro2d_fp64(const Args2D &a, dim3 grid, cudaStream_t s)
{
    if (a.prm.flattening) flat2d_kernel<double><<<148 * 8, 256, 0, s>>>(a, (double *)a.flat);
    if (marquina_solver(a.prm))                          // Marquina solvers (with any other option)
        hydro2d_kernel<double, 2><<<grid, Threads2D<double>::value, smem2d_bytes<double>(), s>>>(a);
    else if (extended_options(a.prm) || a.prm.use_gravity)   // Roe, contact steepening, MUSCL-Hancock, 2-D gravity: their own instantiation
        hydro2d_kernel<double, 1><<<grid, Threads2D<double>::value, smem2d_bytes<double>(), s>>>(a);
    else
        hydro2d_kernel<double, 0><<<grid, Threads2D<double>::value, smem2d_bytes<double>(), s>>>(a);
}
} // namespace fxb
