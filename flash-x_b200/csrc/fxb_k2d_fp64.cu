// FP64 instantiation of the 2-D fused kernel (built with -fmad=false).
#include "fxb_launch.h"
namespace fxb {
cudaError_t setup_hydro2d_fp64()
{
    cudaError_t e = cudaFuncSetAttribute(hydro2d_kernel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem2d_bytes<double>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(hydro2d_kernel<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem2d_bytes<double>());
}
void launch_hydro2d_fp64(const Args2D &a, dim3 grid, cudaStream_t s)
{
    if (a.prm.flattening) flat2d_kernel<double><<<148 * 8, 256, 0, s>>>(a, (double *)a.flat);
    if (extended_options(a.prm) || a.prm.use_gravity)   // Roe, contact steepening, MUSCL-Hancock, 2-D gravity: their own instantiation
        hydro2d_kernel<double, true><<<grid, Threads2D<double>::value, smem2d_bytes<double>(), s>>>(a);
    else
        hydro2d_kernel<double, false><<<grid, Threads2D<double>::value, smem2d_bytes<double>(), s>>>(a);
}
} // namespace fxb
