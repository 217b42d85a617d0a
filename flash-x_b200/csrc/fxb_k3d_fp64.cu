// FP64 instantiation of the 3-D kernels (built with -fmad=false).
#include "fxb_launch.h"
#include "fxb_amr_persist.cuh"
#include "fxb_species.cuh"
namespace fxb {
void launch_gravity_faces_fp64(const DevParams &p, void *out, cudaStream_t s)
{ gravity_faces_kernel<double><<<1, 1, 0, s>>>(p, (double *)out); }
cudaError_t setup_hydro3d_fp64() { return cudaSuccess; }
void launch_hydro3d_fp64(const Args3D &a, cudaStream_t s) { launch_hydro3d_t<double>(a, s); }
void launch_amr3d_fluxes_fp64(const Args3D &a, int entries, int which, cudaStream_t s)
{ launch_amr3d_fluxes_t<double>(a, entries, which, s); }
void launch_amr3d_emit_fp64(const Args3D &a, int entries, void *bflux, long nfc, cudaStream_t s)
{ launch_amr3d_emit_t<double>(a, entries, bflux, nfc, s); }
void launch_amr3d_correct_fp64(const Args3D &a, int entries, const void *bflux, long nfc, const int *fine,
                               const int *finer_mask, cudaStream_t s)
{ launch_amr3d_correct_t<double>(a, entries, bflux, nfc, fine, finer_mask, s); }
void launch_amr3d_update_fp64(const Args3D &a, int entries, cudaStream_t s) { launch_amr3d_update_t<double>(a, entries, s); }
cudaError_t launch_amr_persist_fp64(int which, int clusters, int K, cudaStream_t s)
{ return launch_amr_persist_t<double>(which, clusters, K, s); }
cudaError_t persist_upload_fp64(const PersistArgs p[2]) { return persist_upload_t<double>(p); }
int persist_grid_fp64(int K) { return persist_grid<double>(K); }
void launch_species_fp64(const SpecArgs &a, cudaStream_t s) { launch_species_t<double>(a, s); }
} // namespace fxb
