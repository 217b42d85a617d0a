// Mixed-precision instantiation of the 3-D kernels: FP32 reconstruction, CTU
// terms and Riemann solve with FP32 intermediates; FP64 update, Eos and CFL rate.
#include "fxb_launch.h"
#include "fxb_amr_persist.cuh"
#include "fxb_species.cuh"
namespace fxb {
void launch_gravity_faces_mixed(const DevParams &p, void *out, cudaStream_t s)
{ gravity_faces_kernel<float><<<1, 1, 0, s>>>(p, (float *)out); }
cudaError_t setup_hydro3d_mixed() { return cudaSuccess; }
void launch_hydro3d_mixed(const Args3D &a, cudaStream_t s) { launch_hydro3d_t<float>(a, s); }
void launch_amr3d_fluxes_mixed(const Args3D &a, int entries, int which, cudaStream_t s)
{ launch_amr3d_fluxes_t<float>(a, entries, which, s); }
void launch_amr3d_emit_mixed(const Args3D &a, int entries, void *bflux, long nfc, cudaStream_t s)
{ launch_amr3d_emit_t<float>(a, entries, bflux, nfc, s); }
void launch_amr3d_correct_mixed(const Args3D &a, int entries, const void *bflux, long nfc, const int *fine,
                               const int *finer_mask, cudaStream_t s)
{ launch_amr3d_correct_t<float>(a, entries, bflux, nfc, fine, finer_mask, s); }
void launch_amr3d_update_mixed(const Args3D &a, int entries, cudaStream_t s) { launch_amr3d_update_t<float>(a, entries, s); }
cudaError_t launch_amr_persist_mixed(int which, int clusters, int K, cudaStream_t s)
{ return launch_amr_persist_t<float>(which, clusters, K, s); }
cudaError_t persist_upload_mixed(const PersistArgs p[2]) { return persist_upload_t<float>(p); }
int persist_grid_mixed(int K) { return persist_grid<float>(K); }
void launch_species_mixed(const SpecArgs &a, cudaStream_t s) { launch_species_t<float>(a, s); }
} // namespace fxb
