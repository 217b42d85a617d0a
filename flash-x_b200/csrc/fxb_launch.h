// fxb_launch.h -- launchers of the fused hydro kernels.  Each precision lives
// in its own translation unit so that the FP64 path can be compiled with
// -fmad=false (every product and sum rounded as written, matching the
// oracle bit for bit) while the mixed path keeps fused multiply-adds.
#pragma once
#include <cuda_runtime.h>
#include "fxb_hydro2d.cuh"
#include "fxb_hydro3d.cuh"

namespace fxb {
cudaError_t setup_hydro2d_fp64();
cudaError_t setup_hydro2d_mixed();
void launch_hydro2d_fp64(const Args2D &a, dim3 grid, cudaStream_t s);
void launch_hydro2d_mixed(const Args2D &a, dim3 grid, cudaStream_t s);
cudaError_t setup_hydro3d_fp64();
// gravity_faces of the three directions into out[6] (double, float)
void launch_gravity_faces_fp64(const DevParams &p, void *out, cudaStream_t s);
void launch_gravity_faces_mixed(const DevParams &p, void *out, cudaStream_t s);
cudaError_t setup_hydro3d_mixed();
void launch_hydro3d_fp64(const Args3D &a, cudaStream_t s);
void launch_hydro3d_mixed(const Args3D &a, cudaStream_t s);
void launch_amr3d_fluxes_fp64(const Args3D &a, int entries, int which, cudaStream_t s);
void launch_amr3d_emit_fp64(const Args3D &a, int entries, void *bflux, long nfc, cudaStream_t s);
void launch_amr3d_correct_fp64(const Args3D &a, int entries, const void *bflux, long nfc, const int *fine,
                               const int *finer_mask, cudaStream_t s);
void launch_amr3d_update_fp64(const Args3D &a, int entries, cudaStream_t s);
void launch_amr3d_fluxes_mixed(const Args3D &a, int entries, int which, cudaStream_t s);
void launch_amr3d_emit_mixed(const Args3D &a, int entries, void *bflux, long nfc, cudaStream_t s);
void launch_amr3d_correct_mixed(const Args3D &a, int entries, const void *bflux, long nfc, const int *fine,
                               const int *finer_mask, cudaStream_t s);
void launch_amr3d_update_mixed(const Args3D &a, int entries, cudaStream_t s);
// species and mass scalars after a uniform-grid step (fxb_species.cuh)
struct SpecArgs;
void launch_species_fp64(const SpecArgs &a, cudaStream_t s);
void launch_species_mixed(const SpecArgs &a, cudaStream_t s);
// the persistent AMR step (fxb_amr_persist.cuh): launch and resident CTAs
struct PersistArgs;
cudaError_t launch_amr_persist_fp64(int which, int clusters, int K, cudaStream_t s);
cudaError_t launch_amr_persist_mixed(int which, int clusters, int K, cudaStream_t s);
cudaError_t persist_upload_fp64(const PersistArgs p[2]);   // argument sets for current store 0 and 1
cudaError_t persist_upload_mixed(const PersistArgs p[2]);
int persist_grid_fp64(int K);    // clusters of K CTAs that fit at once
int persist_grid_mixed(int K);
} // namespace fxb
