// fxb_amr.h -- block-structured AMR mode of the library (3-D).
//
// fxb_register_blocks switches the library to this mode when the leaf list
// is not the uniform level-1 block grid.  The leaves keep their UNK slots
// (the order of the list); parents are derived and live only on the device.
#pragma once
#include <cuda_runtime.h>
#include "../../include/flashx_b200.h"
#include "fxb_device.cuh"

namespace fxb {

// what the AMR mode shares with the rest of the library
struct AmrCommon {
    cudaStream_t stream;
    fxb_params prm;
    fxb_domain dom;
    DevParams dprm;
    int nunk;
    int dmap[NV_DEV];             // device variable -> UNK slot
    int *err;                     // device error word
    unsigned long long *rate_max; // device CFL rate (bits of a double)
    double *dtv;                  // device [dt, dtOld]
    double gam1inv, ggprodinv;
};

int amr_create(const AmrCommon &c, const fxb_block_desc *leaves, int nleaf);
bool amr_active();
int amr_cur();      // which interior store holds the current state
void amr_destroy();
int amr_attach(const double *unk_host);
int amr_sync_to_host(double *unk_host);
// Grid_fillGuardCells into the host UNK for some of the variables: pos[v] is
// device variable v's place in the packed cell vector (-1: not copied), n the
// places, slot[q] their UNK slots; Eos on the guard regions next to other
// levels only with do_eos (Paramesh4/Grid_fillGuardCells.F90:531-548)
int amr_fill_to_host(double *unk_host, const int pos[NV_DEV], int n, const int slot[NV_DEV], bool do_eos);
// one Hydro() step enqueued on the stream; dt from dtv when dtv != nullptr
int amr_step(const double *dtv, double dt, int *launches);
int amr_rate();
int amr_eos();
// the registered mesh replaced by the leaf list `leaves` (one level of change
// per block), its data moved on the device: copies, restriction, prolongation, Eos
int amr_regrid(const fxb_block_desc *leaves, int nleaf);
int amr_integrals(double *out7, double *partials, int npartials);
long amr_leaf_cells();
// first leaf cell (leaf, k, j, i linear index) whose CFL rate equals the reduced maximum
int amr_locate(unsigned long long *key);
int amr_leaf_level(int leaf);
// a rank's share of a split mesh: per leaf 1 owned, 2 flux ghost, 0 not stepped (NULL: all owned)
int amr_set_roles(const unsigned char *roles, int nleaf);
long amr_leaf_doubles();
// leaves of the host UNK: every leaf, or with roles set the own leaves in leaf order
int amr_host_leaves();
int amr_copy_leaves(const int *leaves, int n, double *buf, bool pack);
// Grid_markRefineDerefine on the leaves; dvar: device variables, need_eos:
// the variable is an Eos output (the guard regions get the Eos)
int amr_mark_refine(int nvars, const int *dvar, const int *need_eos, const double *refine_cutoff,
                    const double *derefine_cutoff, const double *refine_filter, int max_refine, int *flags,
                    double *error_out);
// the launch shape chosen at the last attach, as text
const char *amr_tuning_log();

// reports through fxb_last_error (defined in fxb_api.cu)
int record_error(int code, const char *msg);
// packed cell vectors (ncell x n doubles in device memory) into their UNK
// slots slot[q] of unk_host (ncell cells of nunk doubles), through a pinned
// staging copy (defined in fxb_api.cu)
int pack_to_host(const double *pack_dev, long ncell, int n, const int *slot, double *unk_host);

} // namespace fxb
