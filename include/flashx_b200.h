/*
 * flashx_b200.h -- C ABI of libflashx_b200.so, the B200 (sm_100a) drop-in for
 * the Flash-X unsplit compressible-hydro hot path.
 *
 * Plain C types only: the Fortran driver binds these with ISO_C_BINDING,
 * Python with ctypes.  Every function returns an int
 * status: FXB_OK (0) or one of the FXB_E* codes; fxb_last_error() gives the
 * message.  The library never calls exit() or abort().
 *
 * Reference interfaces replaced (paths inside the Flash-X project):
 *   Hydro(simTime, dt, dtOld)                 source/physics/Hydro/Hydro_interface.F90,
 *                                             impl .../HydroMain/unsplit/levelFlux/Hydro.F90:20
 *   Hydro_computeDt(tileDesc, ..., U, dtCheck, dtMinLoc, extraInfo)
 *                                             .../HydroMain/unsplit/Hydro_computeDt.F90:28-34
 *   Grid_fillGuardCells(gridDataStruct, idir, ...)
 *                                             source/Grid/Grid_fillGuardCells.F90:283,
 *                                             impl source/Grid/GridMain/UG/Grid_fillGuardCells.F90
 *   Eos_wrapped(MODE_DENS_EI, range, U)       source/physics/Eos/EosMain/Eos_wrapped.F90:60-189
 *   IO_writeIntegralQuantities sums           source/IO/IOMain/IO_writeIntegralQuantities.F90:60-224
 *
 * Data contract: the caller owns unk(var,i,j,k,blk) in host memory (FP64,
 * Fortran order, NGUARD guard cells per side, var_map giving the 0-based
 * slot of each UHD variable as Simulation.h's *_VAR - 1).  The library
 * keeps a device mirror in its own layout (one FP64 array per variable over
 * the whole uniform grid) and all scratch; steady-state steps never cross
 * PCIe.  Single host thread, not re-entrant; one CUDA stream per library
 * instance.
 */
#ifndef FLASHX_B200_H
#define FLASHX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FXB_OK              0
#define FXB_EARG            1   /* bad argument or call order */
#define FXB_ECUDA           2   /* CUDA runtime error (no device, launch failure, OOM) */
#define FXB_ESOUND          3   /* zero or imaginary sound speed (hy_eigenParameters.F90:94-100) */
#define FXB_ERIEMANN        4   /* Riemann solver ierr (hy_getFaceFlux.F90:337-378) */
#define FXB_EDT             5   /* computed dt not positive (Hydro_computeDt.F90:286-288) */
#define FXB_EUNSUPPORTED    6   /* option combination this path does not implement */
#define FXB_ETIMEOUT        7   /* a bounded device-side wait ran out (TMA window, device-wide barrier) */

/* variables of the UHD + Gamma solution vector, used to index var_map */
enum fxb_var { FXB_DENS = 0, FXB_EINT, FXB_ENER, FXB_GAMC, FXB_GAME, FXB_PRES,
               FXB_TEMP, FXB_VELX, FXB_VELY, FXB_VELZ, FXB_NVAR };

enum fxb_bc { FXB_BC_PERIODIC = 0, FXB_BC_OUTFLOW = 1, FXB_BC_REFLECTING = 2 };
enum fxb_precision { FXB_FP64 = 0, FXB_MIXED = 1 };   /* MIXED: FP32 reconstruction and
                                                          Riemann solve, FP64 update/eint/sums/dt */

/* Resolved runtime parameters (names as in the Flash-X Config files). */
typedef struct fxb_params {
    int    order;              /* 2 = MUSCL-Hancock, 3 = PPM, 5 = WENO               */
    int    weno_method;        /* 1 = WENO5, 2 = WENOZ                               */
    int    riemann;            /* 1 = Roe, 2 = LLF, 3 = HLL, 4 = HLLC, 5 = Marquina,
                                  7 = MarquinaModified, 8 = hybrid (HLL next to a
                                  cell the shock detector marks, HLLC elsewhere;
                                  turns shock_detect on) (UHD.h)                    */
    int    limiter;            /* 1 minmod, 2 mc, 3 vanLeer, 4 hybrid, 5 limited     */
    int    char_limiting;      /* charLimiting                                       */
    int    use_3d_full_ctu;    /* use_3dFullCTU                                      */
    int    use_aux_eint;       /* use_auxEintEqn                                     */
    int    use_gravity;        /* constant gravity (Gravity/GravityMain/Constant)    */
    double grav[3];
    double cfl, gamma, eint_switch, small_dens, small_e, small_p, tiny;
    double fpres;              /* hy_fPresInMomFlux                                  */
    double limited_beta;       /* LimitedSlopeBeta                                   */
    double gas_constant, abar; /* Eos Gamma: ideal gas constant, eos_singleSpeciesA  */
    int    precision;          /* enum fxb_precision                                 */
    int    flattening;         /* use_flattening (not combined with gravity)         */
    int    entropy_fix;        /* Roe: entropy = .false. (0), entropyFixMethod
                                  HartenHyman (1) or Harten (2)                     */
    int    steepening;         /* use_steepening: PPM contact steepening            */
    int    use_avisc;          /* use_avisc: artificial viscosity                    */
    double cvisc;              /* cvisc: its constant (Config default 0.1)           */
    int    upwind_tvd;         /* use_upwindTVD: off when NGUARD <= 4, as
                                  unsplit/Hydro_init.F90:137 resets it; rejected
                                  (FXB_EUNSUPPORTED) with more guard cells        */
    int    hybrid_order;       /* use_hybridOrder                                    */
    double hybrid_kappa;       /* hybridOrderKappa (Config default 0)                */
    int    shock_detect;       /* shockDetect: the SHOK flag of every cell before each
                                  step (hy_shockDetectBlk.F90; uniform grids)       */
    int    shock_slot;         /* 0-based UNK slot of SHOK_VAR that fxb_sync_to_host
                                  and unmasked guard fills write (< 0: none)        */
} fxb_params;

/* Domain of a uniform block grid. */
typedef struct fxb_domain {
    int    ndim;               /* 2 or 3 */
    int    nxb, nyb, nzb;      /* block interior (nzb = 1 in 2-D) */
    int    nguard;             /* NGUARD (4) */
    int    nblockx, nblocky, nblockz;
    double bbox[3][2];         /* xmin xmax, ymin ymax, zmin zmax */
    int    bc[6];              /* xl xr yl yr zl zr, enum fxb_bc */
} fxb_domain;

/* One leaf block: its refinement level (1 = the root block grid of
 * fxb_domain) and its 0-based block coordinates at that level, in
 * [0, nblock * 2^(level-1)) per axis.  Flash-X's blkLimits, deltas and
 * bounding box follow from them (PARAMESH lrefine and the block's position). */
typedef struct fxb_block_desc {
    int    level;
    int    bcoord[3];
} fxb_block_desc;

/* This rank's share of a uniform block grid split over ranks (one GPU each)
 * along its slowest axis (y in 2-D, z in 3-D), as UG's iProcs x jProcs x
 * kProcs layout with a single process axis (Grid_data gr_axisComm): the rank
 * holds block layers [layer_lo, layer_hi) of that axis, every block of each
 * layer, and halo_lo / halo_hi planes of cells below / above them that
 * fxb_halo_unpack fills from the neighbouring ranks.  A halo is 0 on a side
 * that is a physical (non-periodic) boundary of the domain and at least
 * NGUARD, at most the rank's own interior planes, on every other side; in
 * 2-D the interior plus both halos must be a multiple of 16 cells. */
typedef struct fxb_slab {
    int    layer_lo, layer_hi;
    int    halo_lo, halo_hi;
} fxb_slab;

typedef struct fxb_error {
    int    code;
    char   message[256];
} fxb_error;

/* Hydro_init + Grid_init: resolve parameters, select the device, allocate the
 * device mirror.  var_map[FXB_NVAR] gives each variable's 0-based slot in a
 * UNK cell vector of nunk doubles. */
int fxb_init(const fxb_params *params, const fxb_domain *domain,
             const int32_t *var_map, int nunk);
/* fxb_init for one slab of a uniform grid shared by several ranks: `domain`
 * is the whole grid, `slab` this rank's part (NULL: the whole grid, no
 * halos, which is fxb_init).  The rank then registers and attaches only its
 * own blocks, in the order of the whole grid's block list, and calls
 * fxb_halo_pack / fxb_halo_unpack around the exchange with its neighbours
 * before every fxb_hydro_step and before fxb_sync_to_host (the guard cells
 * next to another slab come from the halo).  fxb_compute_dt and
 * fxb_integrals cover the rank's own cells; the caller reduces them over
 * ranks (MIN and SUM).  fxb_advance needs an exchange per step and returns
 * FXB_EUNSUPPORTED on a slab with halos.  Block-structured AMR meshes are
 * not split (FXB_EUNSUPPORTED at fxb_register_blocks). */
int fxb_init_slab(const fxb_params *params, const fxb_domain *domain,
                  const int32_t *var_map, int nunk, const fxb_slab *slab);
/* Species and mass scalars (NSPECIES + NMASS_SCALARS of Simulation.h),
 * advected with every step as hy_fullSpecMsFluxHandling does (unsplit/
 * Config:165): mass fractions reconstructed along each direction and traced
 * with the entropy wave (hy_DataReconstructNormalDir_{PPM,WENO,MH}.F90),
 * upwind transverse and 3-D CTU terms (hy_upwindTransverseFlux.F90,
 * hy_getRiemannState.F90:1063-1100), fluxes = mass flux x upwind value
 * (hy_getFaceFlux.F90:464-477), the conservative update and the species'
 * renormalisation (hy_unsplitUpdate.F90:846-881).  Call after fxb_init and
 * before fxb_attach_unk: unk_slots[nspec] are the 0-based UNK slots of the
 * values (SPECIES_BEGIN - 1 ...), the first nspecies of them species that are
 * renormalised to add up to one, the rest mass scalars.  Uniform grids
 * without halos only (FXB_EUNSUPPORTED on AMR meshes and slabs). */
#define FXB_MAX_SPECIES 32
int fxb_init_species(int nspec, int nspecies, const int32_t *unk_slots);
/* The leaf-block list (Grid_getTileIterator(LEAF)); block b is UNK slot b.
 * All leaves at level 1 covering the root grid: the uniform-grid path.
 * Otherwise (3-D only) a block-structured AMR mesh: the leaves must tile the
 * domain with neighbours, across faces, edges and corners, at most one level
 * apart (PARAMESH proper nesting); parents are derived and kept on the device.
 * Each Hydro() step then restricts the parents, fills guard cells by
 * same-level copy or multilinear prolongation (PARAMESH's default
 * interpolation, conserved form), applies Eos to the guard regions next to
 * other levels and corrects the fluxes on fine/coarse faces
 * (Paramesh4/Grid_fillGuardCells.F90:446-541, levelFlux/Hydro.F90:161-270,
 * levelFlux/Grid_conserveFluxes.F90).  Errors: FXB_EARG for a list that does
 * not tile the domain or is not balanced, FXB_EUNSUPPORTED for 2-D AMR and
 * non-cubic blocks. */
int fxb_register_blocks(const fxb_block_desc *blocks, int nblk);
/* Copy the host UNK (all blocks, guard cells included) into the device mirror. */
int fxb_attach_unk(const double *unk_host);
/* Grid_fillGuardCells(CENTER, ALLDIR, doEos=do_eos, mask=mask_bits): the
 * device mirror has no stored guard cells (the hydro kernel resolves
 * neighbour and boundary cells on load), so this writes the filled guard
 * cells, with the interiors, of the selected variables into unk_host (NULL:
 * the UNK of the last fxb_attach_unk / fxb_sync_from_host).  mask_bits: bit
 * (1 << fxb_var) selects a variable, 0 selects all of them (the call without
 * a mask); only the selected variables cross PCIe and are written, the other
 * UNK entries keep their host values.  do_eos: on AMR meshes, Eos_guardCells
 * on the guard regions next to other refinement levels
 * (Paramesh4/Grid_fillGuardCells.F90:531-548); the uniform grid ignores it,
 * as UG/Grid_fillGuardCells.F90 does.  FXB_EARG for bits outside the fxb_var
 * range. */
int fxb_fill_guardcells(int mask_bits, int do_eos, double *unk_host);
/* Hydro(simTime, dt, dtOld): one unsplit step of every leaf block on the
 * device (guard resolution, reconstruction, Riemann solve, conserved update,
 * energyFix, Eos), followed on the device by the CFL reduction that
 * fxb_compute_dt reports. */
int fxb_hydro_step(double sim_time, double dt, double dt_old);
/* Hydro_computeDt reduced over all blocks (Driver_computeDt's MPI_AllReduce
 * MIN of the per-block dtCheck): the CFL time step of the current state.
 * Driver_computeDt.F90:306 calls Hydro_computeDt once per leaf block: the
 * first call after the state changed (a step, an attach, Eos, a regrid)
 * reduces on the device and synchronises; later calls return the cached
 * result (and the cached location, once one was computed) with no launch and
 * no synchronisation (fxb_counters counts both kinds).
 * loc[5] receives, when loc is not NULL, the limiting cell as
 * Hydro_computeDt.F90:231-235 records it: i, j, k in the block's 1-based
 * guard-inclusive index space and the refinement level; the fifth entry is
 * the 1-based UNK block (the reference keeps its MPI rank there).  Ties go to
 * the first cell in block order, then k, j, i, as the reference's strict '>'
 * scan does.  Locating costs one read of the state. */
int fxb_compute_dt(double *dt_out, int32_t loc[5]);
/* Driver loop on the device: nsteps of Hydro + Driver_computeDt dt control
 * (dtNew = min(dtCFL, tstep_change_factor*dtOld), clamped to [dtmin, dtmax]),
 * captured once as a CUDA graph.  *dt and *dt_old are read and updated. */
int fxb_advance(int nsteps, double *dt, double *dt_old, double tstep_change_factor,
                double dtmin, double dtmax);
/* Eos_wrapped(MODE_DENS_EI) on all block interiors of the device mirror. */
int fxb_eos(void);
/* Copy the device mirror back into unk_host (interiors and guard cells). */
int fxb_sync_to_host(double *unk_host);
/* Re-read unk_host after a host-side write (init, restart, regrid). */
int fxb_sync_from_host(const double *unk_host);
/* Interior transfers, for drivers whose host units read or write UNK
 * between hydro steps.  Hydro fills the guard cells from the interiors
 * before it reconstructs (levelFlux/Hydro.F90:161) and hy_unsplitUpdate
 * writes only the cells inside blkLimits (hy_unsplitUpdate.F90:84-131), so a
 * step depends on, and changes, block interiors only.  fxb_put_interior
 * replaces the interiors of the device state with unk_host's (the ten hydro
 * variables dens, velx, vely, velz, pres, gamc, game, eint, ener, temp and
 * the advected mass fractions of fxb_init_species); fxb_get_interior writes
 * the current interiors of the same variables, and SHOK when the shock
 * detector ran, into unk_host and leaves its guard cells as they are.  Both
 * move whole interior rows (nxb cells x nunk slots, contiguous in UNK) with
 * strided copies on the copy engine, so the other slots of interior cells
 * receive the values last read from the host (fxb_attach_unk,
 * fxb_sync_from_host or fxb_put_interior): the caller changes them after
 * fxb_get_interior, not between a put and the next get.  The first call
 * page-locks unk_host (unless it already is); there is no host-side copy.
 * unk_host stays locked until fxb_finalize or a call with another UNK and
 * must stay allocated until then.  fxb_put_interior needs a prior
 * fxb_attach_unk (FXB_EARG otherwise).  AMR meshes move whole blocks, as
 * fxb_sync_from_host and fxb_sync_to_host do. */
int fxb_put_interior(const double *unk_host);
int fxb_get_interior(double *unk_host);
/* Volume integrals: mass, x/y/z momentum, total, internal, kinetic energy. */
int fxb_integrals(double out[7]);
/* Guard-cell exchange between slabs (UG/Grid_fillGuardCells.F90:261-306 and
 * UG/gr_shiftData.F90:63-191, which MPI_SendRecv the guard layers of each
 * axis to the neighbours).  A message holds `planes` whole planes of the
 * slab's cells for each of the 10 device variables (dens, velx, vely, velz,
 * pres, gamc, game, eint, ener, temp), variable-major: fxb_halo_doubles
 * gives its length.  fxb_halo_pack copies the current state's lowest n_lo
 * interior planes to send_lo (for the rank below, whose halo_hi is n_lo)
 * and its highest n_hi planes to send_hi (for the rank above, whose halo_lo
 * is n_hi); fxb_halo_unpack stores recv_lo in the halo_lo planes below the
 * slab and recv_hi in the halo_hi planes above it.  All buffers are device
 * memory (NULL where the count or halo is 0); the copies are queued on the
 * library stream (fxb_stream), so a caller orders its transfers after
 * fxb_halo_pack and before fxb_halo_unpack on that stream. */
long fxb_halo_doubles(int planes);
int fxb_halo_pack(double *send_lo, int n_lo, double *send_hi, int n_hi);
int fxb_halo_unpack(const double *recv_lo, const double *recv_hi);
/* Grid_markRefineDerefine (Grid/GridMain/AMR/Grid_markRefineDerefine.F90:77-150)
 * on the registered AMR mesh, from the attached state: a guard fill of the
 * leaves and of the parents with a leaf child (Eos on the guard regions when
 * a refinement variable is an Eos output: pres, temp, ener, eint or game),
 * then per refinement variable the error of gr_estimateBlkError.F90 for every
 * such block and the marks of Paramesh4/gr_markRefineDerefine.F90:110-160.
 * refine_var[nvars]: fxb_var ids; the cutoffs and filters are the runtime
 * parameters refine_cutoff_#, derefine_cutoff_#, refine_filter_#;
 * max_refine = lrefine_max.  flags[nleaf] (registration order): 1 refine,
 * -1 derefine, 0 neither; error[nleaf] (may be NULL): the error estimate of
 * the last variable.  The tree update itself stays with the caller's PARAMESH
 * (amr_refine_derefine); fxb_regrid then moves the data to the new leaves.
 * FXB_EUNSUPPORTED on a uniform grid. */
int fxb_mark_refine_derefine(int nvars, const int *refine_var, const double *refine_cutoff,
                             const double *derefine_cutoff, const double *refine_filter, int max_refine,
                             int *flags, double *error);
/* A block-structured AMR mesh split over ranks (one GPU each), PARAMESH's
 * Morton distribution (PM4_package/source/amr_morton_order.F90): every rank
 * registers the whole leaf list (the device keeps every leaf's interior);
 * roles[nleaf] (registration order, set before fxb_attach_unk) give this
 * rank's share of each step, and from then on the host UNK of
 * fxb_attach_unk, fxb_sync_to_host and fxb_fill_guardcells holds the own
 * leaves only, in leaf order (Flash-X's local blocks): 1 = own leaf
 * (stepped and updated; the only leaves fxb_compute_dt and fxb_integrals
 * cover), 2 = another rank's leaf one level finer across a face of an own
 * leaf (its fluxes are computed here, for the own leaf's Grid_conserveFluxes,
 * mpi_amr_flux_conserve.F90:87-132, but it is not updated), 0 = not stepped.
 * Before every step the rank receives, with fxb_amr_unpack_leaves, the
 * current interiors of the other ranks' leaves its active leaves' guard fills
 * read (mpi_amr_comm_setup.F90:531 -> mpi_xchange_blocks), packed by their
 * owners with fxb_amr_pack_leaves; a message holds fxb_amr_leaf_doubles()
 * values per leaf, [leaf][var][k][j][i] over the leaf's interior cells with
 * var in the order DENS VELX VELY VELZ PRES GAMC GAME EINT ENER TEMP, in
 * 16-byte aligned device memory, queued on the library stream.  roles NULL:
 * every leaf own. */
int fxb_amr_set_roles(const unsigned char *roles, int nleaf);
long fxb_amr_leaf_doubles(void);
int fxb_amr_pack_leaves(const int32_t *leaves, int n, double *buf);
int fxb_amr_unpack_leaves(const int32_t *leaves, int n, const double *buf);
/* Grid_updateRefinement's data movement on the device, after the caller's
 * tree update (Paramesh4/Grid_updateRefinement.F90:109,
 * gr_updateRefinement.F90:130-265): `blocks` is the new leaf list of the
 * registered AMR mesh (its order becomes the UNK slot order).  Parents of the
 * old tree are restricted from their children first (amr_restrict); each
 * block of the new tree that existed in the old one keeps its data, so a
 * derefined parent holds its children's average; new children, level by
 * level from coarse to fine, are interpolated from their parent and its
 * same-level neighbours in conserved form (amr_prolong:
 * amr_1blk_cc_prol_linear with flash_convert_cc_hook /
 * flash_unconvert_cc_hook); then Eos_wrapped(MODE_DENS_EI) runs on every
 * leaf.  The caller then resizes its UNK to the new leaf count and reads it
 * with fxb_sync_to_host.  Errors: FXB_EARG when the list is not a balanced
 * tiling or a new block's parent was not an old leaf (more than one level of
 * change); the old mesh and its data are then kept.  FXB_EUNSUPPORTED on a
 * uniform grid. */
int fxb_regrid(const fxb_block_desc *blocks, int nblk);
/* PARAMESH's tree update (PM4_package/source/mpi_amr_refine_derefine.F90:157-240,
 * amr_check_refine.F90, mpi_amr_check_derefine.F90), host only, for callers
 * without PARAMESH: from the leaves (any order) and their marks flags[n]
 * (1 refine, -1 derefine, 0 neither, as fxb_mark_refine_derefine returns
 * them), the new leaf list in PARAMESH's Morton order.  Level limits first
 * (no refinement at lrefine_max, no derefinement at lrefine_min, refinement
 * below it); a leaf one level coarser than a refining neighbour, across
 * faces, edges and corners (periodic axes wrapped), refines too; a leaf
 * derefines only if it is not a root block, no same-level neighbour is a
 * parent or refines, and all its siblings derefine, whereupon the siblings
 * become their parent.  out[cap] receives the list and *nout its length
 * (FXB_EARG with *nout set when cap is too small). */
int fxb_refine_derefine(const fxb_domain *domain, const fxb_block_desc *leaves, int n, const int *flags,
                        int lrefine_min, int lrefine_max, fxb_block_desc *out, int cap, int *nout);
/* Call counters, cumulative since fxb_init (no reference counterpart). */
#define FXB_COUNT_STEPS      0   /* hydro steps: fxb_hydro_step calls and fxb_advance steps  */
#define FXB_COUNT_DT_DEVICE  1   /* fxb_compute_dt calls that read the device (reduction, sync) */
#define FXB_COUNT_DT_CACHED  2   /* fxb_compute_dt calls answered from the cached result     */
#define FXB_COUNT_GC_FILLS   3   /* fxb_fill_guardcells / fxb_sync_to_host copies to the host */
#define FXB_COUNT_GC_DOUBLES 4   /* doubles those copies moved device -> host                */
#define FXB_NCOUNTERS        5
int fxb_counters(long long counts[FXB_NCOUNTERS]);
/* Volume integrals of caller-owned device arrays without allocating any
 * device memory (no counterpart in the reference: an addition of this
 * library).  For callers that cannot call cudaMalloc, e.g. a Fortran code
 * whose GPU memory belongs to another runtime's pool.  Inputs are device
 * pointers to ncell FP64 values each; out_dev receives the 7 sums of
 * fxb_integrals in device memory; work is queued on `stream` (0 = legacy
 * default stream) and not synchronised.  Scratch lives in a fixed static
 * device array (8192 partial sums of 4096 cells: at most 33,554,432 cells,
 * larger ncell is rejected with FXB_EARG).  The first call on each device
 * looks up that array's address, so make it before any stream capture; the
 * address stays cached for the process, so do not call it on a device after
 * a cudaDeviceReset of that device.  Calls that overlap on one GPU race on
 * the shared array: serialise them.  Results are deterministic for a given
 * ncell but differ from fxb_integrals' by roundoff (another summation
 * order). */
int fxb_integrals_noalloc(const double *dens, const double *velx, const double *vely,
                          const double *velz, const double *ener, const double *eint,
                          long ncell, double cell_volume, double *out_dev, void *stream);
/* Device time of the last fxb_hydro_step / fxb_advance, measured with CUDA
 * events on the library stream (milliseconds), and the number of kernel
 * launches it made. */
int fxb_last_timing(double *ms, int *kernel_launches);
/* The library's CUDA stream (cudaStream_t), for callers that order their own
 * work after the library's. */
void *fxb_stream(void);
/* The kernel launch shape in use, as text (no reference counterpart: the
 * batched-block path picks its CTAs per block for each stage by timing 1, 2,
 * 4, 8 and 16 at the first fxb_attach_unk of a registered mesh, and keeps
 * them for later attaches and regrids; FXB_AMR_TUNE=0 in the environment
 * keeps the defaults).  The choice changes timings, never results. */
int fxb_tuning(char *buf, int len);
int fxb_last_error(fxb_error *err);
void fxb_finalize(void);

#ifdef __cplusplus
}
#endif
#endif /* FLASHX_B200_H */
