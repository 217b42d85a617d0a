/*
 * fx_oracle.h -- CPU oracle for the Flash-X unsplit-hydro (UHD) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64, line-by-line
 * restatement of the reference Fortran solver, used as the checker for the
 * CUDA path (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg).
 * The product library never links, loads or calls it.
 *
 * Parity status: the reference is Fortran and cannot be compiled in this
 * image (no gfortran/MPI), and it ships no golden vectors for this path, so
 * the oracle is pinned by known-answer tests (exact Sod Riemann solution,
 * HLLC/HLL hand cases, conservation on periodic domains, Eos identities)
 * rather than by reference outputs: "parity unpinned" against the reference
 * binary itself.
 *
 * Storage layout follows Flash-X UNK: unk(var,i,j,k,blk) with var fastest,
 * NGUARD guard cells per side, variables in the alphabetical order the Flash-X
 * setup script assigns for UHD + Gamma:
 *   dens eint ener gamc game pres shok temp velx vely velz
 * (FX/physics/Hydro/HydroMain/unsplit/Config:66-76; bin/unitCfg.py:763-764).
 */
#ifndef FX_ORACLE_H
#define FX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { FXO_DENS = 0, FXO_EINT, FXO_ENER, FXO_GAMC, FXO_GAME, FXO_PRES,
       FXO_SHOK, FXO_TEMP, FXO_VELX, FXO_VELY, FXO_VELZ, FXO_NUNK };

enum { FXO_BC_PERIODIC = 0, FXO_BC_OUTFLOW = 1, FXO_BC_REFLECTING = 2 };
enum { FXO_ROE = 1, FXO_LLF = 2, FXO_HLL = 3, FXO_HLLC = 4, FXO_MARQ = 5, FXO_MARM = 7, FXO_HYBR = 8 };   /* UHD.h:365-371 */
enum { FXO_MINMOD = 1, FXO_MC = 2, FXO_VANLEER = 3, FXO_HYBRID = 4,
       FXO_LIMITED = 5 };

typedef struct {
    int ndim;                       /* 2 or 3 */
    int nxb, nyb, nzb;              /* block interior cells (nzb = 1 in 2-D) */
    int nblockx, nblocky, nblockz;  /* uniform block grid */
    int nguard;                     /* NGUARD (4) */
    double xmin, xmax, ymin, ymax, zmin, zmax;
    int bc[6];                      /* xl xr yl yr zl zr */
    int order;                      /* 2 = MUSCL-Hancock, 3 = PPM, 5 = WENO */
    int weno_method;                /* 1 = WENO5 (Jiang-Shu), 2 = WENO-Z */
    int riemann;                    /* FXO_ROE .. FXO_MARM */
    int limiter;                    /* FXO_MINMOD ... */
    int char_limiting;
    int use_3d_full_ctu;
    int use_aux_eint;
    int use_gravity;
    double grav[3];                 /* constant gravitational acceleration */
    double cfl, gamma, eint_switch, small_dens, small_e, small_p, tiny;
    double fpres;                   /* hy_fPresInMomFlux */
    double limited_beta;            /* LimitedSlopeBeta */
    double gas_constant, abar;      /* Eos Gamma: R and singleSpeciesA */
    int flattening;                 /* use_flattening */
    int entropy_fix;                /* Roe: entropy off (0), HartenHyman (1), Harten (2) */
    int steepening;                 /* use_steepening (PPM contact steepening) */
    int use_avisc;                  /* artificial viscosity (hy_getFaceFlux.F90:397-438) */
    double cvisc;                   /* its constant */
    int use_hybrid;                 /* use_hybridOrder (hy_dataReconstOneStep.F90:864-913) */
    double hybrid_kappa;            /* hybridOrderKappa */
    int shock_detect;               /* shockDetect: the SHOK flag before each step (hy_shockDetectBlk.F90) */
} fxo_params;

/* Number of doubles in one UNK array for the given geometry. */
long fxo_unk_size(const fxo_params *p);
/* Flop-free helpers for tests: linear UNK index of (var,i,j,k,blk). */
long fxo_index(const fxo_params *p, int var, int i, int j, int k, int blk);

/* Grid_fillGuardCells for a uniform block grid with physical BCs. */
int fxo_fill_guardcells(const fxo_params *p, double *unk);
/* Eos_wrapped(MODE_DENS_EI) on every block interior. */
int fxo_eos_interior(const fxo_params *p, double *unk);
/* Hydro(): guard fill, then per leaf block hy_computeFluxes with in-place
 * update, hy_energyFix, Eos_wrapped.  Returns 0, or a nonzero error code
 * (1 imaginary sound speed, 2 Riemann solver failure). */
int fxo_hydro_step(const fxo_params *p, double *unk, double dt, double dt_old,
                   int nthreads);
/* fxo_hydro_step with ns advected mass fractions per cell, spec[blk][k][j][i][ns]
 * (guard cells included, like UNK), the first nsp of them species that are
 * renormalised to add up to one, the rest mass scalars (fx_oracle_spec.inc) */
int fxo_hydro_step_spec(const fxo_params *p, double *unk, double *spec, int ns, int nsp, double dt,
                        double dt_old, int nthreads);
int fxo_fill_guardcells_spec(const fxo_params *p, double *spec, int ns);
/* Hydro_computeDt over all blocks: returns the global CFL time step. */
int fxo_compute_dt(const fxo_params *p, const double *unk, double *dt_out);
/* Driver_computeDt growth limit and clamp (Driver_computeDt.F90:452,460). */
double fxo_driver_dt(double dt_cfl, double dt_old, double tstep_change_factor,
                     double dtmin, double dtmax);
/* Volume integrals of mass, x/y/z momentum, total energy, internal energy,
 * kinetic energy (IO_writeIntegralQuantities.F90:60-224). */
int fxo_integrals(const fxo_params *p, const double *unk, double out[7]);
/* One Riemann problem (hy_HLLC / hy_HLL + the aux-eint fluxes of
 * hy_getFaceFlux.F90:444-453).  V = dens velx vely velz pres gamc game eint;
 * F = dens xmom ymom zmom ener pres eint volume fluxes.  Returns ierr. */
int fxo_riemann(const fxo_params *p, int dir, const double VL[8], const double VR[8], double F[8]);
/* Number of flops counted by the instrumented build (0 otherwise). */
double fxo_flops_last_step(void);

/* ---- block-structured AMR (PARAMESH) -------------------------------------
 * Leaves are given by level (1-based) and block coordinates at that level;
 * the oracle derives the parents, checks that the leaves tile the domain
 * with 2:1 balance across faces, edges and corners, and keeps restricted
 * parent data internally.  Leaf UNK is unk(var,i,j,k,leaf) as above, with
 * cell sizes halving per level.  Error codes of create: 1 bad geometry,
 * 2 level/coordinate out of range, 3 overlapping leaves, 4 incomplete tree,
 * 5 not 2:1 balanced.  Step/fill codes: 3 unsupported options, 6 a guard
 * cell with no covering block (unbalanced tree). */
typedef struct fxo_amr fxo_amr;
fxo_amr *fxo_amr_create(const fxo_params *p, int nleaf, const int *level, const int *bcoord, int *err);
void fxo_amr_free(fxo_amr *a);
int fxo_amr_info(const fxo_amr *a, int *nblk, int *maxlev);
void fxo_amr_leaf_flags(const fxo_amr *a, int leaf, int finer[6], int eos[27]);
/* Grid_fillGuardCells: restriction, same-level copies, prolongation,
 * boundary conditions, Eos on the guard regions next to other levels. */
int fxo_amr_fill_guardcells(fxo_amr *a, double *unk);
/* levelFlux Hydro(): guard fill, fluxes of every leaf, flux correction at
 * fine/coarse faces, update, energyFix, Eos. */
int fxo_amr_hydro_step(fxo_amr *a, double *unk, double dt, int nthreads);
/* one rank's share of the step of a mesh split over ranks: role[leaf] 1 owned,
 * 2 finer leaf of another rank across an owned leaf's refined face (fluxes
 * only), 0 not stepped; and dt and integrals over the owned leaves */
int fxo_amr_hydro_step_roles(fxo_amr *a, double *unk, double dt, const unsigned char *role, int nthreads);
int fxo_amr_compute_dt_roles(const fxo_amr *a, const double *unk, const unsigned char *role, double *dt_out);
int fxo_amr_integrals_roles(const fxo_amr *a, const double *unk, const unsigned char *role, double out[7]);
int fxo_amr_compute_dt(const fxo_amr *a, const double *unk, double *dt_out);
int fxo_amr_integrals(const fxo_amr *a, const double *unk, double out[7]);
/* Grid_markRefineDerefine on the leaves: flags[leaf] = 1 refine, -1 derefine,
 * 0 neither; error_out[leaf] (may be NULL) the error of the last variable;
 * ivar: UNK indices (FXO_DENS ...); 0 or 6 (guard cell without a source). */
int fxo_amr_mark_refine(fxo_amr *a, const double *unk, int nvars, const int *ivar, const double *refine_cutoff,
                        const double *derefine_cutoff, const double *refine_filter, int max_refine, int *flags,
                        double *error_out);
/* Grid_updateRefinement's data movement after the caller's tree update: the
 * leaf UNK of `old` (old_unk) becomes the leaf UNK of `nw` (new_unk, guard
 * cells zero): kept blocks copied, derefined parents restricted, new children
 * prolonged in conserved form, Eos on every leaf; 0, 6 (stencil cell without
 * a block) or 7 (a new block's parent was not an old leaf). */
int fxo_amr_regrid(fxo_amr *old, const double *old_unk, fxo_amr *nw, double *new_unk);

#ifdef __cplusplus
}
#endif
#endif
