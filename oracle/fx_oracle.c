/*
 * fx_oracle.c -- CPU oracle (test infrastructure) for the Flash-X unsplit
 * hydro block update.  See fx_oracle.h for the role and parity status.
 *
 * This file restates, in FP64 C with the reference's operation order, the
 * pure-hydro (FLASH_UHD_HYDRO), gamma-law (FLASH_EOS_GAMMA) branch of
 *   FX = Flash-X/source, UHD = FX/physics/Hydro/HydroMain/unsplit
 *   UHD/hy_computeFluxes.F90:87-417        per-block driver
 *   UHD/hy_getRiemannState.F90:79-1487     cell loop, face-state storage, 3-D CTU
 *   UHD/hy_dataReconstOneStep.F90:93-1222  per-direction dispatch, transverse terms
 *   UHD/hy_DataReconstructNormalDir_PPM.F90:84-969
 *   UHD/hy_DataReconstructNormalDir_WENO.F90:85-919
 *   UHD/hy_eigenParameters.F90:53-299, hy_eigenValue.F90:44-75,
 *   UHD/OnlyHydro/hy_eigenVector.F90:57-281
 *   UHD/hy_TVDslope.F90:65-276, hy_slopeLimiters.F90
 *   UHD/hy_upwindTransverseFlux.F90:54-222
 *   UHD/hy_getFaceFlux.F90:64-1286, hy_HLLC.F90:64-335, hy_HLL.F90:64-182,
 *   UHD/hy_prim2con.F90:34-67, hy_prim2flx.F90:36-151
 *   UHD/hy_unsplitUpdate.F90:84-1306, hy_energyFix.F90:76-480
 *   UHD/Hydro_computeDt.F90:151-291
 *   FX/physics/Eos/EosMain/{Eos_getData,Eos_putData}.F90, Gamma/Eos.F90:227-250
 *   FX/Grid/GridMain/UG/Grid_fillGuardCells.F90:260-306,
 *   FX/Grid/GridBoundaryConditions/Grid_bcApplyToRegion.F90:458-531
 *
 * Build with -ffp-contract=off: no fused multiply-adds, every operation
 * rounded as written, so results are reproducible bit for bit.
 */
#include "fx_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Primitive slots of UHD.h:373-388 (0-based): HY_DENS..HY_EINT, HY_GRAV. */
enum { H_D = 0, H_VX, H_VY, H_VZ, H_P, H_GC, H_GE, H_EI, H_GR, H_NV };
/* Flux slots UHD.h:399-406 (0-based). */
enum { F_D = 0, F_MX, F_MY, F_MZ, F_E, F_P, F_EI, F_VOL, F_NF };

/* ---- Fortran intrinsics with gfortran semantics ------------------------ */
/* MIN(a1,a2): mvar = a1; if (a2 < mvar) mvar = a2.  MAX likewise. */
static inline double fmin2(double a, double b) { return (b < a) ? b : a; }
static inline double fmax2(double a, double b) { return (b > a) ? b : a; }
static inline double fmin3(double a, double b, double c) { return fmin2(fmin2(a, b), c); }
static inline double fsign1(double b) { return copysign(1.0, b); }

/* ---- limiters: hy_slopeLimiters.F90 ------------------------------------ */
static inline double lim_minmod(double a, double b)
{ return .5 * (fsign1(a) + fsign1(b)) * fmin2(fabs(a), fabs(b)); }
static inline double lim_mc(double a, double b)
{ return (fsign1(a) + fsign1(b)) * fmin3(fabs(a), .25 * fabs(a + b), fabs(b)); }
static inline double lim_vanleer(double a, double b)
{ if (a * b <= 0.) return 0.; return 2. * a * b / (a + b); }

/* Per-block geometry shared by all routines. */
typedef struct {
    const fxo_params *p;
    int ng, nig, njg, nkg, k2, k3;
    int i0, imax, j0, jmax, k0, kmax;
    double dx, dy, dz;
    long ncell;                  /* nig*njg*nkg */
} blk_t;

static inline long cidx(const blk_t *b, int i, int j, int k)
{ return ((long)k * b->njg + j) * b->nig + i; }

static int n_end_vars(const fxo_params *p) { return p->use_gravity ? 9 : 8; }  /* HY_END_VARS */

/* Load the primitive vector V(HY_DENS:HY_GRAV) of one cell. */
static void load_v(const fxo_params *p, const double *u, double grav_dir, double V[H_NV])
{
    V[H_D] = u[FXO_DENS]; V[H_VX] = u[FXO_VELX]; V[H_VY] = u[FXO_VELY]; V[H_VZ] = u[FXO_VELZ];
    V[H_P] = u[FXO_PRES]; V[H_GC] = u[FXO_GAMC]; V[H_GE] = u[FXO_GAME]; V[H_EI] = u[FXO_EINT];
    V[H_GR] = p->use_gravity ? grav_dir : 0.;
}

/* ---- eigensystem (pure hydro, primitive form) --------------------------- */
/* hy_eigenParameters.F90:84-100, hy_eigenValue.F90:58-62,
 * OnlyHydro/hy_eigenVector.F90:87-167.  L[var][wave], R[var][wave]. */
static int eigen(const double *V, int dir, double lam[5], double L[5][5], double R[5][5])
{
    double uN = V[H_VX + dir];
    double a2 = V[H_GC] * V[H_P] / V[H_D];
    if (a2 <= 0.) return 1;
    double cf = sqrt(a2);
    lam[0] = uN - cf; lam[1] = uN; lam[2] = uN; lam[3] = uN; lam[4] = uN + cf;
    int v1 = H_VX + dir;
    int v2 = (dir == 0) ? H_VY : (dir == 1) ? H_VZ : H_VX;
    int v3 = (dir == 0) ? H_VZ : (dir == 1) ? H_VX : H_VY;
    memset(L, 0, sizeof(double) * 25);
    memset(R, 0, sizeof(double) * 25);
    double dinv = 1. / V[H_D];
    double aa2 = cf * cf;
    double a2inv = 1. / aa2;
    double ahinv = 0.5 / cf;
    double Na = 0.5 * a2inv;
    L[v1][0] = -ahinv;  L[H_P][0] = dinv * Na;
    L[v2][1] = 1.;
    L[H_D][2] = 1.;     L[H_P][2] = -a2inv;
    L[v3][3] = 1.;
    L[v1][4] = ahinv;   L[H_P][4] = L[H_P][0];
    R[H_D][0] = V[H_D]; R[v1][0] = -cf; R[H_P][0] = V[H_D] * aa2;
    R[v2][1] = 1.;
    R[H_D][2] = 1.;
    R[v3][3] = 1.;
    R[H_D][4] = V[H_D]; R[v1][4] = cf;  R[H_P][4] = R[H_P][0];
    return 0;
}

/* Fortran dot_product over HY_DENS:HY_PRES with a zero-initialised sum. */
static inline double dot5(double L[5][5], int w, const double *x)
{
    double s = 0.;
    for (int v = 0; v < 5; v++) s = s + L[v][w] * x[v];
    return s;
}

/* ---- hy_TVDslope.F90:65-276 -------------------------------------------- */
static void tvd_slope(const fxo_params *p, const double *VL, const double *V0, const double *VR,
                      double L[5][5], double delbar[H_NV])
{
    double dL[H_NV], dR[H_NV];
    int nend = n_end_vars(p);
    for (int k = 0; k < H_NV; k++) { delbar[k] = 0.; dL[k] = V0[k] - VL[k]; dR[k] = VR[k] - V0[k]; }
    int lim = p->limiter;
    if (lim == FXO_MINMOD || lim == FXO_MC || lim == FXO_VANLEER) {
        double (*f)(double, double) = (lim == FXO_MINMOD) ? lim_minmod : (lim == FXO_MC) ? lim_mc : lim_vanleer;
        if (p->char_limiting) {
            for (int w = 0; w < 5; w++) delbar[w] = f(dot5(L, w, dL), dot5(L, w, dR));
            for (int k = H_GC; k < nend; k++) delbar[k] = f(dL[k], dR[k]);
        } else {
            for (int k = 0; k < nend; k++) delbar[k] = f(dL[k], dR[k]);
        }
    } else if (lim == FXO_HYBRID) {
        if (p->char_limiting) {
            delbar[0] = lim_minmod(dot5(L, 0, dL), dot5(L, 0, dR));
            delbar[1] = lim_minmod(dot5(L, 1, dL), dot5(L, 1, dR));
            delbar[2] = lim_mc(dot5(L, 2, dL), dot5(L, 2, dR));
            delbar[3] = lim_minmod(dot5(L, 3, dL), dot5(L, 3, dR));
            delbar[4] = lim_minmod(dot5(L, 4, dL), dot5(L, 4, dR));
            for (int k = H_GC; k < nend; k++) delbar[k] = lim_mc(dL[k], dR[k]);
        } else {
            for (int k = 0; k < nend; k++) {
                if (k == H_D || k == H_GC || k == H_GE || k == H_GR) delbar[k] = lim_mc(dL[k], dR[k]);
                else if (k >= H_VX && k <= H_P) delbar[k] = lim_minmod(dL[k], dR[k]);
            }
        }
    } else { /* LIMITED */
        double beta = p->limited_beta;
        int nw = p->char_limiting ? 5 : 0;
        for (int k = 0; k < nend; k++) {
            double d1, d2;
            if (k < nw) { d1 = dot5(L, k, dL); d2 = dot5(L, k, dR); }
            else if (p->char_limiting && k < H_GC) continue;
            else { d1 = dL[k]; d2 = dR[k]; }
            if (d2 > 0.) delbar[k] = fmax2(fmax2(0., fmin2(beta * d1, d2)), fmin2(d1, beta * d2));
            else         delbar[k] = fmin2(fmin2(0., fmax2(beta * d1, d2)), fmax2(d1, beta * d2));
        }
    }
}

/* ---- hy_upwindTransverseFlux.F90:54-222 (hydro variables) -------------- */
static void upwind_trans(const fxo_params *p, const double *vm1, const double *vc0, const double *vp1,
                         const double lam[5], double L[5][5], double R[5][5], int sig_size, double *sig)
{
    double TF[H_NV];
    for (int k = 0; k < sig_size; k++) sig[k] = 0.;
    for (int n = 0; n < 5; n++) {
        if (lam[n] > 0.) { for (int v = 0; v < 5; v++) TF[v] = vc0[v] - vm1[v]; }
        else             { for (int v = 0; v < 5; v++) TF[v] = vp1[v] - vc0[v]; }
        double d = dot5(L, n, TF);
        for (int v = 0; v < 5; v++) { TF[v] = lam[n] * R[v][n] * d; sig[v] = sig[v] + TF[v]; }
    }
    if (p->use_aux_eint) {          /* hyBeg = hyVarEnd = HY_EINT */
        double t = (lam[2] > 0.) ? (vc0[H_EI] - vm1[H_EI]) : (vp1[H_EI] - vc0[H_EI]);
        sig[H_EI] = lam[2] * t;
        if (p->use_gravity && H_GR < sig_size) sig[H_GR] = 0.;
    }
}

/* ---- hy_DataReconstructNormalDir_PPM.F90:84-969 ------------------------ */
/* S[0..4] = Vmm, Vm, Vc, Vp, Vpp (Vmm/Vpp unused when trans_only). */
static int recon_ppm(const fxo_params *p, int dir, double dt, double delta,
                     const double *S[5], int trans_only, double flat,
                     double lam0[5], double L0[5][5], double R0[5][5],
                     double Wp[H_NV], double Wm[H_NV], double sig[H_NV])
{
    const int nend = p->use_gravity ? 9 : (p->use_aux_eint ? 8 : 5);   /* hyEndVar */
    const int npr = 5;                                                   /* hyEndPrimVar */
    const double *Vm = S[1], *Vc = S[2], *Vp = S[3];
    double dtn = dt / delta, hdtn = 0.5 * dtn;
    for (int k = 0; k < H_NV; k++) { Wp[k] = 0.; Wm[k] = 0.; }
    if (eigen(Vc, dir, lam0, L0, R0)) return 1;
    if (p->ndim > 1) upwind_trans(p, Vm, Vc, Vp, lam0, L0, R0, n_end_vars(p), sig);
    if (trans_only) return 0;

    double lamP[5], LP[5][5], RP[5][5], lamN[5], LN[5][5], RN[5][5];
    if (eigen(Vp, dir, lamP, LP, RP)) return 1;
    if (eigen(Vm, dir, lamN, LN, RN)) return 1;
    double dbN[H_NV], db0[H_NV], dbP[H_NV];
    tvd_slope(p, S[0], Vm, Vc, LN, dbN);
    tvd_slope(p, Vm, Vc, Vp, L0, db0);
    tvd_slope(p, Vc, Vp, S[4], LP, dbP);
    if (p->char_limiting) {
        double t0[5], tP[5], tN[5];
        for (int v = 0; v < 5; v++) {
            t0[v] = R0[v][0] * db0[0] + R0[v][1] * db0[1] + R0[v][2] * db0[2] + R0[v][3] * db0[3] + R0[v][4] * db0[4];
            tP[v] = RP[v][0] * dbP[0] + RP[v][1] * dbP[1] + RP[v][2] * dbP[2] + RP[v][3] * dbP[3] + RP[v][4] * dbP[4];
            tN[v] = RN[v][0] * dbN[0] + RN[v][1] * dbN[1] + RN[v][2] * dbN[2] + RN[v][3] * dbN[3] + RN[v][4] * dbN[4];
        }
        for (int v = 0; v < 5; v++) { db0[v] = t0[v]; dbP[v] = tP[v]; dbN[v] = tN[v]; }
    }
    double vecL[H_NV], vecR[H_NV], delW[H_NV], W6[H_NV];
    for (int k = 0; k < H_NV; k++) { vecL[k] = 0.; vecR[k] = 0.; }
    for (int n = 0; n < nend; n++) {
        vecL[n] = 0.5 * (Vc[n] + Vm[n]) - (db0[n] - dbN[n]) / 6.;
        vecR[n] = 0.5 * (Vc[n] + Vp[n]) - (dbP[n] - db0[n]) / 6.;
    }
    /* [4] contact steepening, hy_DataReconstructNormalDir_PPM.F90:650-681
     * (eta1 = 20, eta2 = 0.05, epsln = 0.01, K0 = 0.1 from :149) */
    if (p->steepening) {
        const double temp1 = Vp[H_D] - Vm[H_D];
        if (fabs(temp1) > p->tiny) {
            const double d2R = (S[4][H_D] - 2. * Vp[H_D] + Vc[H_D]) / (6. * delta * delta);
            const double d2L = (Vc[H_D] - 2. * Vm[H_D] + S[0][H_D]) / (6. * delta * delta);
            double eta = (d2L - d2R) * (delta * delta) / temp1;
            if (d2R * d2L >= 0.) eta = 0.;
            if (0.01 * fmin2(Vp[H_D], Vm[H_D]) - fabs(Vp[H_D] - Vm[H_D]) >= 0.) eta = 0.;
            eta = fmax2(0., fmin2(1., 20. * (eta - 0.05)));
            const double temp2 = fabs(Vp[H_P] - Vm[H_P]) / fmin2(Vp[H_P], Vm[H_P]);
            const double temp3 = fabs(Vp[H_D] - Vm[H_D]) / fmin2(Vp[H_D], Vm[H_D]);
            if (Vc[H_GE] * 0.1 * temp3 - temp2 < 0.0) eta = 0.;
            vecL[H_D] = vecL[H_D] * (1. - eta) + (Vm[H_D] + 0.5 * dbN[H_D]) * eta;
            vecR[H_D] = vecR[H_D] * (1. - eta) + (Vp[H_D] - 0.5 * dbP[H_D]) * eta;
        }
    }
    /* [5] flattening, hy_DataReconstructNormalDir_PPM.F90:687-690 */
    if (p->flattening)
        for (int n = 0; n < nend; n++) {
            vecL[n] = flat * Vc[n] + (1.0 - flat) * vecL[n];
            vecR[n] = flat * Vc[n] + (1.0 - flat) * vecR[n];
        }
    /* monotonicity, CW84 eq. 1.10 */
    for (int n = 0; n < nend; n++) {
        if ((vecR[n] - Vc[n]) * (Vc[n] - vecL[n]) <= 0.) { vecL[n] = Vc[n]; vecR[n] = Vc[n]; }
        if (6. * (vecR[n] - vecL[n]) * (Vc[n] - 0.5 * (vecL[n] + vecR[n])) > (vecR[n] - vecL[n]) * (vecR[n] - vecL[n]))
            vecL[n] = 3. * Vc[n] - 2. * vecR[n];
        if (6. * (vecR[n] - vecL[n]) * (Vc[n] - 0.5 * (vecL[n] + vecR[n])) < -((vecR[n] - vecL[n]) * (vecR[n] - vecL[n])))
            vecR[n] = 3. * Vc[n] - 2. * vecL[n];
    }
    for (int n = 0; n < nend; n++) {
        delW[n] = vecR[n] - vecL[n];
        W6[n] = 6. * (Vc[n] - 0.5 * (vecR[n] + vecL[n]));
    }
    /* [7] initial guesses: only the secondary variables survive [10] */
    double lmax = fmax2(lam0[2], 0.);
    for (int n = npr; n < nend; n++)
        Wp[n] = vecR[n] - lmax * hdtn * (delW[n] - (1.0 - lmax * hdtn * 4. / 3.) * W6[n]);
    double lmin = -fmin2(lam0[2], 0.);
    for (int n = npr; n < nend; n++)
        Wm[n] = vecL[n] + lmin * hdtn * (delW[n] + (1.0 - lmin * hdtn * 4. / 3.) * W6[n]);
    Wp[H_GC] = Vc[H_GC]; Wp[H_GE] = Vc[H_GE];   /* FLASH_EOS_GAMMA */
    Wm[H_GC] = Vc[H_GC]; Wm[H_GE] = Vc[H_GE];
    if (p->use_gravity) { Wp[H_GR] = vecR[H_GR]; Wm[H_GR] = vecL[H_GR]; }
    /* [8] characteristic tracing, HLL-type branch */
    double sigL[5] = {0., 0., 0., 0., 0.}, sigR[5] = {0., 0., 0., 0., 0.};
    double mW6[5];
    for (int v = 0; v < 5; v++) mW6[v] = -W6[v];
    for (int n = 0; n < 5; n++) {
        double cA = dot5(L0, n, delW);
        double cB = dot5(L0, n, mW6);
        double lt = dtn * lam0[n];
        double aL = .5 * (-1. - dtn * lam0[n]);
        double bL = .25 * (1. + 2. * dtn * lam0[n] + 4. / 3. * (lt * lt));
        double aR = .5 * (1. - dtn * lam0[n]);
        double bR = .25 * (1. - 2. * dtn * lam0[n] + 4. / 3. * (lt * lt));
        for (int v = 0; v < 5; v++) {
            sigL[v] = sigL[v] + (aL * R0[v][n] * cA + bL * R0[v][n] * cB);
            sigR[v] = sigR[v] + (aR * R0[v][n] * cA + bR * R0[v][n] * cB);
        }
    }
    for (int v = 0; v < npr; v++) {
        Wm[v] = Vc[v] + W6[v] / 12. + sigL[v];
        Wp[v] = Vc[v] + W6[v] / 12. + sigR[v];
    }
    return 0;
}

/* ---- hy_DataReconstructNormalDir_MH.F90 (MUSCL-Hancock, order 2) -------- */
/* S[1..3] = Vm, Vc, Vp.  One TVD slope of the cell (characteristic amplitudes
 * for the waves when charLimiting, primitive otherwise), flattened; eint (and
 * the gravity slot) reconstructed linearly, clamped between the cell value
 * and the face value and traced with the entropy wave (not gravity); the
 * primitive variables traced over the five waves (Roe: the upwind side
 * only); gamc and game constant (FLASH_EOS_GAMMA). */
static int recon_mh(const fxo_params *p, int dir, double dt, double delta,
                    const double *S[5], int trans_only, double flat,
                    double lam0[5], double L0[5][5], double R0[5][5],
                    double Wp[H_NV], double Wm[H_NV], double sig[H_NV])
{
    const int nend = p->use_gravity ? 9 : (p->use_aux_eint ? 8 : 5);   /* hyEndVar + 1 */
    const double *Vm = S[1], *Vc = S[2], *Vp = S[3];
    const double dtn = dt / delta, hdtn = 0.5 * dtn;
    for (int k = 0; k < H_NV; k++) { Wp[k] = 0.; Wm[k] = 0.; }
    if (eigen(Vc, dir, lam0, L0, R0)) return 1;
    if (p->ndim > 1) upwind_trans(p, Vm, Vc, Vp, lam0, L0, R0, n_end_vars(p), sig);
    if (trans_only) return 0;
    double delbar[H_NV];
    tvd_slope(p, Vm, Vc, Vp, L0, delbar);
    if (p->flattening)
        for (int k = 0; k < H_NV; k++) delbar[k] = delbar[k] * (1. - flat);
    Wp[H_GC] = Vc[H_GC]; Wp[H_GE] = Vc[H_GE];
    Wm[H_GC] = Vc[H_GC]; Wm[H_GE] = Vc[H_GE];
    for (int n = H_EI; n < nend; n++) {
        Wp[n] = Vc[n] + 0.5 * delbar[n];
        Wm[n] = Vc[n] - 0.5 * delbar[n];
        Wm[n] = fmax2(fmin2(Vc[n], Wm[n]), fmin2(fmax2(Vc[n], Wm[n]), Wm[n]));
        Wp[n] = fmax2(fmin2(Vc[n], Wp[n]), fmin2(fmax2(Vc[n], Wp[n]), Wp[n]));
        if (n != H_GR) {
            Wp[n] = Wp[n] - fmax2(lam0[3], 0.) * hdtn * delbar[n];
            Wm[n] = Wm[n] - fmin2(lam0[3], 0.) * hdtn * delbar[n];
        }
    }
    double sigL[5] = {0., 0., 0., 0., 0.}, sigR[5] = {0., 0., 0., 0., 0.};
    const int roe = p->riemann == FXO_ROE;
    for (int n = 0; n < 5; n++) {
        const double amp = p->char_limiting ? delbar[n] : dot5(L0, n, delbar);
        const double cL = .5 * (-1. - dtn * lam0[n]), cR = .5 * (1. - dtn * lam0[n]);
        const int left = !roe || lam0[n] < 0., right = !roe || !(lam0[n] < 0.);
        for (int v = 0; v < 5; v++) {
            if (left) sigL[v] = sigL[v] + cL * R0[v][n] * amp;
            if (right) sigR[v] = sigR[v] + cR * R0[v][n] * amp;
        }
    }
    for (int v = 0; v < 5; v++) {
        Wm[v] = Vc[v] + sigL[v];
        Wp[v] = Vc[v] + sigR[v];
    }
    return 0;
}

/* ---- WENO5 / WENO-Z reconstruction: see recon_weno below --------------- */
static int recon_weno(const fxo_params *p, int dir, double dt, double delta,
                      const double *S[5], int trans_only, double flat,
                      double lam0[5], double L0[5][5], double R0[5][5],
                      double Wp[H_NV], double Wm[H_NV], double sig[H_NV]);

/* ---- Riemann solvers ---------------------------------------------------- */
/* hy_prim2con.F90:34-67 */
static void prim2con(const double *V, double U[5])
{
    double u2 = 0.; u2 = u2 + V[H_VX] * V[H_VX]; u2 = u2 + V[H_VY] * V[H_VY]; u2 = u2 + V[H_VZ] * V[H_VZ];
    U[0] = V[H_D];
    U[1] = V[H_D] * V[H_VX]; U[2] = V[H_D] * V[H_VY]; U[3] = V[H_D] * V[H_VZ];
    U[4] = 0.5 * V[H_D] * u2 + V[H_P] / (V[H_GE] - 1.) + 0.5 * 0.;
}
/* hy_prim2flx.F90:36-151 (hydro) */
static void prim2flx(const fxo_params *p, int dir, const double *V, double F[6])
{
    double u2 = 0.; u2 = u2 + V[H_VX] * V[H_VX]; u2 = u2 + V[H_VY] * V[H_VY]; u2 = u2 + V[H_VZ] * V[H_VZ];
    double E = 0.5 * V[H_D] * u2 + V[H_P] / (V[H_GE] - 1.);
    double fP = p->fpres;
    F[F_P] = V[H_P];
    double vn = V[H_VX + dir];
    F[F_D] = V[H_D] * vn;
    F[F_MX] = F[F_D] * V[H_VX];
    F[F_MY] = F[F_D] * V[H_VY];
    F[F_MZ] = F[F_D] * V[H_VZ];
    F[F_MX + dir] = F[F_D] * V[H_VX + dir] + fP * V[H_P];
    F[F_E] = (E + V[H_P]) * vn;
}

/* hy_HLLC.F90:64-335 (hydro).  Returns ierr. */
static int riemann_hllc(const fxo_params *p, int dir, const double *Vm, const double *Vp, double Fs[6], double *speed)
{
    double velNL = Vm[H_VX + dir], velNR = Vp[H_VX + dir];
    double aL2 = Vm[H_GC] * Vm[H_P] / Vm[H_D];
    double aR2 = Vp[H_GC] * Vp[H_P] / Vp[H_D];
    double tiny = p->tiny;
    if ((Vm[H_D] < tiny && Vm[H_D] > 0.) || (Vp[H_D] < tiny && Vp[H_D] > 0.) ||
        (Vm[H_P] < tiny && Vm[H_P] > 0.) || (Vp[H_P] < tiny && Vp[H_P] > 0.)) {
        for (int k = 0; k < 6; k++) Fs[k] = 0.;
        *speed = 0.;
        return 0;
    } else if (aL2 < 0. || aR2 < 0.) {
        return 1;
    }
    double cfL = sqrt(aL2), cfR = sqrt(aR2);
    double SL = fmin2(velNL - cfL, velNR - cfR);
    double SR = fmax2(velNL + cfL, velNR + cfR);
    *speed = fmax2(fabs(SL), fabs(SR));
    double pL = Vm[H_P], pR = Vp[H_P];
    double UL[5], UR[5], FL[6], FR[6];
    prim2con(Vm, UL); prim2con(Vp, UR);
    prim2flx(p, dir, Vm, FL); prim2flx(p, dir, Vp, FR);
    /* (the HLL average state Uhll of :155-168 only feeds the MHD branch) */
    double qStar = (Vp[H_D] * velNR * (SR - velNR) - Vm[H_D] * velNL * (SL - velNL) + pL - pR - 0. * 0. + 0. * 0.);
    qStar = qStar / (Vp[H_D] * (SR - velNR) - Vm[H_D] * (SL - velNL));
    double numerL = SL - velNL, denomL = SL - qStar;
    double numerR = SR - velNR, denomR = SR - qStar;
    double pStar = Vm[H_D] * numerL * (qStar - velNL) + pL;
    double dStarL = UL[0] * numerL / denomL;
    double dStarR = UR[0] * numerR / denomR;
    double UCL[5], UCR[5];
    UCL[0] = dStarL;
    UCL[4] = UL[4] * numerL / denomL + ((pStar * qStar - pL * velNL)) / denomL;
    UCR[0] = dStarR;
    UCR[4] = UR[4] * numerR / denomR + ((pStar * qStar - pR * velNR)) / denomR;
    for (int d = 0; d < 3; d++) {
        if (d == dir) { UCL[1 + d] = dStarL * qStar; UCR[1 + d] = dStarR * qStar; }
        else { UCL[1 + d] = UL[1 + d] * numerL / denomL; UCR[1 + d] = UR[1 + d] * numerR / denomR; }
    }
    if (SL >= 0.) {
        for (int k = 0; k < 6; k++) Fs[k] = FL[k];
    } else if (SL < 0. && qStar >= 0.) {
        for (int k = 0; k < 5; k++) Fs[k] = FL[k] + SL * (UCL[k] - UL[k]);
        Fs[F_P] = FL[F_P];
    } else if (qStar < 0. && SR >= 0.) {
        for (int k = 0; k < 5; k++) Fs[k] = FR[k] + SR * (UCR[k] - UR[k]);
        Fs[F_P] = FR[F_P];
    } else {
        for (int k = 0; k < 6; k++) Fs[k] = FR[k];
    }
    return 0;
}

/* hy_HLL.F90:64-182 (hydro).  Note the solver's own tiny = 1e-32. */
static int riemann_hll(const fxo_params *p, int dir, const double *Vm, const double *Vp, double Fs[6], double *speed)
{
    (void)p;
    const double tiny = 1.e-32;
    double velNL = Vm[H_VX + dir], velNR = Vp[H_VX + dir];
    double aL2 = Vm[H_GC] * Vm[H_P] / Vm[H_D];
    double aR2 = Vp[H_GC] * Vp[H_P] / Vp[H_D];
    if ((Vm[H_D] < tiny && Vm[H_D] > 0.) || (Vp[H_D] < tiny && Vp[H_D] > 0.) ||
        (Vm[H_P] < tiny && Vm[H_P] > 0.) || (Vp[H_P] < tiny && Vp[H_P] > 0.)) {
        for (int k = 0; k < 6; k++) Fs[k] = 0.;
        *speed = 0.;
        return 0;
    } else if (aL2 < 0. || aR2 < 0.) {
        return 1;
    }
    double cfL = sqrt(aL2), cfR = sqrt(aR2);
    double SL = fmin2(velNL - cfL, velNR - cfR);
    double SR = fmax2(velNL + cfL, velNR + cfR);
    *speed = fmax2(fabs(SL), fabs(SR));
    double UL[6], UR[6], FL[6], FR[6];
    prim2con(Vm, UL); prim2con(Vp, UR);
    UL[5] = 0.; UR[5] = 0.;
    prim2flx(p, dir, Vm, FL); prim2flx(p, dir, Vp, FR);
    if (SL > 0.) {
        for (int k = 0; k < 6; k++) Fs[k] = FL[k];
    } else if (SR < 0.) {
        for (int k = 0; k < 6; k++) Fs[k] = FR[k];
    } else {
        for (int k = 0; k < 6; k++)
            Fs[k] = (SR * FL[k] - SL * FR[k] + SR * SL * (UR[k] - UL[k])) / (SR - SL);
    }
    return 0;
}

/* hy_slopeLimiters.F90:74-82 */
static double signum_(double x) { return x == 0. ? 0. : (x > 0. ? 1. : -1.); }

/* largest |eigenvalue| of hy_eigenValue.F90 (hydro: u-c, u, u, u, u+c), in maxval order */
static double maxabs_lambda(double un, double cf)
{
    const double l[5] = {un - cf, un, un, un, un + cf};
    double m = fabs(l[0]);
    for (int k = 1; k < 5; k++) if (fabs(l[k]) > m) m = fabs(l[k]);
    return m;
}

/* hy_LLF.F90:62-183 (hydro): the largest |wave speed| of the averaged
 * (hy_avgState.F90:34-60), left and right states (hy_eigenParameters.F90:
 * 83-100, which aborts on a2 <= 0) times the jump of the conserved state,
 * subtracted from the mean of the two physical fluxes. */
static int riemann_llf(const fxo_params *p, int dir, const double *Vm, const double *Vp, double Fs[6], double *speed)
{
    const double tiny = 1.e-32;
    double aL2 = Vm[H_GC] * Vm[H_P] / Vm[H_D];
    double aR2 = Vp[H_GC] * Vp[H_P] / Vp[H_D];
    if ((Vm[H_D] < tiny && Vm[H_D] > 0.) || (Vp[H_D] < tiny && Vp[H_D] > 0.) ||
        (Vm[H_P] < tiny && Vm[H_P] > 0.) || (Vp[H_P] < tiny && Vp[H_P] > 0.)) {
        for (int k = 0; k < 6; k++) Fs[k] = 0.;
        *speed = 0.;
        return 0;
    } else if (aL2 < 0. || aR2 < 0.) {
        return 1;
    }
    /* hy_avgState: the mean state, gammas taken upwind of the mean normal velocity */
    double Va[H_NV];
    for (int k = 0; k < H_NV; k++) Va[k] = 0.;
    Va[H_D] = .5 * (Vm[H_D] + Vp[H_D]);
    Va[H_VX] = .5 * (Vm[H_VX] + Vp[H_VX]);
    Va[H_VY] = .5 * (Vm[H_VY] + Vp[H_VY]);
    Va[H_VZ] = .5 * (Vm[H_VZ] + Vp[H_VZ]);
    Va[H_P] = .5 * (Vm[H_P] + Vp[H_P]);
    const double sig = signum_(Va[H_VX + dir]);
    Va[H_GC] = 0.5 * ((1. + sig) * Vm[H_GC] + (1. - sig) * Vp[H_GC]);
    Va[H_GE] = 0.5 * ((1. + sig) * Vm[H_GE] + (1. - sig) * Vp[H_GE]);
    const double a2 = Va[H_GC] * Va[H_P] / Va[H_D];
    const double a2L = Vm[H_GC] * Vm[H_P] / Vm[H_D], a2R = Vp[H_GC] * Vp[H_P] / Vp[H_D];
    if (a2 <= 0. || a2L <= 0. || a2R <= 0.) return 1;
    const double lm = maxabs_lambda(Va[H_VX + dir], sqrt(a2));
    const double lL = maxabs_lambda(Vm[H_VX + dir], sqrt(a2L));
    const double lR = maxabs_lambda(Vp[H_VX + dir], sqrt(a2R));
    const double smax = fmax2(fmax2(lm, lL), lR);
    *speed = fabs(Vp[H_VX + dir]) + fabs(sqrt(a2R));
    double UL[6], UR[6], FL[6], FR[6];
    prim2con(Vm, UL); prim2con(Vp, UR);
    UL[5] = 0.; UR[5] = 0.;
    prim2flx(p, dir, Vm, FL); prim2flx(p, dir, Vp, FR);
    for (int k = 0; k < 6; k++) Fs[k] = (FR[k] + FL[k] - smax * (UR[k] - UL[k])) * 0.5;
    return 0;
}

/* OnlyHydro/hy_eigenVector.F90:128-166 (cons = .true.): conservative left
 * and right eigenvectors of state V (D, VX, VY, VZ, P, GC, GE), rows D, MX,
 * MY, MZ, E, columns the five waves */
static void cons_eigen(const double *Va, int dir, double cf, double L[5][5], double R[5][5])
{
    /* conservative eigenvectors: rows D, MX, MY, MZ, E; columns the five waves */
    const int v1 = H_VX + dir, v2 = H_VX + (dir + 1) % 3, v3 = H_VX + (dir + 2) % 3;
    const double V1 = Va[v1], V2 = Va[v2], V3 = Va[v3];
    const double k = 1. - Va[H_GE];
    const double a2e = cf * cf, a2inv = 1. / a2e, Na = 0.5 * a2inv;
    double u2 = 0.;
    u2 = u2 + Va[H_VX] * Va[H_VX]; u2 = u2 + Va[H_VY] * Va[H_VY]; u2 = u2 + Va[H_VZ] * Va[H_VZ];
    u2 = 0.5 * u2;
    const double H = (Va[H_D] * u2 - Va[H_P] / k + Va[H_P]) / Va[H_D];
    memset(L, 0, sizeof(double) * 25); memset(R, 0, sizeof(double) * 25);
    const int E = H_P;
    L[H_D][0] = Na * (-(k * u2) + V1 * cf); L[v1][0] = -(Na * (-(k * V1) + cf));
    L[v2][0] = Na * k * V2; L[v3][0] = Na * k * V3; L[E][0] = -(Na * k);
    L[H_D][1] = -V2; L[v2][1] = 1.;
    L[H_D][2] = 1. + Na * k * u2 * 2.;
    L[v1][2] = -(k * V1 * a2inv); L[v2][2] = -(k * V2 * a2inv); L[v3][2] = -(k * V3 * a2inv); L[E][2] = k * a2inv;
    L[H_D][3] = -V3; L[v3][3] = 1.;
    L[H_D][4] = Na * (-(k * u2) - V1 * cf); L[v1][4] = -(Na * (-(k * V1) - cf));
    L[v2][4] = Na * k * V2; L[v3][4] = Na * k * V3; L[E][4] = -(Na * k);
    R[H_D][0] = 1.; R[v1][0] = V1 - cf; R[v2][0] = V2; R[v3][0] = V3; R[E][0] = H - V1 * cf;
    R[v2][1] = 1.; R[E][1] = V2;
    R[H_D][2] = 1.; R[v1][2] = V1; R[v2][2] = V2; R[v3][2] = V3; R[E][2] = u2;
    R[v3][3] = 1.; R[E][3] = V3;
    R[H_D][4] = 1.; R[v1][4] = V1 + cf; R[v2][4] = V2; R[v3][4] = V3; R[E][4] = H + V1 * cf;
}

/* hy_Roe.F90:62-205 (hydro): the mean state of hy_avgState, its eigenvalues
 * (the acoustic ones corrected by hy_entropyFix.F90 when entropy = .true.)
 * and conservative eigenvectors (OnlyHydro/hy_eigenVector.F90:128-166,
 * cons = .true.), and the flux
 * (FL + FR - sum_k |lambda_k| r_k (l_k . (UR - UL))) / 2; the dot products
 * run over all five rows, zeros included, as dot_product does. */
static int riemann_roe(const fxo_params *p, int dir, const double *Vm, const double *Vp, double Fs[6], double *speed)
{
    const double tiny = 1.e-32;
    double aL2 = Vm[H_GC] * Vm[H_P] / Vm[H_D];
    double aR2 = Vp[H_GC] * Vp[H_P] / Vp[H_D];
    if ((Vm[H_D] < tiny && Vm[H_D] > 0.) || (Vp[H_D] < tiny && Vp[H_D] > 0.) ||
        (Vm[H_P] < tiny && Vm[H_P] > 0.) || (Vp[H_P] < tiny && Vp[H_P] > 0.)) {
        for (int k = 0; k < 6; k++) Fs[k] = 0.;
        *speed = 0.;
        return 0;
    } else if (aL2 < 0. || aR2 < 0.) {
        return 1;
    }
    double Va[H_NV];
    for (int k = 0; k < H_NV; k++) Va[k] = 0.;
    Va[H_D] = .5 * (Vm[H_D] + Vp[H_D]);
    Va[H_VX] = .5 * (Vm[H_VX] + Vp[H_VX]);
    Va[H_VY] = .5 * (Vm[H_VY] + Vp[H_VY]);
    Va[H_VZ] = .5 * (Vm[H_VZ] + Vp[H_VZ]);
    Va[H_P] = .5 * (Vm[H_P] + Vp[H_P]);
    const double sig = signum_(Va[H_VX + dir]);
    Va[H_GC] = 0.5 * ((1. + sig) * Vm[H_GC] + (1. - sig) * Vp[H_GC]);
    Va[H_GE] = 0.5 * ((1. + sig) * Vm[H_GE] + (1. - sig) * Vp[H_GE]);
    const double a2 = Va[H_GC] * Va[H_P] / Va[H_D];
    if (a2 <= 0.) return 1;
    const double cf = sqrt(a2), un = Va[H_VX + dir];
    double lam[5] = {un - cf, un, un, un, un + cf};
    if (p->entropy_fix) {   /* hy_entropyFix.F90 on the two acoustic waves */
        const double a2L = Vm[H_GC] * Vm[H_P] / Vm[H_D], a2R = Vp[H_GC] * Vp[H_P] / Vp[H_D];
        if (a2L <= 0. || a2R <= 0.) return 1;
        const double uL = Vm[H_VX + dir], uR = Vp[H_VX + dir], cL = sqrt(a2L), cR = sqrt(a2R);
        const double lL[5] = {uL - cL, uL, uL, uL, uL + cL}, lR[5] = {uR - cR, uR, uR, uR, uR + cR};
        for (int w = 0; w < 5; w += 4) {
            if (lR[w] > 0. && lL[w] < 0.) {
                if (p->entropy_fix == 1) {          /* HartenHyman */
                    const double Lh = lL[w] * (lR[w] - lam[w]) / (lR[w] - lL[w]);
                    const double Rh = lR[w] * (lam[w] - lL[w]) / (lR[w] - lL[w]);
                    lam[w] = Rh - Lh;
                } else {                             /* Harten */
                    const double dl = fmax2(4.0 * (lR[w] - lL[w]), 0.0);
                    if (fabs(lam[w]) < 0.5 * dl) {
                        if (lam[w] >= 0.0) lam[w] = (lam[w] * lam[w] / dl + .25 * dl);
                        else lam[w] = -(lam[w] * lam[w] / dl + .25 * dl);
                    }
                }
            }
        }
    }
    double L[5][5], R[5][5];
    cons_eigen(Va, dir, cf, L, R);
    *speed = fabs(un) + fabs(cf);
    double UL[5], UR[5], FL[6], FR[6], dU[5];
    prim2con(Vm, UL); prim2con(Vp, UR);
    prim2flx(p, dir, Vm, FL); prim2flx(p, dir, Vp, FR);
    for (int v = 0; v < 5; v++) dU[v] = UR[v] - UL[v];
    double sigF[6] = {0., 0., 0., 0., 0., 0.};
    for (int w = 0; w < 5; w++) {
        double dp = 0.;
        for (int v = 0; v < 5; v++) dp = dp + L[v][w] * dU[v];
        for (int v = 0; v < 5; v++) sigF[v] = sigF[v] + fabs(lam[w]) * R[v][w] * dp;
    }
    for (int v = 0; v < 6; v++) Fs[v] = (FR[v] + FL[v] - sigF[v]) * 0.5;
    return 0;
}

/* hy_eigenValue.F90 (hydro): u - c, u, u, u, u + c */
static void eigen_values(double un, double cf, double lam[5])
{
    lam[0] = un - cf; lam[1] = un; lam[2] = un; lam[3] = un; lam[4] = un + cf;
}

/* hy_Marquina.F90:52-227 (hydro), restated as written: the eigenvalues and
 * conservative eigenvectors (OnlyHydro/hy_eigenVector.F90, cons = .true.)
 * of the left and of the right state; per wave k, where both states move
 * the same way, the upwind state's characteristic flux, else half of each
 * state's flux plus or minus the largest |eigenvalue| times its conserved
 * state; the flux is the sum of both sides' parts along their right
 * eigenvectors.  Two details of the reference are kept: the left
 * eigenvectors, stored as leig(variable, wave), are read as leig(k, 1:5)
 * (:165-183), and each projection adds leig(k, XMOM + dir - 1) times the
 * face pressure to a momentum flux that already carries hy_fPresInMomFlux
 * times the pressure (hy_prim2flx.F90).  The face-pressure slot is zero
 * (:186). */
static int riemann_marquina(const fxo_params *p, int dir, const double *Vm, const double *Vp, double Fs[6],
                            double *speed)
{
    const double tiny = 1.e-32;
    const double aL2 = Vm[H_GC] * Vm[H_P] / Vm[H_D];
    const double aR2 = Vp[H_GC] * Vp[H_P] / Vp[H_D];
    if ((Vm[H_D] < tiny && Vm[H_D] > 0.) || (Vp[H_D] < tiny && Vp[H_D] > 0.) ||
        (Vm[H_P] < tiny && Vm[H_P] > 0.) || (Vp[H_P] < tiny && Vp[H_P] > 0.)) {
        for (int k = 0; k < 6; k++) Fs[k] = 0.;
        *speed = 0.;
        return 0;
    } else if (aL2 < 0. || aR2 < 0.) {
        return 1;
    }
    if (aL2 <= 0. || aR2 <= 0.) return 1;      /* hy_eigenParameters aborts */
    const double cL = sqrt(aL2), cR = sqrt(aR2);
    double lamL[5], lamR[5], LL[5][5], RL[5][5], LR[5][5], RR[5][5];
    eigen_values(Vm[H_VX + dir], cL, lamL);
    cons_eigen(Vm, dir, cL, LL, RL);
    eigen_values(Vp[H_VX + dir], cR, lamR);
    cons_eigen(Vp, dir, cR, LR, RR);
    double UL[5], UR[5], FL[6], FR[6];
    prim2con(Vm, UL); prim2con(Vp, UR);
    prim2flx(p, dir, Vm, FL); prim2flx(p, dir, Vp, FR);
    *speed = fmax2(fabs(lamL[4]), fabs(lamR[4]));
    double mL = fabs(lamL[0]), mR = fabs(lamR[0]);
    for (int k = 1; k < 5; k++) {
        if (fabs(lamL[k]) > mL) mL = fabs(lamL[k]);
        if (fabs(lamR[k]) > mR) mR = fabs(lamR[k]);
    }
    const double amax = fmax2(mL, mR);
    const int mom = 1 + dir;
    double vecL[5], vecR[5];
    for (int k = 0; k < 5; k++) {
        double lf = 0., lu = 0., rf = 0., ru = 0.;   /* dot_product(leig(k, 1:5), .) */
        for (int j = 0; j < 5; j++) {
            lf = lf + LL[k][j] * FL[j]; lu = lu + LL[k][j] * UL[j];
            rf = rf + LR[k][j] * FR[j]; ru = ru + LR[k][j] * UR[j];
        }
        if (lamL[k] * lamR[k] > 0.) {
            if (lamL[k] > 0.) {
                vecL[k] = lf + LL[k][mom] * FL[F_P];
                vecR[k] = 0.;
            } else {
                vecL[k] = 0.;
                vecR[k] = rf + LR[k][mom] * FR[F_P];
            }
        } else {
            vecL[k] = 0.5 * (lf + amax * lu + LL[k][mom] * FL[F_P]);
            vecR[k] = 0.5 * (rf - amax * ru + LR[k][mom] * FR[F_P]);
        }
    }
    for (int v = 0; v < 5; v++) {
        double fl = vecL[0] * RL[v][0], fr = vecR[0] * RR[v][0];
        for (int w = 1; w < 5; w++) {
            fl = fl + vecL[w] * RL[v][w];
            fr = fr + vecR[w] * RR[v][w];
        }
        Fs[v] = fl + fr;
    }
    Fs[F_P] = 0.0;
    return 0;
}

/* hy_MarquinaModified.F90:52-195 (hydro): per wave k the mean of the two
 * states' |eigenvalues| times the jump of the wave's conserved part,
 * r_R (l_R . U_R) - r_L (l_L . U_L), subtracted from the sum of the two
 * fluxes and halved; the wave speed reported is |u| + c of the right state
 * (the last hy_eigenParameters call). */
static int riemann_marquina_mod(const fxo_params *p, int dir, const double *Vm, const double *Vp, double Fs[6],
                                double *speed)
{
    const double tiny = 1.e-32;
    const double aL2 = Vm[H_GC] * Vm[H_P] / Vm[H_D];
    const double aR2 = Vp[H_GC] * Vp[H_P] / Vp[H_D];
    if ((Vm[H_D] < tiny && Vm[H_D] > 0.) || (Vp[H_D] < tiny && Vp[H_D] > 0.) ||
        (Vm[H_P] < tiny && Vm[H_P] > 0.) || (Vp[H_P] < tiny && Vp[H_P] > 0.)) {
        for (int k = 0; k < 6; k++) Fs[k] = 0.;
        *speed = 0.;
        return 0;
    } else if (aL2 < 0. || aR2 < 0.) {
        return 1;
    }
    if (aL2 <= 0. || aR2 <= 0.) return 1;      /* hy_eigenParameters aborts */
    const double cL = sqrt(aL2), cR = sqrt(aR2);
    double lamL[5], lamR[5], LL[5][5], RL[5][5], LR[5][5], RR[5][5];
    eigen_values(Vm[H_VX + dir], cL, lamL);
    cons_eigen(Vm, dir, cL, LL, RL);
    eigen_values(Vp[H_VX + dir], cR, lamR);
    cons_eigen(Vp, dir, cR, LR, RR);
    double UL[5], UR[5], FL[6], FR[6];
    prim2con(Vm, UL); prim2con(Vp, UR);
    prim2flx(p, dir, Vm, FL); prim2flx(p, dir, Vp, FR);
    *speed = fabs(Vp[H_VX + dir]) + fabs(cR);
    double sigF[6] = {0., 0., 0., 0., 0., 0.};
    for (int k = 0; k < 5; k++) {
        double dR = 0., dL = 0.;
        for (int v = 0; v < 5; v++) { dR = dR + LR[v][k] * UR[v]; dL = dL + LL[v][k] * UL[v]; }
        const double c = 0.5 * (fabs(lamL[k]) + fabs(lamR[k]));
        for (int v = 0; v < 5; v++) sigF[v] = sigF[v] + c * (RR[v][k] * dR - RL[v][k] * dL);
    }
    for (int v = 0; v < 6; v++) Fs[v] = (FR[v] + FL[v] - sigF[v]) * 0.5;
    return 0;
}

/* hy_shockDetectBlk.F90 on one block: SHOK = 0 over the whole block, then
 * 1 in every interior cell where the pressure jump |grad p| (central
 * differences, summed over the axes) reaches half the smallest pressure of
 * the cell's 3^d box and the velocity divergence is below -0.1 times the
 * smallest sound speed of that box (beta = 0.5, delta = 0.1). */
static void shock_detect_block(const blk_t *b, double *U)
{
    const fxo_params *p = b->p;
    const int k2 = p->ndim > 1, k3 = p->ndim > 2;
#define UV(var, ii, jj, kk) U[cidx(b, ii, jj, kk) * FXO_NUNK + (var)]
    for (long c = 0; c < b->ncell; c++) U[c * FXO_NUNK + FXO_SHOK] = 0.;
    const double beta = 0.5, delta = 0.1;
    for (int k = b->k0; k <= b->kmax; k++)
    for (int j = b->j0; j <= b->jmax; j++)
    for (int i = b->i0; i <= b->imax; i++) {
        double minP = 0., minC = 0.;
        int first = 1;
        for (int kk = k - k3; kk <= k + k3; kk++)
        for (int jj = j - k2; jj <= j + k2; jj++)
        for (int ii = i - 1; ii <= i + 1; ii++) {
            const double pr = UV(FXO_PRES, ii, jj, kk);
            const double cs = sqrt(UV(FXO_GAMC, ii, jj, kk) * UV(FXO_PRES, ii, jj, kk) / UV(FXO_DENS, ii, jj, kk));
            if (first || pr < minP) minP = pr;
            if (first || cs < minC) minC = cs;
            first = 0;
        }
        double divv = UV(FXO_VELX, i + 1, j, k) - UV(FXO_VELX, i - 1, j, k);
        if (p->ndim > 1) divv = divv + UV(FXO_VELY, i, j + 1, k) - UV(FXO_VELY, i, j - 1, k);
        if (p->ndim > 2) divv = divv + UV(FXO_VELZ, i, j, k + 1) - UV(FXO_VELZ, i, j, k - 1);
        divv = 0.5 * divv;
        const double gx = 0.5 * (UV(FXO_PRES, i + 1, j, k) - UV(FXO_PRES, i - 1, j, k));
        double gy = 0., gz = 0.;
        if (p->ndim > 1) gy = 0.5 * (UV(FXO_PRES, i, j + 1, k) - UV(FXO_PRES, i, j - 1, k));
        if (p->ndim > 2) gz = 0.5 * (UV(FXO_PRES, i, j, k + 1) - UV(FXO_PRES, i, j, k - 1));
        const int sw1 = fabs(gx) + fabs(gy) + fabs(gz) >= beta * minP;
        const int sw2 = -delta * minC >= divv;
        if (sw1 && sw2) UV(FXO_SHOK, i, j, k) = 1.;
    }
#undef UV
}

/* the Riemann solver of the runtime parameter RiemannSolver */
static int riemann_solve(const fxo_params *p, int dir, const double *Vm, const double *Vp, double Fs[6], double *speed)
{
    if (p->riemann == FXO_HLL) return riemann_hll(p, dir, Vm, Vp, Fs, speed);
    if (p->riemann == FXO_LLF) return riemann_llf(p, dir, Vm, Vp, Fs, speed);
    if (p->riemann == FXO_ROE) return riemann_roe(p, dir, Vm, Vp, Fs, speed);
    if (p->riemann == FXO_MARQ) return riemann_marquina(p, dir, Vm, Vp, Fs, speed);
    if (p->riemann == FXO_MARM) return riemann_marquina_mod(p, dir, Vm, Vp, Fs, speed);
    return riemann_hllc(p, dir, Vm, Vp, Fs, speed);
}

/* ======================================================================= */
/* Per-block hy_computeFluxes with in-place update (Uout => Uin).          */
/* ======================================================================= */
typedef struct {
    double *scr[3];     /* scrchFace{X,Y,Z}: [cell][16]: P01..P08 then N01..N08 */
    double *flx[3];     /* fluxes: [cell][8] at face (i-1/2) etc. */
    double *sig;        /* [cell][3][9] */
    double *lam;        /* [cell][3][5] */
    double *leig;       /* [cell][3][5][5] */
    double *reig;       /* [cell][3][5][5] */
    double *pav;        /* VAR1 averaged pressure [cell] */
    double *flat;       /* flattening: FlatTilde [3][cell], then FlatCoeff [3][cell] */
    double *divu;       /* hybrid order: undivided velocity divergence [cell] */
    unsigned char *ctufb;   /* 3-D CTU: 1 where the face states of (cell, dir) fell back to first order */
} scratch_t;

static void scratch_alloc(scratch_t *s, long ncell)
{
    for (int d = 0; d < 3; d++) {
        s->scr[d] = (double *)calloc((size_t)ncell * 16, sizeof(double));
        s->flx[d] = (double *)calloc((size_t)ncell * 8, sizeof(double));
    }
    s->sig = (double *)calloc((size_t)ncell * 27, sizeof(double));
    s->lam = (double *)calloc((size_t)ncell * 15, sizeof(double));
    s->leig = (double *)calloc((size_t)ncell * 75, sizeof(double));
    s->reig = (double *)calloc((size_t)ncell * 75, sizeof(double));
    s->pav = (double *)calloc((size_t)ncell, sizeof(double));
    s->flat = (double *)calloc((size_t)ncell * 6, sizeof(double));
    s->divu = (double *)calloc((size_t)ncell, sizeof(double));
    s->ctufb = (unsigned char *)calloc((size_t)ncell * 3, 1);
}
static void scratch_free(scratch_t *s)
{
    for (int d = 0; d < 3; d++) { free(s->scr[d]); free(s->flx[d]); }
    free(s->sig); free(s->lam); free(s->leig); free(s->reig); free(s->pav); free(s->flat); free(s->divu); free(s->ctufb);
}

static void blk_init(blk_t *b, const fxo_params *p)
{
    b->p = p;
    b->ng = p->nguard;
    b->k2 = p->ndim >= 2; b->k3 = p->ndim == 3;
    b->nig = p->nxb + 2 * b->ng;
    b->njg = b->k2 ? p->nyb + 2 * b->ng : 1;
    b->nkg = b->k3 ? p->nzb + 2 * b->ng : 1;
    b->i0 = b->ng; b->imax = b->ng + p->nxb - 1;
    b->j0 = b->k2 ? b->ng : 0; b->jmax = b->k2 ? b->ng + p->nyb - 1 : 0;
    b->k0 = b->k3 ? b->ng : 0; b->kmax = b->k3 ? b->ng + p->nzb - 1 : 0;
    b->dx = (p->xmax - p->xmin) / (double)(p->nxb * p->nblockx);
    b->dy = b->k2 ? (p->ymax - p->ymin) / (double)(p->nyb * p->nblocky) : 1.;
    b->dz = b->k3 ? (p->zmax - p->zmin) / (double)(p->nzb * p->nblockz) : 1.;
    b->ncell = (long)b->nig * b->njg * b->nkg;
}

/* hy_getRiemannState.F90:482-912 and 963-1338 for one block. */
static int riemann_states(const blk_t *b, const double *U, double dt, scratch_t *s)
{
    const fxo_params *p = b->p;
    const int ndim = p->ndim;
    const double del[3] = {b->dx, b->dy, b->dz};
    const double hdt = 0.5 * dt;
    const double hdtx = 0.5 * dt / b->dx, hdty = 0.5 * dt / b->dy, hdtz = 0.5 * dt / b->dz;
    const int nev = n_end_vars(p);
    const int klo = b->k3 ? b->k0 - 1 : 0, khi = b->k3 ? b->kmax + 1 : 0;
    const int jlo = b->k2 ? b->j0 - 1 : 0, jhi = b->k2 ? b->jmax + 1 : 0;
    double *FT = s->flat, *FC = s->flat + 3 * b->ncell;
    /* hybrid order: DivU = (u(i+1) - u(i-1) + v(j+1) - v(j-1) + w(k+1) - w(k-1)) / 2 on
     * [lo - 1 - k4, hi + 1 + k4] (hy_getRiemannState.F90:322-361, kHydro = 1) */
    const int k4 = p->order - 1 > 2 ? 2 : p->order - 1;
    if (p->use_hybrid) {
        const int hk0 = b->k3 ? b->k0 - 1 - k4 : 0, hk1 = b->k3 ? b->kmax + 1 + k4 : 0;
        const int hj0 = b->k2 ? b->j0 - 1 - k4 : 0, hj1 = b->k2 ? b->jmax + 1 + k4 : 0;
        for (int k = hk0; k <= hk1; k++)
        for (int j = hj0; j <= hj1; j++)
        for (int i = b->i0 - 1 - k4; i <= b->imax + 1 + k4; i++) {
            double dv = U[cidx(b, i + 1, j, k) * FXO_NUNK + FXO_VELX] - U[cidx(b, i - 1, j, k) * FXO_NUNK + FXO_VELX];
            if (ndim > 1) {
                dv = dv + U[cidx(b, i, j + 1, k) * FXO_NUNK + FXO_VELY] - U[cidx(b, i, j - 1, k) * FXO_NUNK + FXO_VELY];
                if (ndim > 2)
                    dv = dv + U[cidx(b, i, j, k + 1) * FXO_NUNK + FXO_VELZ] - U[cidx(b, i, j, k - 1) * FXO_NUNK + FXO_VELZ];
            }
            s->divu[cidx(b, i, j, k)] = 0.5 * dv;
        }
    }
    if (p->flattening) {
        /* hy_getRiemannState.F90:367-465: FlatTilde on [lo-2, hi+2] (zero
         * elsewhere), then FlatCoeff on the same range (kHydro = 0) */
        memset(s->flat, 0, sizeof(double) * 6 * b->ncell);
        const int fk0 = b->k3 ? b->k0 - 2 : 0, fk1 = b->k3 ? b->kmax + 2 : 0;
        const int fj0 = b->k2 ? b->j0 - 2 : 0, fj1 = b->k2 ? b->jmax + 2 : 0;
        for (int k = fk0; k <= fk1; k++)
        for (int j = fj0; j <= fj1; j++)
        for (int i = b->i0 - 2; i <= b->imax + 2; i++)
            for (int d = 0; d < ndim; d++) {
                int di = d == 0, dj = d == 1, dk = d == 2;
                const double *um2 = U + cidx(b, i - 2 * di, j - 2 * dj, k - 2 * dk) * FXO_NUNK;
                const double *um1 = U + cidx(b, i - di, j - dj, k - dk) * FXO_NUNK;
                const double *up1 = U + cidx(b, i + di, j + dj, k + dk) * FXO_NUNK;
                const double *up2 = U + cidx(b, i + 2 * di, j + 2 * dj, k + 2 * dk) * FXO_NUNK;
                double dp1 = (up1[FXO_PRES] - um1[FXO_PRES]);
                double dp2 = (up2[FXO_PRES] - um2[FXO_PRES]);
                double dv1 = up1[FXO_VELX + d] - um1[FXO_VELX + d];
                double presL = um1[FXO_PRES], presR = up1[FXO_PRES];
                double Sp = (fabs(dp2) > 1.e-15) ? dp1 / dp2 - 0.75 : 0.;
                double ft = fmax2(0.0, fmin2(1.0, 10.0 * Sp));
                if ((fabs(dp1) / fmin2(presL, presR) < 1. / 3.) || dv1 > 0.) ft = 0.;
                FT[d * b->ncell + cidx(b, i, j, k)] = ft;
            }
        for (int k = fk0; k <= fk1; k++)
        for (int j = fj0; j <= fj1; j++)
        for (int i = b->i0 - 2; i <= b->imax + 2; i++)
            for (int d = 0; d < ndim; d++) {
                int di = d == 0, dj = d == 1, dk = d == 2;
                long c = cidx(b, i, j, k);
                double dp1 = (U[cidx(b, i + di, j + dj, k + dk) * FXO_NUNK + FXO_PRES] -
                              U[cidx(b, i - di, j - dj, k - dk) * FXO_NUNK + FXO_PRES]);
                double f0 = FT[d * b->ncell + c];
                /* FlatTilde beyond the computed range is zero */
                int ip = i + di, jp = j + dj, kp = k + dk, im = i - di, jm = j - dj, km = k - dk;
                int inP = ip <= b->imax + 2 && jp <= fj1 && kp <= fk1;
                int inM = im >= b->i0 - 2 && jm >= fj0 && km >= fk0;
                double fP = inP ? FT[d * b->ncell + cidx(b, ip, jp, kp)] : 0.;
                double fM = inM ? FT[d * b->ncell + cidx(b, im, jm, km)] : 0.;
                double fc;
                if (dp1 < 0.0) fc = fmax2(f0, fP);
                else if (dp1 == 0.) fc = f0;
                else fc = fmax2(f0, fM);
                FC[d * b->ncell + c] = fc;
            }
    }
    for (int k = klo; k <= khi; k++)
    for (int j = jlo; j <= jhi; j++)
    for (int i = b->i0 - 1; i <= b->imax + 1; i++) {
        long c = cidx(b, i, j, k);
        int tr[3] = {0, 0, 0};
        if (i > b->imax + 1 || i < b->i0 - 1) tr[0] = 1;
        if (i > b->imax || i < b->i0) { tr[1] = 1; tr[2] = 1; }
        if (ndim > 1) {
            if (j > b->jmax + 1 || j < b->j0 - 1) tr[1] = 1;
            if (j > b->jmax || j < b->j0) { tr[0] = 1; tr[2] = 1; }
            if (ndim > 2) {
                if (k > b->kmax + 1 || k < b->k0 - 1) tr[2] = 1;
                if (k > b->kmax || k < b->k0) { tr[0] = 1; tr[1] = 1; }
            }
        }
        double Wp[3][H_NV], Wn[3][H_NV];
        double *sig = s->sig + c * 27;
        double *lam = s->lam + c * 15;
        double (*leig)[5][5] = (double (*)[5][5])(s->leig + c * 75);
        double (*reig)[5][5] = (double (*)[5][5])(s->reig + c * 75);
        /* hy_dataReconstOneStep: per-direction reconstruction */
        for (int d = 0; d < ndim; d++) {
            int ko = tr[d] ? 1 : 2;
            double V[5][H_NV];
            const double *S[5] = {NULL, NULL, NULL, NULL, NULL};
            for (int o = -ko; o <= ko; o++) {
                int ii = i + (d == 0 ? o : 0), jj = j + (d == 1 ? o : 0), kk = k + (d == 2 ? o : 0);
                load_v(p, U + cidx(b, ii, jj, kk) * FXO_NUNK, p->grav[d], V[o + 2]);
                S[o + 2] = V[o + 2];
            }
            double flat = p->flattening ? FC[d * b->ncell + c] : 0.;
            int err = (p->order == 5)
                ? recon_weno(p, d, dt, del[d], S, tr[d], flat, lam + 5 * d, leig[d], reig[d], Wp[d], Wn[d], sig + 9 * d)
                : (p->order == 2)
                ? recon_mh(p, d, dt, del[d], S, tr[d], flat, lam + 5 * d, leig[d], reig[d], Wp[d], Wn[d], sig + 9 * d)
                : recon_ppm(p, d, dt, del[d], S, tr[d], flat, lam + 5 * d, leig[d], reig[d], Wp[d], Wn[d], sig + 9 * d);
            if (err) return 1;
        }
        /* hybrid order, hy_dataReconstOneStep.F90:864-913: where the velocity
         * converges (min of DivU over the cell's (2 k4 + 1)^d box below kappa
         * times the sound speed), a face state that breaks the density bounds
         * of a shock (hy_checkRHjumpCond) falls back to first order */
        if (p->use_hybrid) {
            const double *u = U + c * FXO_NUNK;
            double cs = u[FXO_GAMC] * u[FXO_PRES];
            cs = sqrt(cs / u[FXO_DENS]);
            const double eps = p->hybrid_kappa * cs;
            double mn = 0.;
            int first = 1;
            for (int kk = k - k4 * b->k3; kk <= k + k4 * b->k3; kk++)
            for (int jj = j - k4 * b->k2; jj <= j + k4 * b->k2; jj++)
            for (int ii = i - k4; ii <= i + k4; ii++) {
                double v = s->divu[cidx(b, ii, jj, kk)];
                if (first || v < mn) mn = v;
                first = 0;
            }
            if (mn < eps) {
                const double gamc = u[FXO_GAMC], dens = u[FXO_DENS];
                const double gr = (gamc + 1.) / (gamc - 1.);
                double m2 = 0.;
                for (int e = 0; e < ndim; e++) m2 = m2 + u[FXO_VELX + e] * u[FXO_VELX + e];
                m2 = m2 * dens / (gamc * u[FXO_PRES]);
                for (int d = 0; d < ndim; d++) {
                    int sw = 0;
                    if (m2 > 1.e-4) {
                        if (Wn[d][H_D] > gr * dens || gr * Wn[d][H_D] < dens) sw = 1;
                        if (Wp[d][H_D] > gr * dens || gr * Wp[d][H_D] < dens) sw = 1;
                    }
                    if (sw) {
                        Wp[d][H_D] = dens; Wp[d][H_VX] = u[FXO_VELX]; Wp[d][H_VY] = u[FXO_VELY];
                        Wp[d][H_VZ] = u[FXO_VELZ]; Wp[d][H_P] = u[FXO_PRES]; Wp[d][H_GC] = gamc;
                        Wp[d][H_GE] = u[FXO_GAME]; Wp[d][H_EI] = u[FXO_EINT];
                        for (int v = H_D; v <= H_EI; v++) Wn[d][v] = Wp[d][v];
                    }
                }
            }
        }
        /* transverse contributions, hy_dataReconstOneStep.F90:931-962 */
        if (ndim > 1) {
            for (int v = 0; v < nev; v++) {
                Wn[0][v] = Wn[0][v] - hdty * sig[9 + v];
                Wp[0][v] = Wp[0][v] - hdty * sig[9 + v];
                Wn[1][v] = Wn[1][v] - hdtx * sig[v];
                Wp[1][v] = Wp[1][v] - hdtx * sig[v];
            }
            if (ndim > 2) {
                for (int v = 0; v < nev; v++) {
                    Wn[0][v] = Wn[0][v] - hdtz * sig[18 + v];
                    Wp[0][v] = Wp[0][v] - hdtz * sig[18 + v];
                    Wn[1][v] = Wn[1][v] - hdtz * sig[18 + v];
                    Wp[1][v] = Wp[1][v] - hdtz * sig[18 + v];
                    Wn[2][v] = Wn[2][v] - hdtx * sig[v] - hdty * sig[9 + v];
                    Wp[2][v] = Wp[2][v] - hdtx * sig[v] - hdty * sig[9 + v];
                }
            }
        }
        /* last negativity check, hy_dataReconstOneStep.F90:1131-1165 */
        for (int d = 0; d < ndim; d++) {
            if (Wn[d][H_D] < 0. || Wp[d][H_D] < 0. || Wn[d][H_P] < 0. || Wp[d][H_P] < 0.) {
                double Vc[H_NV];
                load_v(p, U + c * FXO_NUNK, p->grav[d], Vc);
                for (int v = 0; v < H_GR; v++) { Wn[d][v] = Vc[v]; Wp[d][v] = Vc[v]; }
            }
        }
        /* gravity half update and storage, hy_getRiemannState.F90:843-891 */
        for (int d = 0; d < ndim; d++) {
            if (p->use_gravity) {
                for (int e = 0; e < 3; e++) {
                    double gp = (e == d) ? Wp[d][H_GR] : p->grav[e];
                    double gn = (e == d) ? Wn[d][H_GR] : p->grav[e];
                    Wp[d][H_VX + e] = Wp[d][H_VX + e] + hdt * gp;
                    Wn[d][H_VX + e] = Wn[d][H_VX + e] + hdt * gn;
                }
            }
            if (!tr[d]) {
                double *sc = s->scr[d] + c * 16;
                for (int v = 0; v < 8; v++) { sc[v] = Wp[d][v]; sc[8 + v] = Wn[d][v]; }
            }
        }
    }

    /* 3-D full CTU corner coupling, hy_getRiemannState.F90:963-1338 */
    if (ndim == 3 && p->use_3d_full_ctu) {
        const double dt2dxdy6 = dt * dt / (6. * b->dx * b->dy);
        const double dt2dydz6 = dt * dt / (6. * b->dy * b->dz);
        const double dt2dzdx6 = dt * dt / (6. * b->dz * b->dx);
        for (int k = b->k0 - 2; k <= b->kmax + 2; k++)
        for (int j = b->j0 - 2; j <= b->jmax + 2; j++)
        for (int i = b->i0 - 2; i <= b->imax + 2; i++) {
            long c = cidx(b, i, j, k);
            double Vc[H_NV];
            load_v(p, U + c * FXO_NUNK, 0., Vc);
            /* pairs: (face dir, first transverse dir a with sig of dir sa, second b with sig sb) */
            for (int fd = 0; fd < 3; fd++) {
                int ii[3] = {i, j, k}, lo[3] = {b->i0, b->j0, b->k0}, hi[3] = {b->imax, b->jmax, b->kmax};
                int ok = 1;
                for (int e = 0; e < 3; e++) {
                    if (e == fd) { if (ii[e] < lo[e] - 1 || ii[e] > hi[e] + 1) ok = 0; }
                    else if (ii[e] < lo[e] || ii[e] > hi[e]) ok = 0;
                }
                if (!ok) continue;
                /* X: TransFluxYZ (sig Z along y, eig Y) + TransFluxZY (sig Y along z, eig Z), factor dt2dydz6
                 * Y: TransFluxZX (sig X along z, eig Z) + TransFluxXZ (sig Z along x, eig X), factor dt2dzdx6
                 * Z: TransFluxXY (sig Y along x, eig X) + TransFluxYX (sig X along y, eig Y), factor dt2dxdy6 */
                int e1, s1, e2, s2; double fac;
                if (fd == 0)      { e1 = 1; s1 = 2; e2 = 2; s2 = 1; fac = dt2dydz6; }
                else if (fd == 1) { e1 = 2; s1 = 0; e2 = 0; s2 = 2; fac = dt2dzdx6; }
                else              { e1 = 0; s1 = 1; e2 = 1; s2 = 0; fac = dt2dxdy6; }
                double T1[H_NV], T2[H_NV];
                int es[2] = {e1, e2}, ss[2] = {s1, s2};
                double *T[2] = {T1, T2};
                for (int q = 0; q < 2; q++) {
                    int e = es[q], sd = ss[q];
                    int im = i - (e == 0), jm = j - (e == 1), km = k - (e == 2);
                    int ip = i + (e == 0), jp = j + (e == 1), kp = k + (e == 2);
                    const double *sm = s->sig + cidx(b, im, jm, km) * 27 + 9 * sd;
                    const double *sc = s->sig + c * 27 + 9 * sd;
                    const double *sp = s->sig + cidx(b, ip, jp, kp) * 27 + 9 * sd;
                    double (*le)[5][5] = (double (*)[5][5])(s->leig + c * 75);
                    double (*re)[5][5] = (double (*)[5][5])(s->reig + c * 75);
                    upwind_trans(p, sm, sc, sp, s->lam + c * 15 + 5 * e, le[e], re[e], nev, T[q]);
                }
                double *scr = s->scr[fd] + c * 16;
                for (int v = 0; v < 8; v++) {
                    scr[v] = scr[v] + (T1[v] + T2[v]) * fac;
                    scr[8 + v] = scr[8 + v] + (T1[v] + T2[v]) * fac;
                }
                s->ctufb[c * 3 + fd] = 0;
                if (scr[0] <= 0. || scr[8] <= 0. || scr[4] <= 0. || scr[12] <= 0.) {
                    for (int v = 0; v < 8; v++) { scr[v] = Vc[v]; scr[8 + v] = Vc[v]; }
                    s->ctufb[c * 3 + fd] = 1;
                }
            }
        }
    }
    return 0;
}

/* Artificial viscosity of one face (hy_getFaceFlux.F90:397-438 x, 700-745 y,
 * 955-990 z; Colella and Woodward 1984): cvisc times the negative part of the
 * undivided velocity divergence at the face (the normal difference plus the
 * quarter-weighted transverse central differences of both cells, scaled by
 * the cell-width ratios), times the jump of the conserved dens, momenta and
 * total energy from the cell behind the face to the cell ahead. */
static void avisc_face(const blk_t *b, const double *U, int d, int i, int j, int k, double fl[8])
{
    const fxo_params *p = b->p;
    const int ndim = p->ndim;
    const double del[3] = {b->dx, b->dy, b->dz};
#define UV(var, ii, jj, kk) U[cidx(b, ii, jj, kk) * FXO_NUNK + (var)]
    const int it = d == 0, jt = d == 1, kt = d == 2;
    const int im = i - it, jm = j - jt, km = k - kt;
    /* quarter-weighted central difference of velocity e across axis e, in both cells */
    double tr[3] = {0., 0., 0.};
    for (int e = 0; e < ndim; e++) {
        if (e == d) continue;
        const int ie = e == 0, je = e == 1, ke = e == 2;
        const int v = FXO_VELX + e;
        tr[e] = 0.25 * (UV(v, i + ie, j + je, k + ke) - UV(v, i - ie, j - je, k - ke) +
                        UV(v, im + ie, jm + je, km + ke) - UV(v, im - ie, jm - je, km - ke)) * del[d] / del[e];
    }
    const int vn = FXO_VELX + d;
    const double nd = UV(vn, i, j, k), ndm = UV(vn, im, jm, km);
    double div;
    if (d == 0) {
        div = nd - ndm;
        if (ndim > 1) div = div + tr[1];
        if (ndim > 2) div = div + tr[2];
    } else if (d == 1) {
        div = tr[0] + nd - ndm;
        if (ndim > 2) div = div + tr[2];
    } else {
        div = tr[0] + tr[1] + nd - ndm;
    }
    const double cv = p->cvisc * fmax2(-(div), 0.);
    const double dl = UV(FXO_DENS, im, jm, km), dr = UV(FXO_DENS, i, j, k);
    fl[F_D] = fl[F_D] + cv * (dl - dr);
    fl[F_MX] = fl[F_MX] + cv * (dl * UV(FXO_VELX, im, jm, km) - dr * UV(FXO_VELX, i, j, k));
    fl[F_MY] = fl[F_MY] + cv * (dl * UV(FXO_VELY, im, jm, km) - dr * UV(FXO_VELY, i, j, k));
    fl[F_MZ] = fl[F_MZ] + cv * (dl * UV(FXO_VELZ, im, jm, km) - dr * UV(FXO_VELZ, i, j, k));
    fl[F_E] = fl[F_E] + cv * (dl * UV(FXO_ENER, im, jm, km) - dr * UV(FXO_ENER, i, j, k));
#undef UV
}

/* hy_getFaceFlux.F90:300-572 (+y, z) for one block. */
static int face_fluxes(const blk_t *b, const double *U, scratch_t *s)
{
    const fxo_params *p = b->p;
    const int ndim = p->ndim;
    for (int d = 0; d < ndim; d++) {
        int kt = (d == 2), jt = (d == 1), it = (d == 0);
        for (int k = b->k0; k <= b->kmax + kt; k++)
        for (int j = b->j0; j <= b->jmax + jt; j++)
        for (int i = b->i0; i <= b->imax + it; i++) {
            long c = cidx(b, i, j, k);
            long cm = cidx(b, i - it, j - jt, k - kt);
            double VL[H_NV], VR[H_NV];
            for (int v = 0; v < 8; v++) { VL[v] = s->scr[d][cm * 16 + v]; VR[v] = s->scr[d][c * 16 + 8 + v]; }
            VL[H_GR] = 0.; VR[H_GR] = 0.;
            double F[6], speed;
            int err;
            if (p->riemann == FXO_HYBR)     /* hy_getFaceFlux.F90:364-383: HLL next to a shocked cell */
                err = U[cm * FXO_NUNK + FXO_SHOK] + U[c * FXO_NUNK + FXO_SHOK] > 0.
                    ? riemann_hll(p, d, VL, VR, F, &speed) : riemann_hllc(p, d, VL, VR, F, &speed);
            else
                err = riemann_solve(p, d, VL, VR, F, &speed);
            if (err) return 2;
            double *fl = s->flx[d] + c * 8;
            for (int v = 0; v < 6; v++) fl[v] = F[v];
            if (p->use_avisc) avisc_face(b, U, d, i, j, k, fl);
            if (p->use_aux_eint) {
                if (fl[F_D] > 0.) { fl[F_VOL] = fl[F_D] / VL[H_D]; fl[F_EI] = fl[F_D] * VL[H_EI]; }
                else              { fl[F_VOL] = fl[F_D] / VR[H_D]; fl[F_EI] = fl[F_D] * VR[H_EI]; }
            } else { fl[F_VOL] = 0.; fl[F_EI] = 0.; }
        }
        /* cell-averaged n+1/2 pressure for the aux eint update */
        if (p->use_aux_eint) {
            for (int k = b->k0; k <= b->kmax; k++)
            for (int j = b->j0; j <= b->jmax; j++)
            for (int i = b->i0; i <= b->imax; i++) {
                long c = cidx(b, i, j, k);
                double sum = s->scr[d][c * 16 + 8 + 4] + s->scr[d][c * 16 + 4];   /* N05 + P05 */
                if (d == 0) s->pav[c] = 0.5 * sum;
                else if (d == 1) s->pav[c] = s->pav[c] * 0.5 + sum * 0.25;
                else s->pav[c] = (s->pav[c] * 4.0 + sum) / 6.0;
            }
        }
    }
    return 0;
}

/* hy_unsplitUpdate.F90:392-933 + helpers :1195-1306 (Cartesian, UPDATE_ALL). */
static void unsplit_update(const blk_t *b, double *U, double dt, scratch_t *s)
{
    const fxo_params *p = b->p;
    const int ndim = p->ndim;
    const double fP = p->fpres;
    double dl[3] = {b->dx, b->dy, b->dz};
    for (int k = b->k0; k <= b->kmax; k++)
    for (int j = b->j0; j <= b->jmax; j++)
    for (int i = b->i0; i <= b->imax; i++) {
        long c = cidx(b, i, j, k);
        double *u = U + c * FXO_NUNK;
        double FLd[3][8], FRd[3][8];
        for (int d = 0; d < 3; d++) {
            if (d < ndim) {
                long cp = cidx(b, i + (d == 0), j + (d == 1), k + (d == 2));
                for (int v = 0; v < 8; v++) { FLd[d][v] = s->flx[d][c * 8 + v]; FRd[d][v] = s->flx[d][cp * 8 + v]; }
            } else {
                for (int v = 0; v < 8; v++) { FLd[d][v] = 0.; FRd[d][v] = 0.; }
            }
        }
        double Sphys[5] = {0., 0., 0., 0., 0.};
        Sphys[1] = (FLd[0][F_P] - FRd[0][F_P]) * (1.0 - fP) / dl[0];
        if (ndim >= 2) Sphys[2] = (FLd[1][F_P] - FRd[1][F_P]) * (1.0 - fP) / dl[1];
        if (ndim == 3) Sphys[3] = (FLd[2][F_P] - FRd[2][F_P]) * (1.0 - fP) / dl[2];
        double U0[5];
        U0[0] = u[FXO_DENS];
        double IntEner = 0.;
        if (p->use_aux_eint) {
            IntEner = u[FXO_DENS] * u[FXO_EINT];
            double pres = s->pav[c];
            for (int d = 0; d < ndim; d++)
                IntEner = IntEner + dt / dl[d] * (FLd[d][F_EI] - FRd[d][F_EI] + pres * (FLd[d][F_VOL] - FRd[d][F_VOL]));
            IntEner = IntEner + dt * 0.0;
        }
        U0[1] = u[FXO_VELX] * u[FXO_DENS];
        U0[2] = u[FXO_VELY] * u[FXO_DENS];
        U0[3] = u[FXO_VELZ] * u[FXO_DENS];
        U0[4] = u[FXO_DENS] * u[FXO_ENER];
        /* updateConservedVariable */
        double densOld = U0[0], momOld[3] = {U0[1], U0[2], U0[3]};
        for (int d = 0; d < ndim; d++)
            for (int v = 0; v < 5; v++) U0[v] = U0[v] - dt / dl[d] * (FRd[d][v] - FLd[d][v]);
        for (int v = 0; v < 5; v++) U0[v] = U0[v] + dt * (0. + Sphys[v]);
        if (p->use_gravity) {
            for (int d = 0; d < 3; d++) U0[1 + d] = U0[1 + d] + 0.5 * dt * densOld * p->grav[d];
            double dp = 0.; for (int d = 0; d < 3; d++) dp = dp + momOld[d] * p->grav[d];
            U0[4] = U0[4] + 0.5 * dt * dp;
        }
        u[FXO_DENS] = fmax2(U0[0], p->small_dens);
        u[FXO_ENER] = U0[4];
        u[FXO_VELX] = U0[1] / u[FXO_DENS];
        u[FXO_VELY] = U0[2] / u[FXO_DENS];
        u[FXO_VELZ] = U0[3] / u[FXO_DENS];
        u[FXO_ENER] = U0[4] / u[FXO_DENS];
        if (p->use_aux_eint) u[FXO_EINT] = IntEner / u[FXO_DENS];
    }
}

/* hy_energyFix.F90:240-260 on the block interior. */
/* hy_gravityStep -> hy_gravityStepBlk.F90:54-78 -> hy_addGravity for constant
 * gravity: the n+1 half step v += dt/2 g, E += dt/2 v.g on the interior of one
 * block.  With gravity, energyFix and Eos come after it (hy_updateSolution.F90
 * defers them under GRAVITY), on uniform grids and AMR meshes alike. */
static void gravity_step_block(const blk_t *b, double *U, double dt)
{
    const fxo_params *p = b->p;
    for (int k = b->k0; k <= b->kmax; k++)
    for (int j = b->j0; j <= b->jmax; j++)
    for (int i = b->i0; i <= b->imax; i++) {
        double *u = U + cidx(b, i, j, k) * FXO_NUNK;
        double vold[3] = {u[FXO_VELX], u[FXO_VELY], u[FXO_VELZ]};
        double hdt = 0.5 * dt;
        double dp = 0.;
        for (int d = 0; d < 3; d++) u[FXO_VELX + d] = vold[d] + hdt * p->grav[d];
        for (int d = 0; d < 3; d++) dp = dp + u[FXO_VELX + d] * p->grav[d];
        u[FXO_ENER] = u[FXO_ENER] + hdt * dp;
    }
}

static void energy_fix(const blk_t *b, double *U)
{
    const fxo_params *p = b->p;
    for (int k = b->k0; k <= b->kmax; k++)
    for (int j = b->j0; j <= b->jmax; j++)
    for (int i = b->i0; i <= b->imax; i++) {
        double *u = U + cidx(b, i, j, k) * FXO_NUNK;
        double ekin = 0.; ekin = ekin + u[FXO_VELX] * u[FXO_VELX]; ekin = ekin + u[FXO_VELY] * u[FXO_VELY];
        ekin = ekin + u[FXO_VELZ] * u[FXO_VELZ];
        ekin = 0.5 * ekin;
        double eint = u[FXO_ENER] - ekin - 0.0;
        double IntEner = u[FXO_EINT];
        double newEint;
        if (!p->use_aux_eint || eint > p->eint_switch * (ekin + 0.0)) newEint = fmax2(p->small_e, eint);
        else newEint = fmax2(p->small_e, IntEner);
        u[FXO_ENER] = newEint + ekin;
        u[FXO_EINT] = newEint;
    }
}

/* Eos_wrapped(MODE_DENS_EI) for one cell: Eos_getData.F90:116-150,
 * Gamma/Eos.F90:238-250, Eos_putData.F90:208-222. */
static void eos_cell(const fxo_params *p, double *u)
{
    double ekin = 0.5 * (u[FXO_VELX] * u[FXO_VELX] + u[FXO_VELY] * u[FXO_VELY] + u[FXO_VELZ] * u[FXO_VELZ]);
    double eint = u[FXO_EINT];
    if (u[FXO_ENER] - ekin > fmax2(p->small_e, p->eint_switch * ekin)) eint = u[FXO_ENER] - ekin;
    double dens = u[FXO_DENS];
    double gammam1 = 1.0 / (p->gamma - 1.0);          /* eos_gammam1, Gamma/Eos_init.F90:86 */
    double ggprod = gammam1 * p->gas_constant;
    double ggprodinv = 1. / ggprod;
    double gam1inv = 1. / gammam1;
    double pres = dens * eint * gam1inv;
    double temp = eint * ggprodinv * p->abar;
    u[FXO_PRES] = pres;
    u[FXO_TEMP] = temp;
    u[FXO_GAMC] = p->gamma;
    u[FXO_EINT] = eint;
    u[FXO_ENER] = eint + ekin;
    u[FXO_GAME] = pres / (eint * dens) + 1;
}

static void eos_block(const blk_t *b, double *U)
{
    for (int k = b->k0; k <= b->kmax; k++)
    for (int j = b->j0; j <= b->jmax; j++)
    for (int i = b->i0; i <= b->imax; i++)
        eos_cell(b->p, U + cidx(b, i, j, k) * FXO_NUNK);
}

/* ======================================================================= */
long fxo_unk_size(const fxo_params *p)
{
    blk_t b; blk_init(&b, p);
    return b.ncell * FXO_NUNK * (long)p->nblockx * p->nblocky * p->nblockz;
}

long fxo_index(const fxo_params *p, int var, int i, int j, int k, int blk)
{
    blk_t b; blk_init(&b, p);
    return ((long)blk * b.ncell + cidx(&b, i, j, k)) * FXO_NUNK + var;
}

/* Grid_fillGuardCells for a uniform block grid.  The neighbour exchange of
 * UG/gr_shiftData.F90 (periodic wrap included) is done axis by axis over the
 * full guard extent of the other axes, followed by the physical boundary
 * conditions applied in the order Z, Y, X over whole guard vectors
 * (gr_bcApplyToAllBlks with WHOLE_VECTOR), as Grid_fillGuardCells.F90:300. */
#include "fx_oracle_spec.inc"

/* UG guard fill of nv values per cell (UNK: nv = FXO_NUNK with the normal
 * velocity flipped at reflecting faces; mass fractions: nv = ns, no flip) */
static int fill_guard_nv(const fxo_params *p, double *unk, int nv, int flip);

int fxo_fill_guardcells(const fxo_params *p, double *unk) { return fill_guard_nv(p, unk, FXO_NUNK, 1); }

int fxo_fill_guardcells_spec(const fxo_params *p, double *spec, int ns)
{
    if (ns <= 0) return 0;
    return fill_guard_nv(p, spec, ns, 0);
}

static int fill_guard_nv(const fxo_params *p, double *unk, int nv, int flip)
{
    blk_t b; blk_init(&b, p);
    const int ng = b.ng, ndim = p->ndim;
    int nb[3] = {p->nblockx, ndim >= 2 ? p->nblocky : 1, ndim == 3 ? p->nblockz : 1};
    int nn[3] = {p->nxb, ndim >= 2 ? p->nyb : 1, ndim == 3 ? p->nzb : 1};
    int gx[3] = {ng, ndim >= 2 ? ng : 0, ndim == 3 ? ng : 0};
    long N[3], G[3];
    for (int d = 0; d < 3; d++) { N[d] = (long)nb[d] * nn[d]; G[d] = N[d] + 2 * gx[d]; }
    /* global grid with a guard ring */
    double *g = (double *)malloc(sizeof(double) * G[0] * G[1] * G[2] * nv);
#define GI(i, j, k) ((((long)(k) * G[1] + (j)) * G[0] + (i)) * nv)
    long nblk = (long)nb[0] * nb[1] * nb[2];
    for (long blk = 0; blk < nblk; blk++) {
        int bx = blk % nb[0], by = (blk / nb[0]) % nb[1], bz = blk / ((long)nb[0] * nb[1]);
        const double *U = unk + blk * b.ncell * nv;
        for (int k = b.k0; k <= b.kmax; k++)
        for (int j = b.j0; j <= b.jmax; j++)
        for (int i = b.i0; i <= b.imax; i++) {
            long gi = (long)bx * nn[0] + (i - b.i0) + gx[0];
            long gj = (long)by * nn[1] + (j - b.j0) + gx[1];
            long gk = (long)bz * nn[2] + (k - b.k0) + gx[2];
            memcpy(g + GI(gi, gj, gk), U + cidx(&b, i, j, k) * nv, sizeof(double) * nv);
        }
    }
    /* periodic exchanges, axis order X, Y, Z, full extent of the other axes */
    for (int a = 0; a < ndim; a++) {
        if (p->bc[2 * a] != FXO_BC_PERIODIC) continue;
        for (long k = 0; k < G[2]; k++) for (long j = 0; j < G[1]; j++) for (long i = 0; i < G[0]; i++) {
            long idx[3] = {i, j, k};
            long x = idx[a];
            if (x >= gx[a] && x < gx[a] + N[a]) continue;
            long src = (x < gx[a]) ? x + N[a] : x - N[a];
            long sidx[3] = {i, j, k}; sidx[a] = src;
            memcpy(g + GI(i, j, k), g + GI(sidx[0], sidx[1], sidx[2]), sizeof(double) * nv);
        }
    }
    /* physical boundaries, order Z, Y, X */
    for (int a = ndim - 1; a >= 0; a--) {
        for (int side = 0; side < 2; side++) {
            int bc = p->bc[2 * a + side];
            if (bc == FXO_BC_PERIODIC) continue;
            for (long k = 0; k < G[2]; k++) for (long j = 0; j < G[1]; j++) for (long i = 0; i < G[0]; i++) {
                long idx[3] = {i, j, k};
                long x = idx[a];
                long sidx[3] = {i, j, k};
                if (side == 0) {
                    if (x >= gx[a]) continue;
                    sidx[a] = (bc == FXO_BC_OUTFLOW) ? gx[a] : 2 * gx[a] - 1 - x;
                } else {
                    if (x < gx[a] + N[a]) continue;
                    long last = gx[a] + N[a] - 1;
                    sidx[a] = (bc == FXO_BC_OUTFLOW) ? last : 2 * last + 1 - x;
                }
                double *dst = g + GI(i, j, k);
                const double *src = g + GI(sidx[0], sidx[1], sidx[2]);
                for (int v = 0; v < nv; v++) {
                    double sgn = (flip && bc == FXO_BC_REFLECTING && v == FXO_VELX + a) ? -1. : 1.;
                    dst[v] = src[v] * sgn;
                }
            }
        }
    }
    /* scatter windows back into each block's guard cells */
    for (long blk = 0; blk < nblk; blk++) {
        int bx = blk % nb[0], by = (blk / nb[0]) % nb[1], bz = blk / ((long)nb[0] * nb[1]);
        double *U = unk + blk * b.ncell * nv;
        for (int k = 0; k < b.nkg; k++)
        for (int j = 0; j < b.njg; j++)
        for (int i = 0; i < b.nig; i++) {
            long gi = (long)bx * nn[0] + i;
            long gj = (long)by * nn[1] + j;
            long gk = (long)bz * nn[2] + k;
            memcpy(U + cidx(&b, i, j, k) * nv, g + GI(gi, gj, gk), sizeof(double) * nv);
        }
    }
#undef GI
    free(g);
    return 0;
}

int fxo_eos_interior(const fxo_params *p, double *unk)
{
    blk_t b; blk_init(&b, p);
    long nblk = (long)p->nblockx * p->nblocky * p->nblockz;
    for (long blk = 0; blk < nblk; blk++) eos_block(&b, unk + blk * b.ncell * FXO_NUNK);
    return 0;
}

int fxo_hydro_step(const fxo_params *p, double *unk, double dt, double dt_old, int nthreads)
{
    return fxo_hydro_step_spec(p, unk, NULL, 0, 0, dt, dt_old, nthreads);
}

int fxo_hydro_step_spec(const fxo_params *p, double *unk, double *spec, int ns, int nsp, double dt, double dt_old,
                        int nthreads)
{
    (void)dt_old;
    if (p->ndim < 2 || p->ndim > 3 || p->nguard < 4 || (p->order != 2 && p->order != 3 && p->order != 5)) return 3;
    if (ns < 0 || nsp < 0 || nsp > ns || (ns > 0 && !spec)) return 3;
    fxo_fill_guardcells(p, unk);
    if (ns) fxo_fill_guardcells_spec(p, spec, ns);
    blk_t b; blk_init(&b, p);
    long nblk = (long)p->nblockx * p->nblocky * p->nblockz;
    if (p->shock_detect) {
        /* levelFlux/Hydro.F90:133-149: the flag of every interior cell from the
         * filled state, then the guard fill again, which carries SHOK too */
        for (long blk = 0; blk < nblk; blk++) shock_detect_block(&b, unk + blk * b.ncell * FXO_NUNK);
        fxo_fill_guardcells(p, unk);
    }
    int status = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
    {
        scratch_t s;
        scratch_alloc(&s, b.ncell);
        spec_t q;
        memset(&q, 0, sizeof(q));
        if (ns) spec_alloc(&q, b.ncell, ns);
        int lerr = 0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (long blk = 0; blk < nblk; blk++) {
            double *U = unk + blk * b.ncell * FXO_NUNK;
            double *SP = ns ? spec + blk * b.ncell * ns : NULL;
            int e = riemann_states(&b, U, dt, &s);
            if (!e) e = face_fluxes(&b, U, &s);
            if (!e) {
                if (ns) {
                    spec_states(&b, U, SP, dt, &s, &q);
                    spec_fluxes(&b, &s, &q);
                    for (long c = 0; c < b.ncell; c++) q.dold[c] = U[c * FXO_NUNK + FXO_DENS];
                }
                unsplit_update(&b, U, dt, &s);
                if (ns) spec_update(&b, U, SP, dt, &q, nsp);
                if (!p->use_gravity) { energy_fix(&b, U); eos_block(&b, U); }
            }
            if (e) lerr = e;
        }
        if (ns) spec_free(&q);
        scratch_free(&s);
#ifdef _OPENMP
#pragma omp critical
#endif
        { if (lerr) status = lerr; }
    }
    if (p->use_gravity) {
        /* hy_gravityStepBlk: the n+1 gravity half step, then energyFix and Eos */
        for (long blk = 0; blk < nblk; blk++) {
            double *U = unk + blk * b.ncell * FXO_NUNK;
            gravity_step_block(&b, U, dt);
            energy_fix(&b, U);
            eos_block(&b, U);
        }
    }
    return status;
}

int fxo_compute_dt(const fxo_params *p, const double *unk, double *dt_out)
{
    blk_t b; blk_init(&b, p);
    long nblk = (long)p->nblockx * p->nblocky * p->nblockz;
    double delinv[3] = {1.0 / b.dx, 1.0 / b.dy, 1.0 / b.dz};
    double dtmin = 1.e300;   /* huge */
    for (long blk = 0; blk < nblk; blk++) {
        const double *U = unk + blk * b.ncell * FXO_NUNK;
        double dt_temp = 0.;
        for (int k = b.k0; k <= b.kmax; k++)
        for (int j = b.j0; j <= b.jmax; j++)
        for (int i = b.i0; i <= b.imax; i++) {
            const double *u = U + cidx(&b, i, j, k) * FXO_NUNK;
            double cs2 = u[FXO_GAMC] * u[FXO_PRES] / u[FXO_DENS];
            double r = (fabs(u[FXO_VELX] - 0.) + sqrt(cs2)) * delinv[0];
            if (p->ndim > 1) r = fmax2(r, (fabs(u[FXO_VELY] - 0.) + sqrt(cs2)) * delinv[1]);
            if (p->ndim > 2) r = fmax2(r, (fabs(u[FXO_VELZ] - 0.) + sqrt(cs2)) * delinv[2]);
            if (r * p->cfl > dt_temp * p->cfl) dt_temp = r;
        }
        double dtb = (dt_temp != 0.) ? p->cfl / dt_temp : 1.79769313486231570e308;
        if (dtb < dtmin) dtmin = dtb;
    }
    *dt_out = dtmin;
    return dtmin <= 0. ? 4 : 0;
}

double fxo_driver_dt(double dt_cfl, double dt_old, double f, double dtmin, double dtmax)
{
    double dtNew = fmin2(dt_cfl, dt_old * f);
    return fmin2(fmax2(dtNew, dtmin), dtmax);
}

int fxo_integrals(const fxo_params *p, const double *unk, double out[7])
{
    blk_t b; blk_init(&b, p);
    long nblk = (long)p->nblockx * p->nblocky * p->nblockz;
    double dv = b.dx * b.dy * b.dz;
    for (int q = 0; q < 7; q++) out[q] = 0.;
    for (long blk = 0; blk < nblk; blk++) {
        const double *U = unk + blk * b.ncell * FXO_NUNK;
        for (int k = b.k0; k <= b.kmax; k++)
        for (int j = b.j0; j <= b.jmax; j++)
        for (int i = b.i0; i <= b.imax; i++) {
            const double *u = U + cidx(&b, i, j, k) * FXO_NUNK;
            double rho = u[FXO_DENS];
            double ek = 0.5 * rho * (u[FXO_VELX] * u[FXO_VELX] + u[FXO_VELY] * u[FXO_VELY] + u[FXO_VELZ] * u[FXO_VELZ]);
            out[0] += rho * dv;
            out[1] += rho * u[FXO_VELX] * dv;
            out[2] += rho * u[FXO_VELY] * dv;
            out[3] += rho * u[FXO_VELZ] * dv;
            out[4] += rho * u[FXO_ENER] * dv;
            out[5] += rho * u[FXO_EINT] * dv;
            out[6] += ek * dv;
        }
    }
    return 0;
}

double fxo_flops_last_step(void) { return 0.; }

int fxo_riemann(const fxo_params *p, int dir, const double VL[8], const double VR[8], double F[8])
{
    double vl[H_NV], vr[H_NV], Fs[6], speed;
    for (int k = 0; k < 8; k++) { vl[k] = VL[k]; vr[k] = VR[k]; }
    vl[H_GR] = 0.; vr[H_GR] = 0.;
    int err = riemann_solve(p, dir, vl, vr, Fs, &speed);
    if (err) return err;
    for (int k = 0; k < 6; k++) F[k] = Fs[k];
    if (p->use_aux_eint) {
        if (F[F_D] > 0.) { F[F_VOL] = F[F_D] / vl[H_D]; F[F_EI] = F[F_D] * vl[H_EI]; }
        else             { F[F_VOL] = F[F_D] / vr[H_D]; F[F_EI] = F[F_D] * vr[H_EI]; }
    } else { F[F_VOL] = 0.; F[F_EI] = 0.; }
    return 0;
}

#include "fx_oracle_weno.inc"
#include "fx_oracle_amr.inc"
