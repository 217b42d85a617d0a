// fxb_device.cuh -- per-cell device math of the unsplit hydro path.
//
// Templated on the reconstruction type R (double for the FP64 path, float
// for the mixed path).  The primitive eigensystem of the pure-hydro solver
// is sparse (OnlyHydro/hy_eigenVector.F90:87-167: 7 nonzero left and 9
// nonzero right entries out of 25 each), so every dot product and
// projection below is written with only its nonzero terms, added in the
// reference's summation order.  Dropping a 0*x term from a left-to-right sum
// changes at most the sign of an exact zero, never a nonzero value, so the
// FP64 path built with -fmad=false reproduces the oracle's values.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fxb {

// primitive slots (UHD.h HY_DENS..HY_EINT, 0-based); device arrays use the
// same order for their first eight variables, then ENER and TEMP.
enum { D = 0, VX = 1, VY = 2, VZ = 3, P = 4, GC = 5, GE = 6, EI = 7 };
enum { NV_DEV = 10, DV_ENER = 8, DV_TEMP = 9 };
// flux slots (UHD.h HY_DENS_FLUX..HY_VOLU_FLUX)
enum { FD = 0, FMX = 1, FMY = 2, FMZ = 3, FE = 4, FP = 5, FEI = 6, FVOL = 7, NF = 8 };

enum { LIM_MINMOD = 1, LIM_MC = 2, LIM_VANLEER = 3, LIM_HYBRID = 4, LIM_LIMITED = 5 };
enum { ERR_SOUND = 1, ERR_RIEMANN = 2 };

struct DevParams {
    int order, weno_method, riemann, limiter, char_limiting, use_3d_full_ctu, use_aux_eint, use_gravity;
    double grav[3];
    double cfl, gamma, eint_switch, small_dens, small_e, small_p, tiny, fpres, limited_beta, gas_constant, abar;
    int flattening;
    int entropy_fix;           // Roe: 0 off, 1 Harten-Hyman, 2 Harten
    int steepening;            // PPM contact steepening
    int use_avisc;             // artificial viscosity
    double cvisc;
    int use_hybrid;            // hybrid order: first-order states at shocks
    double hybrid_kappa;
    int nspec;                 // advected mass fractions (species and mass scalars; uniform grids)
    int shock_detect;          // the SHOK flag before each step (uniform grids)
    // Face values (left, right) of the constant gravity component along each
    // sweep direction after the reconstruction (gravity_faces), in FP64 and
    // in FP32: the same for every cell, so fxb_init computes them once with
    // the arithmetic of the kernels that use them, instead of every cell.
    double gface[3][2];
    float gfacef[3][2];
};

// ---- precision helpers ---------------------------------------------------
template <class R> __device__ __forceinline__ R rdiv(R a, R b);
template <> __device__ __forceinline__ double rdiv<double>(double a, double b) { return a / b; }
template <> __device__ __forceinline__ float rdiv<float>(float a, float b) { return __fdividef(a, b); }
// a / b for several numerators over one denominator, given y = rdiv(1, b).
// FP64: the correctly rounded quotient from the correctly rounded
// reciprocal y by two correction steps q + (a - b q) y: q = a y is within
// 1.5 ulp of a/b, the first step leaves it within one ulp, and the second is
// Markstein's (P. Markstein, IBM J. Res. Dev. 34(1), 1990): with y within
// half an ulp of 1/b and q within one ulp, the remainder is exact in one FMA
// and RN(q + r y) = RN(a/b).  copysign gives a zero quotient the sign of
// a / b.  Five FP64 operations per quotient after one division for y.
// Valid for finite nonzero b and quotients and remainders in the normal
// range (|a| >= 2^-960 or a = 0).  FP32: the fast division.
template <class R> __device__ __forceinline__ R rdiv_y(R a, R b, R y);
template <> __device__ __forceinline__ double rdiv_y<double>(double a, double b, double y)
{
    double q = a * y;
    q = fma(fma(-b, q, a), y, q);
    q = fma(fma(-b, q, a), y, q);
    return copysign(q, a * y);
}
template <> __device__ __forceinline__ float rdiv_y<float>(float a, float b, float y) { return __fdividef(a, b); }
template <class R> __device__ __forceinline__ R rsqrt_(R a);
template <> __device__ __forceinline__ double rsqrt_<double>(double a) { return sqrt(a); }
// FP32 (mixed precision): the hardware approximation (PTX sqrt.approx.f32,
// relative error about 2^-23), one instruction instead of the correctly
// rounded sequence
template <> __device__ __forceinline__ float rsqrt_<float>(float a)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

// Division by the literal constants 3, 6 and 12 of the PPM formulas.
// FP64: the correctly rounded quotient x / C (the oracle's operation) without
// a division, by Markstein's correction step (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990): with y = RN(1/C) within half an ulp of 1/C and q0 within
// one ulp of x/C, the remainder r = x - C q0 is exact in one FMA and
// RN(q0 + r y) = RN(x/C).  For C = 3 * 2^k the reciprocal RN(1/C) has a
// relative error of exactly 2^-54, so q0 = RN(x y) is within one ulp of x/C
// for every x.  Three dependent FP64 operations replace the division's
// iteration and its slow-path branch; copysign keeps the sign of a zero
// quotient (x = -0).  Valid for finite x whose quotient is a normal number
// (|x| >= 2^-1018): the values that reach it here are differences of
// primitive slopes and states.  FP32: multiplication by the rounded
// reciprocal.
template <int C> __device__ __forceinline__ double divk(double x)
{
    static_assert(C == 3 || C == 6 || C == 12, "divk: the correction is shown for 3 * 2^k only");
    constexpr double y = 1.0 / C;
    const double q0 = x * y;
    const double r = fma(-double(C), q0, x);
    return copysign(fma(r, y, q0), x);
}
template <int C> __device__ __forceinline__ float divk(float x) { return x * (float)(1.0 / C); }

// options compiled only into kernel instantiations of their own (template
// flag EXT), so the default kernels keep their registers: the Roe solver,
// PPM contact steepening, MUSCL-Hancock reconstruction (order 2), artificial
// viscosity, hybrid order, and the exports species advection reads (2-D mass
// fluxes)
// The kernels come in three instantiations (template flag EXT): 0 the
// default options, 1 the rarely used ones (Roe, contact steepening,
// MUSCL-Hancock, artificial viscosity, hybrid order, species), 2 those with a
// Marquina solver, so that each keeps the register allocation of its own code.
__host__ __device__ inline bool marquina_solver(const DevParams &p) { return p.riemann == 5 || p.riemann == 7; }
__host__ __device__ inline bool extended_options(const DevParams &p)
{
    return p.riemann == 1 || p.riemann == 5 || p.riemann == 7 || p.riemann == 8 || p.steepening || p.order == 2 ||
           p.use_avisc || p.use_hybrid || p.nspec > 0;
}

// Fortran MIN/MAX with gfortran's argument order: mvar = a1; if (a2 < mvar) mvar = a2
template <class R> __device__ __forceinline__ R fmin2(R a, R b) { return (b < a) ? b : a; }
template <class R> __device__ __forceinline__ R fmax2(R a, R b) { return (b > a) ? b : a; }
// FP32 (mixed precision, compared within a tolerance): one min/max
// instruction instead of a compare and a select; the two forms differ only
// for NaN and for the sign of equal zeros
template <> __device__ __forceinline__ float fmin2<float>(float a, float b) { return fminf(a, b); }
template <> __device__ __forceinline__ float fmax2<float>(float a, float b) { return fmaxf(a, b); }
template <class R> __device__ __forceinline__ R sgn1(R b) { return copysign(R(1), b); }

// ---- limiters (hy_slopeLimiters.F90) ----------------------------------------
template <class R> __device__ __forceinline__ R lim_minmod(R a, R b)
{ return R(.5) * (sgn1(a) + sgn1(b)) * fmin2(fabs(a), fabs(b)); }
template <class R> __device__ __forceinline__ R lim_mc(R a, R b)
{ return (sgn1(a) + sgn1(b)) * fmin2(fmin2(fabs(a), R(.25) * fabs(a + b)), fabs(b)); }
template <class R> __device__ __forceinline__ R lim_vanleer(R a, R b)
{ return (a * b <= R(0)) ? R(0) : rdiv(R(2) * a * b, a + b); }
template <class R> __device__ __forceinline__ R lim_limited(R a, R b, R beta)
{
    if (b > R(0)) return fmax2(fmax2(R(0), fmin2(beta * a, b)), fmin2(a, beta * b));
    return fmin2(fmin2(R(0), fmax2(beta * a, b)), fmax2(a, beta * b));
}
// limiter used on characteristic wave w (w = -1: a primitive variable of kind k)
template <class R> __device__ __forceinline__ R limit(int lim, int w, int k, R a, R b, R beta)
{
    switch (lim) {
    case LIM_MINMOD:  return lim_minmod(a, b);
    case LIM_MC:      return lim_mc(a, b);
    case LIM_VANLEER: return lim_vanleer(a, b);
    case LIM_HYBRID:
        // characteristic: minmod on the acoustic/shear waves, mc on entropy (hy_TVDslope.F90:146-174);
        // primitive: mc on dens/gamc/game, minmod on velocities and pressure (:176-191)
        if (w >= 0) return (w == 2) ? lim_mc(a, b) : lim_minmod(a, b);
        return (k == D || k == GC || k == GE) ? lim_mc(a, b) : (k <= P ? lim_minmod(a, b) : R(0));
    default:          return lim_limited(a, b, beta);
    }
}

// ---- eigensystem (hy_eigenParameters.F90:84-100, hy_eigenValue.F90:58-62,
//      OnlyHydro/hy_eigenVector.F90:87-127) --------------------------------
template <class R> struct Eig {
    R lam0, un, lam4;       // u-c, u (slow/entropy/slow), u+c
    R cf, rho, ahinv, lp, a2inv, rp;
};

// The direction-independent part of a cell's eigensystem: everything but the
// normal velocity (the divisions and the square root), shared by the
// eigensystems of one cell in several directions.  Returns false on a2 <= 0
// (the reference aborts there).
template <class R> struct EigBase {
    R cf, rho, ahinv, lp, a2inv, rp;
};
template <class R> __device__ __forceinline__ bool eigen_base(R rho, R p, R gamc, EigBase<R> &b)
{
    const R dinv = rdiv(R(1), rho);
    R a2 = rdiv_y(gamc * p, rho, dinv);
    if (a2 <= R(0)) return false;
    R cf = rsqrt_(a2);
    R aa2 = cf * cf;
    b.a2inv = rdiv(R(1), aa2);
    b.ahinv = rdiv(R(.5), cf);
    R Na = R(.5) * b.a2inv;
    b.lp = dinv * Na;
    b.cf = cf; b.rho = rho; b.rp = rho * aa2;
    return true;
}
// the eigensystem along a direction with normal velocity un
template <class R> __device__ __forceinline__ void eigen_dir(const EigBase<R> &b, R un, Eig<R> &e)
{
    e.lam0 = un - b.cf; e.un = un; e.lam4 = un + b.cf;
    e.cf = b.cf; e.rho = b.rho; e.ahinv = b.ahinv; e.lp = b.lp; e.a2inv = b.a2inv; e.rp = b.rp;
}
template <class R> __device__ __forceinline__ bool eigen(R rho, R un, R p, R gamc, Eig<R> &e)
{
    EigBase<R> b;
    if (!eigen_base(rho, p, gamc, b)) return false;
    eigen_dir(b, un, e);
    return true;
}

// Left-eigenvector dot products L(:,w) . x for the five waves; x indexed by
// D, v1 (normal), v2, v3 (transverse, cyclic), P.
template <class R> struct Five { R w[5]; };
template <class R> __device__ __forceinline__ Five<R> ldot(const Eig<R> &e, R xD, R x1, R x2, R x3, R xP)
{
    Five<R> o;
    o.w[0] = e.lp * xP - e.ahinv * x1;
    o.w[1] = x2;
    o.w[2] = xD - e.a2inv * xP;
    o.w[3] = x3;
    o.w[4] = e.ahinv * x1 + e.lp * xP;
    return o;
}

// ---- TVD slope (hy_TVDslope.F90:65-276) projected to primitives ---------------
// Inputs: the three states along the sweep (D, v1, v2, v3, P, EI order).
// Output db[6] = limited slopes of D, v1, v2, v3, P (projected with R when
// charLimiting) and EI (primitive).
template <class R>
__device__ __forceinline__ void tvd_slope(const DevParams &prm, const Eig<R> &e,
                                          const R *VL, const R *V0, const R *VR, R db[6])
{
    R dL[6], dR[6];
#pragma unroll
    for (int k = 0; k < 6; k++) { dL[k] = V0[k] - VL[k]; dR[k] = VR[k] - V0[k]; }
    const R beta = R(prm.limited_beta);
    if (prm.char_limiting) {
        Five<R> a = ldot(e, dL[0], dL[1], dL[2], dL[3], dL[4]);
        Five<R> b = ldot(e, dR[0], dR[1], dR[2], dR[3], dR[4]);
        R d[5];
#pragma unroll
        for (int w = 0; w < 5; w++) d[w] = limit(prm.limiter, w, -1, a.w[w], b.w[w], beta);
        // R * delbar, summed over waves FASTLEFT..FASTRGHT (hy_DataReconstructNormalDir_PPM.F90:539-581)
        db[0] = (e.rho * d[0] + d[2]) + e.rho * d[4];
        db[1] = e.cf * d[4] - e.cf * d[0];
        db[2] = d[1];
        db[3] = d[3];
        db[4] = e.rp * d[0] + e.rp * d[4];
        // gamc/game/eint keep primitive limiting; the hybrid choice is mc for them here (:165-170)
        db[5] = (prm.limiter == LIM_HYBRID) ? lim_mc(dL[5], dR[5]) : limit(prm.limiter, -1, (int)EI, dL[5], dR[5], beta);
    } else {
        const int kind[6] = {D, VX, VY, VZ, P, EI};
#pragma unroll
        for (int k = 0; k < 6; k++) db[k] = limit(prm.limiter, -1, kind[k], dL[k], dR[k], beta);
    }
}

// ---- upwind transverse flux sig (hy_upwindTransverseFlux.F90:54-222) --------
// m, c, p: states along the transverse direction in (D, v1, v2, v3, P, EI)
// order; sig is returned in the same order.
template <class R>
__device__ __forceinline__ void trans_flux(const Eig<R> &e, const R *m, const R *c, const R *p, bool aux, R sig[6])
{
    R t[6];
    // wave 0 (u-c)
    const bool up0 = e.lam0 > R(0);
#pragma unroll
    for (int k = 0; k < 5; k++) t[k] = up0 ? c[k] - m[k] : p[k] - c[k];
    R d0 = e.lp * t[4] - e.ahinv * t[1];
    R sD = (e.lam0 * e.rho) * d0;
    R s1 = (e.lam0 * (-e.cf)) * d0;
    R sP = (e.lam0 * e.rp) * d0;
    // waves 1..3 (u)
    const bool upu = e.un > R(0);
#pragma unroll
    for (int k = 0; k < 5; k++) t[k] = upu ? c[k] - m[k] : p[k] - c[k];
    R s2 = e.un * t[2];
    sD = sD + e.un * (t[0] - e.a2inv * t[4]);
    R s3 = e.un * t[3];
    // wave 4 (u+c)
    const bool up4 = e.lam4 > R(0);
#pragma unroll
    for (int k = 0; k < 5; k++) t[k] = up4 ? c[k] - m[k] : p[k] - c[k];
    R d4 = e.ahinv * t[1] + e.lp * t[4];
    sD = sD + (e.lam4 * e.rho) * d4;
    s1 = s1 + (e.lam4 * e.cf) * d4;
    sP = sP + (e.lam4 * e.rp) * d4;
    sig[0] = sD; sig[1] = s1; sig[2] = s2; sig[3] = s3; sig[4] = sP;
    sig[5] = aux ? e.un * (upu ? c[5] - m[5] : p[5] - c[5]) : R(0);
}

// ---- PPM/WENO common tail: monotonicity, initial guesses and characteristic
// tracing (hy_DataReconstructNormalDir_PPM.F90:697-853).  vecL/vecR hold the
// interface values of D, v1, v2, v3, P, EI; Wm/Wp receive the traced states.
template <class R>
__device__ __forceinline__ void ppm_trace(const Eig<R> &e, R dtn, R hdtn, const R *Vc,
                                          R *vecL, R *vecR, R Wm[6], R Wp[6])
{
    R delW[6], W6[6];
#pragma unroll
    for (int n = 0; n < 6; n++) {
        R L = vecL[n], Rr = vecR[n], C = Vc[n];
        if ((Rr - C) * (C - L) <= R(0)) { L = C; Rr = C; }
        if (R(6) * (Rr - L) * (C - R(.5) * (L + Rr)) > (Rr - L) * (Rr - L)) L = R(3) * C - R(2) * Rr;
        if (R(6) * (Rr - L) * (C - R(.5) * (L + Rr)) < -((Rr - L) * (Rr - L))) Rr = R(3) * C - R(2) * L;
        vecL[n] = L; vecR[n] = Rr;
        delW[n] = Rr - L;
        W6[n] = R(6) * (C - R(.5) * (Rr + L));
    }
    // secondary variable EI: initial guess survives (gamc/game are reset to Vc)
    {
        R lmax = fmax2(e.un, R(0));
        Wp[5] = vecR[5] - lmax * hdtn * (delW[5] - (R(1.0) - divk<3>(lmax * hdtn * R(4.))) * W6[5]);
        R lmin = -fmin2(e.un, R(0));
        Wm[5] = vecL[5] + lmin * hdtn * (delW[5] + (R(1.0) - divk<3>(lmin * hdtn * R(4.))) * W6[5]);
    }
    // tracing over the five waves, HLL-type branch
    Five<R> cA = ldot(e, delW[0], delW[1], delW[2], delW[3], delW[4]);
    Five<R> cB;
    cB.w[0] = e.ahinv * W6[1] - e.lp * W6[4];
    cB.w[1] = -W6[2];
    cB.w[2] = -W6[0] + e.a2inv * W6[4];
    cB.w[3] = -W6[3];
    cB.w[4] = -(e.ahinv * W6[1]) - e.lp * W6[4];
    const R c43 = R(4.) / R(3.);
    R aL[3], bL[3], aR[3], bR[3];
    const R lams[3] = {e.lam0, e.un, e.lam4};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        R lam = lams[q];
        R lt = dtn * lam;
        aL[q] = R(.5) * (R(-1.) - dtn * lam);
        bL[q] = R(.25) * (R(1.) + R(2.) * dtn * lam + c43 * (lt * lt));
        aR[q] = R(.5) * (R(1.) - dtn * lam);
        bR[q] = R(.25) * (R(1.) - R(2.) * dtn * lam + c43 * (lt * lt));
    }
    // wave 0
    R sLD = (aL[0] * e.rho) * cA.w[0] + (bL[0] * e.rho) * cB.w[0];
    R sRD = (aR[0] * e.rho) * cA.w[0] + (bR[0] * e.rho) * cB.w[0];
    R sL1 = (aL[0] * (-e.cf)) * cA.w[0] + (bL[0] * (-e.cf)) * cB.w[0];
    R sR1 = (aR[0] * (-e.cf)) * cA.w[0] + (bR[0] * (-e.cf)) * cB.w[0];
    R sLP = (aL[0] * e.rp) * cA.w[0] + (bL[0] * e.rp) * cB.w[0];
    R sRP = (aR[0] * e.rp) * cA.w[0] + (bR[0] * e.rp) * cB.w[0];
    // waves 1..3 (right eigenvector entries equal to one)
    R sL2 = aL[1] * cA.w[1] + bL[1] * cB.w[1];
    R sR2 = aR[1] * cA.w[1] + bR[1] * cB.w[1];
    sLD = sLD + (aL[1] * cA.w[2] + bL[1] * cB.w[2]);
    sRD = sRD + (aR[1] * cA.w[2] + bR[1] * cB.w[2]);
    R sL3 = aL[1] * cA.w[3] + bL[1] * cB.w[3];
    R sR3 = aR[1] * cA.w[3] + bR[1] * cB.w[3];
    // wave 4
    sLD = sLD + ((aL[2] * e.rho) * cA.w[4] + (bL[2] * e.rho) * cB.w[4]);
    sRD = sRD + ((aR[2] * e.rho) * cA.w[4] + (bR[2] * e.rho) * cB.w[4]);
    sL1 = sL1 + ((aL[2] * e.cf) * cA.w[4] + (bL[2] * e.cf) * cB.w[4]);
    sR1 = sR1 + ((aR[2] * e.cf) * cA.w[4] + (bR[2] * e.cf) * cB.w[4]);
    sLP = sLP + ((aL[2] * e.rp) * cA.w[4] + (bL[2] * e.rp) * cB.w[4]);
    sRP = sRP + ((aR[2] * e.rp) * cA.w[4] + (bR[2] * e.rp) * cB.w[4]);
    const R sl[5] = {sLD, sL1, sL2, sL3, sLP}, sr[5] = {sRD, sR1, sR2, sR3, sRP};
#pragma unroll
    for (int v = 0; v < 5; v++) {
        R base = Vc[v] + divk<12>(W6[v]);
        Wm[v] = base + sl[v];
        Wp[v] = base + sr[v];
    }
}

// ---- flattening (hy_getRiemannState.F90:367-465) ----------------------------
// FlatTilde of a cell from the pressures one and two cells either side and the
// normal velocity one cell either side along the sweep
template <class R>
__device__ __forceinline__ R flat_tilde(R pm2, R pm1, R pp1, R pp2, R vm1, R vp1)
{
    R dp1 = (pp1 - pm1);
    R dp2 = (pp2 - pm2);
    R dv1 = vp1 - vm1;
    R Sp = (fabs(dp2) > R(1.e-15)) ? rdiv(dp1, dp2) - R(0.75) : R(0.);
    R ft = fmax2(R(0.), fmin2(R(1.), R(10.) * Sp));
    if ((rdiv(fabs(dp1), fmin2(pm1, pp1)) < R(1. / 3.)) || dv1 > R(0.)) ft = R(0.);
    return ft;
}
// FlatCoeff: the larger FlatTilde of the cell and its upstream neighbour in pressure
template <class R>
__device__ __forceinline__ R flat_coeff(R dp1, R ftm, R ft0, R ftp)
{
    if (dp1 < R(0.)) return fmax2(ft0, ftp);
    if (dp1 == R(0.)) return ft0;
    return fmax2(ft0, ftm);
}
// [5] of the PPM/WENO reconstructions: interface values pulled toward the
// cell value by the flattening coefficient
template <class R>
__device__ __forceinline__ void flatten(R F, const R *Vc, R vecL[6], R vecR[6])
{
#pragma unroll
    for (int n = 0; n < 6; n++) {
        vecL[n] = F * Vc[n] + (R(1.0) - F) * vecL[n];
        vecR[n] = F * Vc[n] + (R(1.0) - F) * vecR[n];
    }
}

// MUSCL-Hancock face states (hy_DataReconstructNormalDir_MH.F90): one TVD
// slope of the cell (characteristic amplitudes when charLimiting, primitive
// slopes otherwise), scaled by 1 - F with flattening; eint reconstructed
// linearly, clamped and traced with the entropy wave when it is carried
// (aux eint or gravity, hyEndVar >= HY_EINT); D, v1, v2, v3, P traced over
// the five waves from the cell value, the Roe solver keeping only each
// wave's upwind side.  Vm, Vc, Vp in sweep order (D, v1, v2, v3, P, EI).
template <class R>
__device__ __forceinline__ void mh_trace(const DevParams &prm, const Eig<R> &e, R dtn, R hdtn, const R *Vm,
                                         const R *Vc, const R *Vp, R F, R Wm[6], R Wp[6])
{
    R dL[6], dR[6], A[5], d5;
#pragma unroll
    for (int k = 0; k < 6; k++) { dL[k] = Vc[k] - Vm[k]; dR[k] = Vp[k] - Vc[k]; }
    const R beta = R(prm.limited_beta);
    if (prm.char_limiting) {
        Five<R> a = ldot(e, dL[0], dL[1], dL[2], dL[3], dL[4]);
        Five<R> b = ldot(e, dR[0], dR[1], dR[2], dR[3], dR[4]);
#pragma unroll
        for (int w = 0; w < 5; w++) A[w] = limit(prm.limiter, w, -1, a.w[w], b.w[w], beta);
        d5 = (prm.limiter == LIM_HYBRID) ? lim_mc(dL[5], dR[5]) : limit(prm.limiter, -1, (int)EI, dL[5], dR[5], beta);
        if (prm.flattening) {
#pragma unroll
            for (int w = 0; w < 5; w++) A[w] = A[w] * (R(1.) - F);
            d5 = d5 * (R(1.) - F);
        }
    } else {
        const int kind[5] = {D, VX, VY, VZ, P};
        R db[5];
#pragma unroll
        for (int k = 0; k < 5; k++) db[k] = limit(prm.limiter, -1, kind[k], dL[k], dR[k], beta);
        d5 = limit(prm.limiter, -1, (int)EI, dL[5], dR[5], beta);
        if (prm.flattening) {
#pragma unroll
            for (int k = 0; k < 5; k++) db[k] = db[k] * (R(1.) - F);
            d5 = d5 * (R(1.) - F);
        }
        Five<R> c = ldot(e, db[0], db[1], db[2], db[3], db[4]);
#pragma unroll
        for (int w = 0; w < 5; w++) A[w] = c.w[w];
    }
    if (prm.use_aux_eint || prm.use_gravity) {
        R wp = Vc[5] + R(0.5) * d5, wm = Vc[5] - R(0.5) * d5;
        wm = fmax2(fmin2(Vc[5], wm), fmin2(fmax2(Vc[5], wm), wm));
        wp = fmax2(fmin2(Vc[5], wp), fmin2(fmax2(Vc[5], wp), wp));
        Wp[5] = wp - fmax2(e.un, R(0.)) * hdtn * d5;
        Wm[5] = wm - fmin2(e.un, R(0.)) * hdtn * d5;
    } else {
        Wp[5] = R(0.); Wm[5] = R(0.);
    }
    const R lam[5] = {e.lam0, e.un, e.un, e.un, e.lam4};
    const bool roe = prm.riemann == 1;
    R cL[5], cR[5];
    bool useL[5], useR[5];
#pragma unroll
    for (int n = 0; n < 5; n++) {
        cL[n] = R(.5) * (R(-1.) - dtn * lam[n]);
        cR[n] = R(.5) * (R(1.) - dtn * lam[n]);
        useL[n] = !roe || lam[n] < R(0.);
        useR[n] = !roe || !(lam[n] < R(0.));
    }
    // nonzero right-eigenvector entries: D (rho, 1, rho on waves 0, 2, 4),
    // v1 (-c, c on 0, 4), v2 (1 on 1), v3 (1 on 3), P (rho c^2 on 0, 4)
    R sL[5] = {R(0.), R(0.), R(0.), R(0.), R(0.)}, sR[5] = {R(0.), R(0.), R(0.), R(0.), R(0.)};
    if (useL[0]) { sL[0] = sL[0] + cL[0] * e.rho * A[0]; sL[1] = sL[1] + cL[0] * (-e.cf) * A[0];
                   sL[4] = sL[4] + cL[0] * e.rp * A[0]; }
    if (useR[0]) { sR[0] = sR[0] + cR[0] * e.rho * A[0]; sR[1] = sR[1] + cR[0] * (-e.cf) * A[0];
                   sR[4] = sR[4] + cR[0] * e.rp * A[0]; }
    if (useL[1]) sL[2] = sL[2] + cL[1] * A[1];
    if (useR[1]) sR[2] = sR[2] + cR[1] * A[1];
    if (useL[2]) sL[0] = sL[0] + cL[2] * A[2];
    if (useR[2]) sR[0] = sR[0] + cR[2] * A[2];
    if (useL[3]) sL[3] = sL[3] + cL[3] * A[3];
    if (useR[3]) sR[3] = sR[3] + cR[3] * A[3];
    if (useL[4]) { sL[0] = sL[0] + cL[4] * e.rho * A[4]; sL[1] = sL[1] + cL[4] * e.cf * A[4];
                   sL[4] = sL[4] + cL[4] * e.rp * A[4]; }
    if (useR[4]) { sR[0] = sR[0] + cR[4] * e.rho * A[4]; sR[1] = sR[1] + cR[4] * e.cf * A[4];
                   sR[4] = sR[4] + cR[4] * e.rp * A[4]; }
#pragma unroll
    for (int v = 0; v < 5; v++) { Wm[v] = Vc[v] + sL[v]; Wp[v] = Vc[v] + sR[v]; }
}

// Artificial viscosity of one face (hy_getFaceFlux.F90:397-438 x, 700-745 y,
// 955-990 z; Colella and Woodward 1984), added to the Godunov flux before the
// aux-eint fluxes are formed: cvisc times the negative part of the undivided
// velocity divergence at the face (normal difference nm -> n0 of the cells
// behind and ahead, plus the transverse terms tr[e] = quarter-weighted
// central differences of both cells times del[d]/del[e], 0 where absent),
// times the jump of dens, momenta and total energy.  Ul, Ur: D, VX, VY, VZ,
// ENER of the cells behind and ahead.
template <class R>
__device__ __forceinline__ void avisc_flux(R cvisc, int d, int ndim, R nm, R n0, const R tr[3], const R Ul[5],
                                           const R Ur[5], R F[])
{
    R div;
    if (d == 0) {
        div = n0 - nm;
        if (ndim > 1) div = div + tr[1];
        if (ndim > 2) div = div + tr[2];
    } else if (d == 1) {
        div = tr[0] + n0 - nm;
        if (ndim > 2) div = div + tr[2];
    } else {
        div = tr[0] + tr[1] + n0 - nm;
    }
    const R cv = cvisc * fmax2(-(div), R(0.));
    F[0] = F[0] + cv * (Ul[0] - Ur[0]);
#pragma unroll
    for (int q = 1; q < 5; q++) F[q] = F[q] + cv * (Ul[0] * Ul[q] - Ur[0] * Ur[q]);
}
// aux-eint and volume fluxes from the final mass flux (hy_getFaceFlux.F90:444-453)
template <class R>
__device__ __forceinline__ void eint_fluxes(const DevParams &prm, const R *Vm, const R *Vp, R F[])
{
    if (prm.use_aux_eint) {
        if (F[0] > R(0)) { F[FVOL] = rdiv(F[0], Vm[D]); F[FEI] = F[0] * Vm[5]; }
        else             { F[FVOL] = rdiv(F[0], Vp[D]); F[FEI] = F[0] * Vp[5]; }
    } else { F[FVOL] = R(0); F[FEI] = R(0); }
}

// Hybrid order (hy_dataReconstOneStep.F90:864-913, hy_checkRHjumpCond.F90):
// where the velocity converges (the caller found min DivU over the cell's
// box below hybridOrderKappa times the sound speed), face states whose
// density leaves the bounds of a shock jump, (gamc-1)/(gamc+1) to
// (gamc+1)/(gamc-1) times the cell density, in a flow of Mach^2 > 1e-4,
// fall back to the cell values.  g: the cell's 6-vector (D, VX, VY, VZ, P,
// EI) in global order (ndim components in Mach^2); reset: the same values
// in the frame of Wm/Wp.
template <class R>
__device__ __forceinline__ void hybrid_rh(int ndim, const R g[6], const R reset[6], R gamc, R Wm[6], R Wp[6])
{
    const R dens = g[0], pres = g[4];
    const R gr = rdiv(gamc + R(1.), gamc - R(1.));
    R m2 = R(0.);
    for (int e = 0; e < ndim; e++) m2 = m2 + g[1 + e] * g[1 + e];
    m2 = rdiv(m2 * dens, gamc * pres);
    bool sw = false;
    if (m2 > R(1.e-4)) {
        if (Wm[0] > gr * dens || gr * Wm[0] < dens) sw = true;
        if (Wp[0] > gr * dens || gr * Wp[0] < dens) sw = true;
    }
    if (sw) {
#pragma unroll
        for (int k = 0; k < 6; k++) { Wm[k] = reset[k]; Wp[k] = reset[k]; }
    }
}
// the hybrid-order threshold hybridOrderKappa * sqrt(gamc p / rho) of a cell
template <class R> __device__ __forceinline__ R hybrid_eps(const DevParams &prm, R dens, R pres, R gamc)
{
    R cs = gamc * pres;
    cs = rsqrt_(rdiv(cs, dens));
    return R(prm.hybrid_kappa) * cs;
}

// contact steepening of the PPM density interface values
// (hy_DataReconstructNormalDir_PPM.F90:650-681; eta1 = 20, eta2 = 0.05,
// epsln = 0.01, K0 = 0.1 from :149).  Vm, Vc, Vp: the three cells in sweep
// order, rhoMM / rhoPP the densities two cells out, dbN0 / dbP0 the density
// slopes of the two neighbours, delta the cell width along the sweep.
template <class R>
__device__ __forceinline__ void steepen(R tiny, R delta, R rhoMM, const R *Vm, const R *Vc, const R *Vp, R rhoPP,
                                        R gameC, R dbN0, R dbP0, R vecL[6], R vecR[6])
{
    const R temp1 = Vp[0] - Vm[0];
    if (fabs(temp1) > tiny) {
        const R d2R = rdiv(rhoPP - R(2.) * Vp[0] + Vc[0], R(6.) * delta * delta);
        const R d2L = rdiv(Vc[0] - R(2.) * Vm[0] + rhoMM, R(6.) * delta * delta);
        R eta = rdiv((d2L - d2R) * (delta * delta), temp1);
        if (d2R * d2L >= R(0.)) eta = R(0.);
        if (R(0.01) * fmin2(Vp[0], Vm[0]) - fabs(Vp[0] - Vm[0]) >= R(0.)) eta = R(0.);
        eta = fmax2(R(0.), fmin2(R(1.), R(20.) * (eta - R(0.05))));
        const R temp2 = rdiv(fabs(Vp[4] - Vm[4]), fmin2(Vp[4], Vm[4]));
        const R temp3 = rdiv(fabs(Vp[0] - Vm[0]), fmin2(Vp[0], Vm[0]));
        if (gameC * R(0.1) * temp3 - temp2 < R(0.0)) eta = R(0.);
        vecL[0] = vecL[0] * (R(1.) - eta) + (Vm[0] + R(0.5) * dbN0) * eta;
        vecR[0] = vecR[0] * (R(1.) - eta) + (Vp[0] - R(0.5) * dbP0) * eta;
    }
}

// PPM interface values (hy_DataReconstructNormalDir_PPM.F90:590-593)
template <class R>
__device__ __forceinline__ void ppm_interfaces(const R *Vm, const R *Vc, const R *Vp,
                                               const R *dbN, const R *db0, const R *dbP, R vecL[6], R vecR[6])
{
#pragma unroll
    for (int n = 0; n < 6; n++) {
        vecL[n] = R(.5) * (Vc[n] + Vm[n]) - divk<6>(db0[n] - dbN[n]);
        vecR[n] = R(.5) * (Vc[n] + Vp[n]) - divk<6>(dbP[n] - db0[n]);
    }
}

// WENO5 / WENO-Z interface values of one scalar stencil
// (hy_DataReconstructNormalDir_WENO.F90:458-560, tiny = 1e-36, wenoExp = 1).
// One out-of-line body shared by the six stencils of a cell (returned by
// value, so nothing goes through local memory): the inlined copies made the
// 3-D face-state kernels miss the instruction cache (RT 256^3 FP64 16.05 ->
// 15.93 ms, mixed 6.57 -> 6.51 ms; the same operations, bit-identical).
template <class R> struct WenoPair { R r, l; };
template <class R>
__device__ __noinline__ WenoPair<R> weno_scalar_body(int method, R I0, R I1, R I2, R I3, R I4);
template <class R>
__device__ __forceinline__ void weno_scalar(int method, R I0, R I1, R I2, R I3, R I4, R &vr, R &vl)
{
    const WenoPair<R> w = weno_scalar_body<R>(method, I0, I1, I2, I3, I4);
    vr = w.r; vl = w.l;
}
template <class R>
__device__ __noinline__ WenoPair<R> weno_scalar_body(int method, R I0, R I1, R I2, R I3, R I4)
{
    R vr, vl;
    const R c6 = R(6.);
    const R p00 = R(2.) / c6, p01 = R(-7.) / c6, p02 = R(11.) / c6;
    const R p10 = R(-1.) / c6, p11 = R(5.) / c6, p12 = R(2.) / c6;
    const R p20 = R(2.) / c6, p21 = R(5.) / c6, p22 = R(-1.) / c6;
    const R m00 = R(-1.) / c6, m01 = R(5.) / c6, m02 = R(2.) / c6;
    const R m10 = R(2.) / c6, m11 = R(5.) / c6, m12 = R(-1.) / c6;
    const R m20 = R(11.) / c6, m21 = R(-7.) / c6, m22 = R(2.) / c6;
    R w5p0 = p00 * I0 + p01 * I1 + p02 * I2;
    R w5p1 = p10 * I1 + p11 * I2 + p12 * I3;
    R w5p2 = p20 * I2 + p21 * I3 + p22 * I4;
    R w5m0 = m00 * I0 + m01 * I1 + m02 * I2;
    R w5m1 = m10 * I1 + m11 * I2 + m12 * I3;
    R w5m2 = m20 * I2 + m21 * I3 + m22 * I4;
    const R c1312 = R(13.) / R(12.);
    R t1, t2;
    t1 = I0 - R(2.) * I1 + I2; t2 = I0 - R(4.) * I1 + R(3.) * I2;
    R b0 = c1312 * (t1 * t1) + R(0.25) * (t2 * t2);
    t1 = I1 - R(2.) * I2 + I3; t2 = I1 - I3;
    R b1 = c1312 * (t1 * t1) + R(0.25) * (t2 * t2);
    t1 = I2 - R(2.) * I3 + I4; t2 = R(3.) * I2 - R(4.) * I3 + I4;
    R b2 = c1312 * (t1 * t1) + R(0.25) * (t2 * t2);
    const R tiny = R(1.e-36);
    // every quotient below shares its denominator with another: the
    // indicators' with the other side's, the sums' with the other weights
    const R d0 = tiny + b0, d1 = tiny + b1, d2 = tiny + b2;
    const R y0 = rdiv(R(1), d0), y1 = rdiv(R(1), d1), y2 = rdiv(R(1), d2);
    R a0, a1, a2, s, ys;
    // i+1/2, gammas (0.1, 0.6, 0.3)
    if (method == 2) {
        R tau = fabs(b0 - b2);
        a0 = R(0.1) * (R(1.) + rdiv_y(tau, d0, y0));
        a1 = R(0.6) * (R(1.) + rdiv_y(tau, d1, y1));
        a2 = R(0.3) * (R(1.) + rdiv_y(tau, d2, y2));
    } else {
        a0 = rdiv_y(R(0.1), d0, y0); a1 = rdiv_y(R(0.6), d1, y1); a2 = rdiv_y(R(0.3), d2, y2);
    }
    s = a0 + a1 + a2;
    ys = rdiv(R(1), s);
    vr = rdiv_y(a0, s, ys) * w5p0 + rdiv_y(a1, s, ys) * w5p1 + rdiv_y(a2, s, ys) * w5p2;
    // i-1/2, gammas (0.3, 0.6, 0.1)
    if (method == 2) {
        R tau = fabs(b0 - b2);
        a0 = R(0.3) * (R(1.) + rdiv_y(tau, d0, y0));
        a1 = R(0.6) * (R(1.) + rdiv_y(tau, d1, y1));
        a2 = R(0.1) * (R(1.) + rdiv_y(tau, d2, y2));
    } else {
        a0 = rdiv_y(R(0.3), d0, y0); a1 = rdiv_y(R(0.6), d1, y1); a2 = rdiv_y(R(0.1), d2, y2);
    }
    s = a0 + a1 + a2;
    ys = rdiv(R(1), s);
    vl = rdiv_y(a0, s, ys) * w5m0 + rdiv_y(a1, s, ys) * w5m1 + rdiv_y(a2, s, ys) * w5m2;
    return WenoPair<R>{vr, vl};
}

// WENO interface values of D, v1, v2, v3, P (characteristic when charLimiting)
// and EI (primitive).  S[0..4][6] = Vmm, Vm, Vc, Vp, Vpp.
template <class R>
__device__ __forceinline__ void weno_interfaces(const DevParams &prm, const Eig<R> &e, const R S[5][6],
                                                R vecL[6], R vecR[6])
{
    if (prm.char_limiting) {
        Five<R> w[5];
#pragma unroll
        for (int s = 0; s < 5; s++) w[s] = ldot(e, S[s][0], S[s][1], S[s][2], S[s][3], S[s][4]);
        R cr[5], cl[5];
#pragma unroll
        for (int n = 0; n < 5; n++)
            weno_scalar(prm.weno_method, w[0].w[n], w[1].w[n], w[2].w[n], w[3].w[n], w[4].w[n], cr[n], cl[n]);
        vecR[0] = (e.rho * cr[0] + cr[2]) + e.rho * cr[4];
        vecR[1] = e.cf * cr[4] - e.cf * cr[0];
        vecR[2] = cr[1]; vecR[3] = cr[3];
        vecR[4] = e.rp * cr[0] + e.rp * cr[4];
        vecL[0] = (e.rho * cl[0] + cl[2]) + e.rho * cl[4];
        vecL[1] = e.cf * cl[4] - e.cf * cl[0];
        vecL[2] = cl[1]; vecL[3] = cl[3];
        vecL[4] = e.rp * cl[0] + e.rp * cl[4];
    } else {
#pragma unroll
        for (int n = 0; n < 5; n++)
            weno_scalar(prm.weno_method, S[0][n], S[1][n], S[2][n], S[3][n], S[4][n], vecR[n], vecL[n]);
    }
    weno_scalar(prm.weno_method, S[0][5], S[1][5], S[2][5], S[3][5], S[4][5], vecR[5], vecL[5]);
}

// Reconstructed face values of the (constant) gravity component along the
// sweep: PPM returns the constant exactly; WENO's weighted interpolants may
// differ from it by rounding, and the monotonicity check of CW84 eq. 1.10 then
// decides what survives (hy_DataReconstructNormalDir_WENO.F90:772-790, [7-d]).
template <class R>
__device__ __forceinline__ void gravity_faces(const DevParams &prm, R g, R &gl, R &gr)
{
    gl = g; gr = g;
    if (prm.order != 5) return;
    R vr, vl;
    weno_scalar(prm.weno_method, g, g, g, g, g, vr, vl);
    R L = vl, Rr = vr, C = g;
    if ((Rr - C) * (C - L) <= R(0)) { L = C; Rr = C; }
    if (R(6) * (Rr - L) * (C - R(.5) * (L + Rr)) > (Rr - L) * (Rr - L)) L = R(3) * C - R(2) * Rr;
    if (R(6) * (Rr - L) * (C - R(.5) * (L + Rr)) < -((Rr - L) * (Rr - L))) Rr = R(3) * C - R(2) * L;
    gl = L; gr = Rr;
}
// gravity_faces of direction d as computed at initialisation
template <class R> __device__ __forceinline__ void gravity_face_values(const DevParams &prm, int d, R &gl, R &gr);
template <> __device__ __forceinline__ void gravity_face_values<double>(const DevParams &prm, int d, double &gl,
                                                                        double &gr)
{ gl = prm.gface[d][0]; gr = prm.gface[d][1]; }
template <> __device__ __forceinline__ void gravity_face_values<float>(const DevParams &prm, int d, float &gl,
                                                                      float &gr)
{ gl = prm.gfacef[d][0]; gr = prm.gfacef[d][1]; }
template <class R> __global__ void gravity_faces_kernel(DevParams prm, R *out)
{
    for (int d = 0; d < 3; d++) gravity_faces(prm, R(prm.grav[d]), out[2 * d], out[2 * d + 1]);
}

// ---- Riemann solvers (hy_HLLC.F90:64-335, hy_HLL.F90:64-182) ---------------
// Vm/Vp: 6-vectors D, VX, VY, VZ, P (global axes), EI; gamc/game passed separately.
// F[8] receives the HY_*_FLUX slots including the aux-eint pair.
// OnlyHydro/hy_eigenVector.F90:195-260 (cons = .true.): conservative left and
// right eigenvectors of the state Va = D, VX, VY, VZ, P with gamma_e ge and
// sound speed cf along dir; L[variable][wave], Rv[variable][wave], the waves
// u - c, shear, entropy, shear, u + c
template <class R>
__device__ __forceinline__ void cons_eigvec(int dir, const R Va[5], R ge, R cf, R L[5][5], R Rv[5][5])
{
    const int v1 = 1 + dir, v2 = 1 + (dir + 1) % 3, v3 = 1 + (dir + 2) % 3;
    const R V1 = Va[v1], V2 = Va[v2], V3 = Va[v3];
    const R k = R(1.) - ge;
    const R a2e = cf * cf, a2inv = rdiv(R(1.), a2e), Na = R(0.5) * a2inv;
    R u2 = R(0.);
    u2 = u2 + Va[1] * Va[1]; u2 = u2 + Va[2] * Va[2]; u2 = u2 + Va[3] * Va[3];
    u2 = R(0.5) * u2;
    const R H = rdiv(Va[0] * u2 - rdiv(Va[4], k) + Va[4], Va[0]);
#pragma unroll
    for (int a = 0; a < 5; a++)
#pragma unroll
        for (int w = 0; w < 5; w++) { L[a][w] = R(0); Rv[a][w] = R(0); }
    L[0][0] = Na * (-(k * u2) + V1 * cf); L[v1][0] = -(Na * (-(k * V1) + cf));
    L[v2][0] = Na * k * V2; L[v3][0] = Na * k * V3; L[4][0] = -(Na * k);
    L[0][1] = -V2; L[v2][1] = R(1.);
    L[0][2] = R(1.) + Na * k * u2 * R(2.);
    L[v1][2] = -(k * V1 * a2inv); L[v2][2] = -(k * V2 * a2inv); L[v3][2] = -(k * V3 * a2inv);
    L[4][2] = k * a2inv;
    L[0][3] = -V3; L[v3][3] = R(1.);
    L[0][4] = Na * (-(k * u2) - V1 * cf); L[v1][4] = -(Na * (-(k * V1) - cf));
    L[v2][4] = Na * k * V2; L[v3][4] = Na * k * V3; L[4][4] = -(Na * k);
    Rv[0][0] = R(1.); Rv[v1][0] = V1 - cf; Rv[v2][0] = V2; Rv[v3][0] = V3; Rv[4][0] = H - V1 * cf;
    Rv[v2][1] = R(1.); Rv[4][1] = V2;
    Rv[0][2] = R(1.); Rv[v1][2] = V1; Rv[v2][2] = V2; Rv[v3][2] = V3; Rv[4][2] = u2;
    Rv[v3][3] = R(1.); Rv[4][3] = V3;
    Rv[0][4] = R(1.); Rv[v1][4] = V1 + cf; Rv[v2][4] = V2; Rv[v3][4] = V3; Rv[4][4] = H + V1 * cf;
}

// hy_Roe.F90:62-205 (acoustic eigenvalues entropy-fixed by hy_entropyFix.F90
// when entropy = .true.): the mean state of hy_avgState, its
// conservative eigenvectors (OnlyHydro/hy_eigenVector.F90:128-166) and
// F = (FL + FR - sum_w |lambda_w| r_w (l_w . (UR - UL))) / 2, the dot products
// over all five rows, zeros included, as dot_product does.  Only the kernel
// instantiations for the rarely used options (EXT: Roe, contact steepening)
// contain it, so the default kernels keep their register allocation.
template <class R>
__device__ __forceinline__ int riemann_roe(int dir, int entropy_fix, const R *Vm, R gcL, R geL, const R *Vp, R gcR, R geR,
                                        const R UL[5], const R UR[5], const R FL[6], const R FR[6], R F[8])
{
    const R Va[5] = {R(.5) * (Vm[D] + Vp[D]), R(.5) * (Vm[VX] + Vp[VX]), R(.5) * (Vm[VY] + Vp[VY]),
                     R(.5) * (Vm[VZ] + Vp[VZ]), R(.5) * (Vm[P] + Vp[P])};
    const R unA = Va[1 + dir];
    const R sig = unA == R(0) ? R(0) : (unA > R(0) ? R(1) : R(-1));
    const R gcA = R(0.5) * ((R(1.) + sig) * gcL + (R(1.) - sig) * gcR);
    const R geA = R(0.5) * ((R(1.) + sig) * geL + (R(1.) - sig) * geR);
    const R a2 = rdiv(gcA * Va[4], Va[0]);
    if (a2 <= R(0)) return ERR_SOUND;   // hy_eigenParameters aborts
    const R cf = rsqrt_(a2);
    R lam[5] = {unA - cf, unA, unA, unA, unA + cf};
    if (entropy_fix) {   // hy_entropyFix.F90 on the two acoustic waves
        const R a2L = rdiv(gcL * Vm[P], Vm[D]), a2R = rdiv(gcR * Vp[P], Vp[D]);
        if (a2L <= R(0) || a2R <= R(0)) return ERR_SOUND;
        const R uL = Vm[1 + dir], uR = Vp[1 + dir], cL = rsqrt_(a2L), cR = rsqrt_(a2R);
        const R lL[2] = {uL - cL, uL + cL}, lR[2] = {uR - cR, uR + cR};
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int w = 4 * q;
            if (lR[q] > R(0.) && lL[q] < R(0.)) {
                if (entropy_fix == 1) {            // HartenHyman
                    const R Lh = rdiv(lL[q] * (lR[q] - lam[w]), lR[q] - lL[q]);
                    const R Rh = rdiv(lR[q] * (lam[w] - lL[q]), lR[q] - lL[q]);
                    lam[w] = Rh - Lh;
                } else {                            // Harten
                    const R dl = fmax2(R(4.0) * (lR[q] - lL[q]), R(0.0));
                    if (fabs(lam[w]) < R(0.5) * dl) {
                        if (lam[w] >= R(0.0)) lam[w] = (rdiv(lam[w] * lam[w], dl) + R(.25) * dl);
                        else lam[w] = -(rdiv(lam[w] * lam[w], dl) + R(.25) * dl);
                    }
                }
            }
        }
    }
    R L[5][5], Rv[5][5];
    cons_eigvec(dir, Va, geA, cf, L, Rv);
    R dU[5], sigF[5] = {R(0), R(0), R(0), R(0), R(0)};
#pragma unroll
    for (int a = 0; a < 5; a++) dU[a] = UR[a] - UL[a];
#pragma unroll
    for (int w = 0; w < 5; w++) {
        R dp = R(0.);
#pragma unroll
        for (int a = 0; a < 5; a++) dp = dp + L[a][w] * dU[a];
#pragma unroll
        for (int a = 0; a < 5; a++) sigF[a] = sigF[a] + fabs(lam[w]) * Rv[a][w] * dp;
    }
#pragma unroll
    for (int a = 0; a < 5; a++) F[a] = (FR[a] + FL[a] - sigF[a]) * R(0.5);
    F[5] = (FR[5] + FL[5] - R(0.)) * R(0.5);
    return 0;
}

// Columns of the conservative eigenvectors of cons_eigvec, one at a time
// (same expressions): the per-state constants, then column w of L or R in
// variable order D, MX, MY, MZ, E.
template <class R> struct EigC {
    R k, a2inv, Na, u2, H, V1, V2, V3, cf;
    int v1, v2, v3;
};
template <class R>
__device__ __forceinline__ EigC<R> eig_consts(int dir, const R Va[5], R ge, R cf)
{
    EigC<R> e;
    e.v1 = 1 + dir; e.v2 = 1 + (dir + 1) % 3; e.v3 = 1 + (dir + 2) % 3;
    e.V1 = Va[e.v1]; e.V2 = Va[e.v2]; e.V3 = Va[e.v3];
    e.k = R(1.) - ge;
    e.cf = cf;
    const R a2e = cf * cf;
    e.a2inv = rdiv(R(1.), a2e);
    e.Na = R(0.5) * e.a2inv;
    R u2 = R(0.);
    u2 = u2 + Va[1] * Va[1]; u2 = u2 + Va[2] * Va[2]; u2 = u2 + Va[3] * Va[3];
    e.u2 = R(0.5) * u2;
    e.H = rdiv(Va[0] * e.u2 - rdiv(Va[4], e.k) + Va[4], Va[0]);
    return e;
}
// d: density row, n / t1 / t2: momentum along v1 / v2 / v3, en: energy row
template <class R>
__device__ __forceinline__ void eig_place(const EigC<R> &e, R d, R n, R t1, R t2, R en, R c[5])
{
    c[0] = d; c[4] = en;
#pragma unroll
    for (int a = 1; a < 4; a++) c[a] = a == e.v1 ? n : (a == e.v2 ? t1 : t2);
}
template <class R>
__device__ __forceinline__ void eig_lcol(const EigC<R> &e, int w, R c[5])
{
    const R z = R(0);
    if (w == 0)
        eig_place(e, e.Na * (-(e.k * e.u2) + e.V1 * e.cf), -(e.Na * (-(e.k * e.V1) + e.cf)), e.Na * e.k * e.V2,
                  e.Na * e.k * e.V3, -(e.Na * e.k), c);
    else if (w == 1)
        eig_place(e, -e.V2, z, R(1.), z, z, c);
    else if (w == 2)
        eig_place(e, R(1.) + e.Na * e.k * e.u2 * R(2.), -(e.k * e.V1 * e.a2inv), -(e.k * e.V2 * e.a2inv),
                  -(e.k * e.V3 * e.a2inv), e.k * e.a2inv, c);
    else if (w == 3)
        eig_place(e, -e.V3, z, z, R(1.), z, c);
    else
        eig_place(e, e.Na * (-(e.k * e.u2) - e.V1 * e.cf), -(e.Na * (-(e.k * e.V1) - e.cf)), e.Na * e.k * e.V2,
                  e.Na * e.k * e.V3, -(e.Na * e.k), c);
}
template <class R>
__device__ __forceinline__ void eig_rcol(const EigC<R> &e, int w, R c[5])
{
    const R z = R(0);
    if (w == 0) eig_place(e, R(1.), e.V1 - e.cf, e.V2, e.V3, e.H - e.V1 * e.cf, c);
    else if (w == 1) eig_place(e, z, z, R(1.), z, e.V2, c);
    else if (w == 2) eig_place(e, R(1.), e.V1, e.V2, e.V3, e.u2, c);
    else if (w == 3) eig_place(e, z, z, z, R(1.), e.V3, c);
    else eig_place(e, R(1.), e.V1 + e.cf, e.V2, e.V3, e.H + e.V1 * e.cf, c);
}

// hy_Marquina.F90:52-227 and hy_MarquinaModified.F90:52-195 (hydro), with the
// arithmetic of the oracle: eigenvalues and conservative eigenvectors of the
// left and of the right state.  Marquina (modified = false) is restated as
// the reference writes it: per wave k, leig is read as leig(k, 1:5) (the
// stored layout is leig(variable, wave)), each projection adds leig(k, XMOM
// + dir - 1) times the face pressure, the upwind side's part where both
// states' eigenvalues share a sign, else half of each side's flux plus or
// minus the largest |eigenvalue| times its conserved state; the sum along
// the right eigenvectors, face-pressure slot zero.  MarquinaModified: the
// mean flux less half the sum over waves of 0.5 (|lam_L| + |lam_R|)
// (r_R (l_R . U_R) - r_L (l_L . U_L)).  The eigenvectors are built a column
// at a time; only the EXT = 2 kernel instantiations contain this.
template <class R>
__device__ __forceinline__ int riemann_marquina(int dir, bool modified, const R *Vm, R gcL, R geL, const R *Vp, R gcR,
                                                R geR, const R UL[5], const R UR[5], const R FL[6], const R FR[6],
                                                R F[8])
{
    const R aL2 = rdiv(gcL * Vm[P], Vm[D]), aR2 = rdiv(gcR * Vp[P], Vp[D]);
    if (aL2 <= R(0) || aR2 <= R(0)) return ERR_SOUND;   // hy_eigenParameters aborts
    const R cL = rsqrt_(aL2), cR = rsqrt_(aR2);
    const R uL = Vm[1 + dir], uR = Vp[1 + dir];
    // hy_eigenValue: u - c, u, u, u, u + c
    auto lam = [](R u, R c, int k) { return k == 0 ? u - c : (k == 4 ? u + c : u); };
    if (!modified) {
        R mL = fabs(lam(uL, cL, 0)), mR = fabs(lam(uR, cR, 0));
#pragma unroll
        for (int k = 1; k < 5; k++) {
            if (fabs(lam(uL, cL, k)) > mL) mL = fabs(lam(uL, cL, k));
            if (fabs(lam(uR, cR, k)) > mR) mR = fabs(lam(uR, cR, k));
        }
        const R amax = fmax2(mL, mR);
        const int mom = 1 + dir;
        R part0[5];
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const R *Vs = side ? Vp : Vm;
            const R Va[5] = {Vs[D], Vs[VX], Vs[VY], Vs[VZ], Vs[P]};
            const EigC<R> e = eig_consts(dir, Va, side ? geR : geL, side ? cR : cL);
            const R *Fs = side ? FR : FL;
            const R *Us = side ? UR : UL;
            // dot_product(leig(k, 1:5), .): row k across the wave columns
            R lf[5], lu[5], lm[5];
#pragma unroll
            for (int j = 0; j < 5; j++) {
                R c[5];
                eig_lcol(e, j, c);
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    lf[k] = (j == 0 ? R(0.) : lf[k]) + c[k] * Fs[j];
                    lu[k] = (j == 0 ? R(0.) : lu[k]) + c[k] * Us[j];
                    if (j == 0 || j == mom) lm[k] = c[k];
                }
            }
            R vec[5];
#pragma unroll
            for (int k = 0; k < 5; k++) {
                const R lk = lam(uL, cL, k), rk = lam(uR, cR, k);
                if (lk * rk > R(0.))
                    vec[k] = ((lk > R(0.)) == (side == 0)) ? lf[k] + lm[k] * Fs[5] : R(0.);
                else if (side == 0)
                    vec[k] = R(0.5) * (lf[k] + amax * lu[k] + lm[k] * Fs[5]);
                else
                    vec[k] = R(0.5) * (lf[k] - amax * lu[k] + lm[k] * Fs[5]);
            }
            R acc[5];
#pragma unroll
            for (int w = 0; w < 5; w++) {
                R c[5];
                eig_rcol(e, w, c);
#pragma unroll
                for (int v = 0; v < 5; v++) acc[v] = (w == 0 ? vec[0] * c[v] : acc[v] + vec[w] * c[v]);
            }
#pragma unroll
            for (int v = 0; v < 5; v++) {
                if (side == 0) part0[v] = acc[v];
                else F[v] = part0[v] + acc[v];
            }
        }
        F[5] = R(0.0);
    } else {
        const R VaL[5] = {Vm[D], Vm[VX], Vm[VY], Vm[VZ], Vm[P]}, VaR[5] = {Vp[D], Vp[VX], Vp[VY], Vp[VZ], Vp[P]};
        const EigC<R> eL = eig_consts(dir, VaL, geL, cL), eR = eig_consts(dir, VaR, geR, cR);
        R sigF[5] = {R(0), R(0), R(0), R(0), R(0)};
#pragma unroll
        for (int k = 0; k < 5; k++) {
            R cr[5], cl[5];
            eig_lcol(eR, k, cr);
            eig_lcol(eL, k, cl);
            R dR = R(0.), dL = R(0.);
#pragma unroll
            for (int v = 0; v < 5; v++) { dR = dR + cr[v] * UR[v]; dL = dL + cl[v] * UL[v]; }
            const R c = R(0.5) * (fabs(lam(uL, cL, k)) + fabs(lam(uR, cR, k)));
            eig_rcol(eR, k, cr);
            eig_rcol(eL, k, cl);
#pragma unroll
            for (int v = 0; v < 5; v++) sigF[v] = sigF[v] + c * (cr[v] * dR - cl[v] * dL);
        }
#pragma unroll
        for (int v = 0; v < 5; v++) F[v] = (FR[v] + FL[v] - sigF[v]) * R(0.5);
        F[5] = (FR[5] + FL[5] - R(0.)) * R(0.5);
    }
    return 0;
}

// shock: the hybrid solver's face is next to a cell the shock detector marked
template <class R, int EXT>
__device__ __forceinline__ int riemann(const DevParams &prm, int dir, const R *Vm, R gcL, R geL,
                                       const R *Vp, R gcR, R geR, R F[8], bool shock = false)
{
    const R velNL = Vm[1 + dir], velNR = Vp[1 + dir];
    const R aL2 = rdiv(gcL * Vm[P], Vm[D]);
    const R aR2 = rdiv(gcR * Vp[P], Vp[D]);
    const bool roe = EXT == 1 && prm.riemann == 1;
    const bool marq = EXT == 2 && (prm.riemann == 5 || prm.riemann == 7);
    // hy_getFaceFlux.F90:364-383: the hybrid solver is HLL next to a marked cell, HLLC elsewhere
    const bool hybr = EXT == 1 && prm.riemann == 8;
    const bool hllc = !roe && !marq && (prm.riemann == 4 || (hybr && !shock)), llf = !roe && !marq && prm.riemann == 2;
    const R tiny = hllc ? R(prm.tiny) : R(1.e-32);
    if ((Vm[D] < tiny && Vm[D] > R(0)) || (Vp[D] < tiny && Vp[D] > R(0)) ||
        (Vm[P] < tiny && Vm[P] > R(0)) || (Vp[P] < tiny && Vp[P] > R(0))) {
#pragma unroll
        for (int k = 0; k < 6; k++) F[k] = R(0);
    } else if (aL2 < R(0) || aR2 < R(0)) {
        return ERR_RIEMANN;
    } else {
        const R cfL = rsqrt_(aL2), cfR = rsqrt_(aR2);
        const R SL = fmin2(velNL - cfL, velNR - cfR);
        const R SR = fmax2(velNL + cfL, velNR + cfR);
        // prim2con / prim2flx (hy_prim2con.F90:48-62, hy_prim2flx.F90:49-95)
        R u2L = Vm[VX] * Vm[VX]; u2L = u2L + Vm[VY] * Vm[VY]; u2L = u2L + Vm[VZ] * Vm[VZ];
        R u2R = Vp[VX] * Vp[VX]; u2R = u2R + Vp[VY] * Vp[VY]; u2R = u2R + Vp[VZ] * Vp[VZ];
        const R EL = R(0.5) * Vm[D] * u2L + rdiv(Vm[P], geL - R(1.));
        const R ER = R(0.5) * Vp[D] * u2R + rdiv(Vp[P], geR - R(1.));
        R UL[5] = {Vm[D], Vm[D] * Vm[VX], Vm[D] * Vm[VY], Vm[D] * Vm[VZ], EL};
        R UR[5] = {Vp[D], Vp[D] * Vp[VX], Vp[D] * Vp[VY], Vp[D] * Vp[VZ], ER};
        const R fP = R(prm.fpres);
        R FL[6], FR[6];
        FL[0] = Vm[D] * velNL; FR[0] = Vp[D] * velNR;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            FL[1 + d] = FL[0] * Vm[1 + d];
            FR[1 + d] = FR[0] * Vp[1 + d];
        }
        FL[1 + dir] = FL[1 + dir] + fP * Vm[P];
        FR[1 + dir] = FR[1 + dir] + fP * Vp[P];
        FL[4] = (EL + Vm[P]) * velNL; FR[4] = (ER + Vp[P]) * velNR;
        FL[5] = Vm[P]; FR[5] = Vp[P];
        if (llf) {
            // hy_LLF.F90:62-183: the largest |eigenvalue| (hy_eigenValue.F90) of the
            // mean state of hy_avgState.F90:34-60 (gamc upwind of its normal
            // velocity) and of the two states, times the conserved jump
            const R un = R(.5) * (velNL + velNR);
            const R sig = un == R(0) ? R(0) : (un > R(0) ? R(1) : R(-1));
            const R gcA = R(0.5) * ((R(1.) + sig) * gcL + (R(1.) - sig) * gcR);
            const R a2 = rdiv(gcA * (R(.5) * (Vm[P] + Vp[P])), R(.5) * (Vm[D] + Vp[D]));
            if (a2 <= R(0) || aL2 <= R(0) || aR2 <= R(0)) return ERR_SOUND;   // hy_eigenParameters aborts
            const R cf = rsqrt_(a2);
            auto maxabs = [](R u, R c) {
                R m = fabs(u - c);
                if (fabs(u) > m) m = fabs(u);
                if (fabs(u + c) > m) m = fabs(u + c);
                return m;
            };
            const R smax = fmax2(fmax2(maxabs(un, cf), maxabs(velNL, cfL)), maxabs(velNR, cfR));
#pragma unroll
            for (int k = 0; k < 5; k++) F[k] = (FR[k] + FL[k] - smax * (UR[k] - UL[k])) * R(0.5);
            F[5] = (FR[5] + FL[5] - smax * (R(0.0) - R(0.0))) * R(0.5);
        } else if (roe) {
            const int e = riemann_roe(dir, prm.entropy_fix, Vm, gcL, geL, Vp, gcR, geR, UL, UR, FL, FR, F);
            if (e) return e;
        } else if (marq) {
            const int e = riemann_marquina(dir, prm.riemann == 7, Vm, gcL, geL, Vp, gcR, geR, UL, UR, FL, FR, F);
            if (e) return e;
        } else if (hllc) {
            R qStar = Vp[D] * velNR * (SR - velNR) - Vm[D] * velNL * (SL - velNL) + Vm[P] - Vp[P];
            qStar = rdiv(qStar, Vp[D] * (SR - velNR) - Vm[D] * (SL - velNL));
            if (SL >= R(0)) {
#pragma unroll
                for (int k = 0; k < 6; k++) F[k] = FL[k];
            } else if (SL < R(0) && qStar >= R(0)) {
                const R numerL = SL - velNL, denomL = SL - qStar;
                const R pStar = Vm[D] * numerL * (qStar - velNL) + Vm[P];
                const R yd = rdiv(R(1), denomL);
                const R dStar = rdiv_y(UL[0] * numerL, denomL, yd);
                R UC[5];
                UC[0] = dStar;
                UC[4] = rdiv_y(UL[4] * numerL, denomL, yd) + rdiv_y(pStar * qStar - Vm[P] * velNL, denomL, yd);
#pragma unroll
                for (int d = 0; d < 3; d++) UC[1 + d] = (d == dir) ? dStar * qStar : rdiv_y(UL[1 + d] * numerL, denomL, yd);
#pragma unroll
                for (int k = 0; k < 5; k++) F[k] = FL[k] + SL * (UC[k] - UL[k]);
                F[5] = FL[5];
            } else if (qStar < R(0) && SR >= R(0)) {
                const R numerR = SR - velNR, denomR = SR - qStar;
                const R numerL = SL - velNL;
                const R pStar = Vm[D] * numerL * (qStar - velNL) + Vm[P];
                const R yd = rdiv(R(1), denomR);
                const R dStar = rdiv_y(UR[0] * numerR, denomR, yd);
                R UC[5];
                UC[0] = dStar;
                UC[4] = rdiv_y(UR[4] * numerR, denomR, yd) + rdiv_y(pStar * qStar - Vp[P] * velNR, denomR, yd);
#pragma unroll
                for (int d = 0; d < 3; d++) UC[1 + d] = (d == dir) ? dStar * qStar : rdiv_y(UR[1 + d] * numerR, denomR, yd);
#pragma unroll
                for (int k = 0; k < 5; k++) F[k] = FR[k] + SR * (UC[k] - UR[k]);
                F[5] = FR[5];
            } else {
#pragma unroll
                for (int k = 0; k < 6; k++) F[k] = FR[k];
            }
        } else {
            if (SL > R(0)) {
#pragma unroll
                for (int k = 0; k < 6; k++) F[k] = FL[k];
            } else if (SR < R(0)) {
#pragma unroll
                for (int k = 0; k < 6; k++) F[k] = FR[k];
            } else {
                const R inv = SR - SL;
#pragma unroll
                for (int k = 0; k < 5; k++) F[k] = rdiv(SR * FL[k] - SL * FR[k] + SR * SL * (UR[k] - UL[k]), inv);
                F[5] = rdiv(SR * FL[5] - SL * FR[5] + SR * SL * (R(0.0) - R(0.0)), inv);
            }
        }
    }
    // aux internal-energy and volume fluxes (hy_getFaceFlux.F90:444-453)
    if (prm.use_aux_eint) {
        if (F[0] > R(0)) { F[FVOL] = rdiv(F[0], Vm[D]); F[FEI] = F[0] * Vm[5]; }
        else             { F[FVOL] = rdiv(F[0], Vp[D]); F[FEI] = F[0] * Vp[5]; }
    } else { F[FVOL] = R(0); F[FEI] = R(0); }
    return 0;
}

// ---- boundary index mapping for guard cells resolved on load ------------------
// Maps a global index g in [-NG, n+NG) of one axis to an interior index;
// *s becomes -1 when a reflecting face flips the normal velocity
// (Grid_bcApplyToRegion.F90:458-531 for OUTFLOW and REFLECTING; periodic wrap
// as the UG exchange of gr_shiftData.F90).
__device__ __forceinline__ int map_axis(int g, int n, int bclo, int bchi, double *s)
{
    if (g < 0) {
        if (bclo == 0) return g + n;
        if (bclo == 1) return 0;
        *s = -1.0; return -1 - g;
    }
    if (g >= n) {
        if (bchi == 0) return g - n;
        if (bchi == 1) return n - 1;
        *s = -1.0; return 2 * n - 1 - g;
    }
    return g;
}

// the shock flag of cell (i, j, k) of the uniform grid, outside the domain
// mapped as the guard fill maps a scalar (SHOK_VAR after Grid_fillGuardCells);
// ny = 1 in 2-D, nz = 1 in 2-D
__device__ __forceinline__ int shock_flag(const unsigned char *shok, int i, int j, int k, int nx, int ny, int nz,
                                          const int *bc)
{
    double s;
    const int mi = map_axis(i, nx, bc[0], bc[1], &s);
    const int mj = ny > 1 ? map_axis(j, ny, bc[2], bc[3], &s) : 0;
    const int mk = nz > 1 ? map_axis(k, nz, bc[4], bc[5], &s) : 0;
    return shok[((long)mk * ny + mj) * nx + mi];
}

} // namespace fxb
