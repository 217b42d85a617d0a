// fxb_species.cuh -- species and mass scalars advected with the unsplit step
// on a uniform grid (hy_fullSpecMsFluxHandling = .true., the default of
// unsplit/Config:165).
//
// The mass fractions ride on the hydro solve: they are reconstructed along
// each direction and traced with the entropy-wave speed (the cell's normal
// velocity), corrected by upwinded transverse terms (and in 3-D by the CTU
// cross terms, or reset to the cell value where the hydro face states fell
// back to first order), and fluxed with the hydro mass flux of every face
// from the upwind side.  Three kernels after the hydro step:
//   spec_sig     sigma_d of every cell of the grid padded by one layer
//                (hy_upwindTransverseFlux.F90:213-221, speciesScalar)
//   spec_states  left/right face values of every face-state cell of each
//                direction: PPM (minmod slopes, hy_DataReconstructNormalDir_
//                PPM.F90:595-643), WENO5 (_WENO.F90:601-691) or MUSCL-Hancock
//                (_MH.F90:369-388); transverse terms (hy_dataReconstOneStep.
//                F90:1007-1041); 3-D CTU terms or fallback (hy_getRiemannState.
//                F90:1063-1100, :1467-1486)
//   spec_update  F = F_dens x upwind face value (hy_getFaceFlux.F90:464-477);
//                X = (X rho_old + dt sum (F_L - F_R) / dx) / rho_new, then the
//                species (not the mass scalars) renormalised
//                (hy_unsplitUpdate.F90:846-881, :1308-1326)
// The hydro kernels provide the mass fluxes (the 3-D flux arrays; the 2-D
// kernel stores them when species are on) and, in 3-D, a byte per face-state
// cell and direction where the CTU fallback fired.
#pragma once
#include "fxb_device.cuh"
#include "fxb_hydro3d.cuh"

namespace fxb {

struct SpecArgs {
    const double *st_old, *st_new;   // hydro state before and after the step ([var][cell], vstride)
    long vstride;
    const double *sp_in;             // mass fractions [ns][cell] (vstride apart) before the step
    double *sp_out;                  // and after it
    int ns, nsp;                     // values per cell; the first nsp are species
    int ndim, nx, ny, nz;
    int bc[6];
    double dx, dy, dz;
    double dt_arg;
    const double *dtv;
    DevParams prm;
    const void *fd[3];               // mass flux of every face of direction d (Grid3::fidx), type R
    const void *flat;                // flattening coefficients of the hydro step (padded box), type R
    const unsigned char *ctufb[3];   // 3-D: CTU fallback of each face-state cell (Grid3::widx)
    void *sg;                        // [3][ns][npad] of R
    void *sl, *sr;                   // [3][ns][nwmax] of R
    long npad, nwmax;
};

// mass fraction n of a possibly virtual cell (boundary conditions without
// sign flips), and the velocity component d there (normal component flipped
// at reflecting faces, as the guard fill does)
template <class R>
__device__ __forceinline__ R spec_at(const SpecArgs &a, int n, int i, int j, int k)
{
    double s_ = 1.0;
    const int mi = map_axis(i, a.nx, a.bc[0], a.bc[1], &s_);
    const int mj = a.ndim >= 2 ? map_axis(j, a.ny, a.bc[2], a.bc[3], &s_) : 0;
    const int mk = a.ndim == 3 ? map_axis(k, a.nz, a.bc[4], a.bc[5], &s_) : 0;
    return (R)__ldg(a.sp_in + n * a.vstride + ((long)mk * a.ny + mj) * a.nx + mi);
}
template <class R>
__device__ __forceinline__ R vel_at(const SpecArgs &a, int d, int i, int j, int k)
{
    double sx = 1.0, sy = 1.0, sz = 1.0;
    const int mi = map_axis(i, a.nx, a.bc[0], a.bc[1], &sx);
    const int mj = a.ndim >= 2 ? map_axis(j, a.ny, a.bc[2], a.bc[3], &sy) : 0;
    const int mk = a.ndim == 3 ? map_axis(k, a.nz, a.bc[4], a.bc[5], &sz) : 0;
    const double v = __ldg(a.st_old + (VX + d) * a.vstride + ((long)mk * a.ny + mj) * a.nx + mi);
    return (R)(d == 0 ? v * sx : d == 1 ? v * sy : v * sz);
}

__device__ __forceinline__ long spec_pidx(const SpecArgs &a, int i, int j, int k)
{
    return a.ndim == 3 ? (((long)(k + 1) * (a.ny + 2) + (j + 1)) * (a.nx + 2) + (i + 1))
                       : ((long)(j + 1) * (a.nx + 2) + (i + 1));
}

// ---- sigma_d of every padded cell ------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) spec_sig_kernel(const SpecArgs a)
{
    R *sg = (R *)a.sg;
    const int px = a.nx + 2, py = a.ny + 2;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < a.npad; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % px) - 1, j = (int)((t / px) % py) - 1, k = a.ndim == 3 ? (int)(t / ((long)px * py)) - 1 : 0;
        for (int d = 0; d < a.ndim; d++) {
            const int di = d == 0, dj = d == 1, dk = d == 2;
            const R lam = vel_at<R>(a, d, i, j, k);
            for (int n = 0; n < a.ns; n++) {
                const R sm = spec_at<R>(a, n, i - di, j - dj, k - dk), sc = spec_at<R>(a, n, i, j, k),
                        sp = spec_at<R>(a, n, i + di, j + dj, k + dk);
                const R tt = lam > R(0) ? sc - sm : sp - sc;
                sg[((long)d * a.ns + n) * a.npad + t] = lam * tt;
            }
        }
    }
}

// one mass fraction's face values along a direction: s[0..4] = cells -2..2
template <class R>
__device__ __forceinline__ void spec_recon(const DevParams &prm, const R s[5], R lam, R hdtn, R flat, R &SLo, R &SRo)
{
    R Sl, Sr;
    const R Sc = s[2], Sm = s[1], Sp = s[3];
    if (prm.order == 2) {
        const R db = lim_mc(Sc - Sm, Sp - Sc);
        Sr = Sc + R(0.5) * db;
        Sr = Sr - fmax2(lam, R(0)) * hdtn * db;
        Sl = Sc - R(0.5) * db;
        Sl = Sl - fmin2(lam, R(0)) * hdtn * db;
        Sr = fmax2(fmin2(Sc, Sr), fmin2(fmax2(Sc, Sr), Sr));
        Sl = fmax2(fmin2(Sc, Sl), fmin2(fmax2(Sc, Sl), Sl));
        SLo = Sl; SRo = Sr;
        return;
    }
    if (prm.order == 5) {
        weno_scalar(prm.weno_method, s[0], s[1], s[2], s[3], s[4], Sr, Sl);
    } else {
        const R dP = lim_minmod(s[3] - s[2], s[4] - s[3]);
        const R d0 = lim_minmod(s[2] - s[1], s[3] - s[2]);
        const R dN = lim_minmod(s[1] - s[0], s[2] - s[1]);
        Sl = R(0.5) * (Sc + Sm) - divk<6>(d0 - dN);
        Sr = R(0.5) * (Sc + Sp) - divk<6>(dP - d0);
        Sl = fmax2(fmin2(Sc, Sm), fmin2(fmax2(Sc, Sm), Sl));
        Sr = fmax2(fmin2(Sc, Sp), fmin2(fmax2(Sc, Sp), Sr));
        if ((Sr - Sc) * (Sc - Sl) <= R(0)) { Sr = Sc; Sl = Sc; }
    }
    if (R(6.) * (Sr - Sl) * (Sc - R(0.5) * (Sr + Sl)) > (Sr - Sl) * (Sr - Sl)) Sl = R(3.) * Sc - R(2.) * Sr;
    if (R(6.) * (Sr - Sl) * (Sc - R(0.5) * (Sr + Sl)) < -((Sr - Sl) * (Sr - Sl))) Sr = R(3.) * Sc - R(2.) * Sl;
    const R del0 = Sr - Sl;
    const R S6 = R(6.) * (Sc - R(0.5) * (Sr + Sl));
    const R lmn = fmin2(lam, R(0)), lmx = fmax2(lam, R(0));
    Sl = Sl - lmn * hdtn * (del0 + (R(1.) + divk<3>(lmn * R(4.)) * hdtn) * S6);
    Sr = Sr - lmx * hdtn * (del0 - (R(1.) - divk<3>(lmx * R(4.)) * hdtn) * S6);
    if (prm.flattening) {
        Sl = flat * Sc + (R(1.0) - flat) * Sl;
        Sr = flat * Sc + (R(1.0) - flat) * Sr;
    }
    SLo = Sl; SRo = Sr;
}

// number of face-state cells of direction d: coordinate d in [-1, n_d], the others interior
__device__ __forceinline__ long spec_nw(const SpecArgs &a, int d)
{
    const long nz = a.ndim == 3 ? a.nz : 1;
    return d == 0 ? (long)(a.nx + 2) * a.ny * nz : d == 1 ? (long)a.nx * (a.ny + 2) * nz : (long)a.nx * a.ny * (a.nz + 2);
}

// ---- face values of every face-state cell, all directions ----------------------
template <class R>
__global__ void __launch_bounds__(256) spec_states_kernel(const SpecArgs a)
{
    const R *sg = (const R *)a.sg;
    R *sl = (R *)a.sl, *sr = (R *)a.sr;
    const double dt = a.dtv ? a.dtv[0] : a.dt_arg;
    const double del[3] = {a.dx, a.dy, a.dz};
    const R hdtx = R(0.5 * dt / a.dx), hdty = R(0.5 * dt / a.dy), hdtz = R(0.5 * dt / a.dz);
    const Grid3 G{a.nx, a.ny, a.ndim == 3 ? a.nz : 1};
    for (int d = 0; d < a.ndim; d++) {
        const long nw = spec_nw(a, d);
        const int ex = a.nx + (d == 0 ? 2 : 0), ey = a.ny + (d == 1 ? 2 : 0);
        const R hdtn = R(0.5 * (dt / del[d]));
        const int di = d == 0, dj = d == 1, dk = d == 2;
        for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nw; t += (long)gridDim.x * blockDim.x) {
            int i = (int)(t % ex), j = (int)((t / ex) % ey), k = (int)(t / ((long)ex * ey));
            if (d == 0) i -= 1; else if (d == 1) j -= 1; else k -= 1;
            const long pc = spec_pidx(a, i, j, k);
            const R lam = vel_at<R>(a, d, i, j, k);
            const R flat = a.prm.flattening ? ((const R *)a.flat)[d * a.npad + pc] : R(0);
            int e1 = 0, s1 = 0, e2 = 0, s2 = 0;
            double fac = 0.;
            bool ctu = false, fb = false;
            if (a.ndim == 3 && a.prm.use_3d_full_ctu) {
                ctu = true;
                if (d == 0)      { e1 = 1; s1 = 2; e2 = 2; s2 = 1; fac = dt * dt / (6. * a.dy * a.dz); }
                else if (d == 1) { e1 = 2; s1 = 0; e2 = 0; s2 = 2; fac = dt * dt / (6. * a.dz * a.dx); }
                else             { e1 = 0; s1 = 1; e2 = 1; s2 = 0; fac = dt * dt / (6. * a.dx * a.dy); }
                fb = a.ctufb[d][G.widx(d, i, j, k)] != 0;
            }
            for (int n = 0; n < a.ns; n++) {
                R st[5];
                st[1] = spec_at<R>(a, n, i - di, j - dj, k - dk);
                st[2] = spec_at<R>(a, n, i, j, k);
                st[3] = spec_at<R>(a, n, i + di, j + dj, k + dk);
                st[0] = a.prm.order == 2 ? R(0) : spec_at<R>(a, n, i - 2 * di, j - 2 * dj, k - 2 * dk);
                st[4] = a.prm.order == 2 ? R(0) : spec_at<R>(a, n, i + 2 * di, j + 2 * dj, k + 2 * dk);
                R SL, SR;
                spec_recon(a.prm, st, lam, hdtn, flat, SL, SR);
                const R *g0 = sg + (long)(0 * a.ns + n) * a.npad, *g1 = sg + (long)(1 * a.ns + n) * a.npad;
                if (d == 0) {
                    SL = SL - hdty * g1[pc]; SR = SR - hdty * g1[pc];
                } else if (d == 1) {
                    SL = SL - hdtx * g0[pc]; SR = SR - hdtx * g0[pc];
                }
                if (a.ndim == 3) {
                    const R *g2 = sg + (long)(2 * a.ns + n) * a.npad;
                    if (d == 0 || d == 1) {
                        SL = SL - hdtz * g2[pc]; SR = SR - hdtz * g2[pc];
                    } else {
                        SL = SL - hdtx * g0[pc] - hdty * g1[pc];
                        SR = SR - hdtx * g0[pc] - hdty * g1[pc];
                    }
                }
                if (ctu) {
                    if (fb) {   // fallbackToFirstOrder: the cell's own value
                        SL = st[2]; SR = st[2];
                    } else {
                        R T[2];
                        const int es[2] = {e1, e2}, ss[2] = {s1, s2};
#pragma unroll
                        for (int r = 0; r < 2; r++) {
                            const int e = es[r];
                            const R *gs = sg + (long)(ss[r] * a.ns + n) * a.npad;
                            const R le = vel_at<R>(a, e, i, j, k);
                            const R vm = gs[spec_pidx(a, i - (e == 0), j - (e == 1), k - (e == 2))];
                            const R vc = gs[pc];
                            const R vp = gs[spec_pidx(a, i + (e == 0), j + (e == 1), k + (e == 2))];
                            const R tt = le > R(0) ? vc - vm : vp - vc;
                            T[r] = le * tt;
                        }
                        const R f = R(fac);
                        SR = SR + (T[0] + T[1]) * f;
                        SL = SL + (T[0] + T[1]) * f;
                    }
                }
                sl[((long)d * a.ns + n) * a.nwmax + t] = SL;
                sr[((long)d * a.ns + n) * a.nwmax + t] = SR;
            }
        }
    }
}

// ---- fluxes and update of every interior cell -----------------------------------
template <class R>
__global__ void __launch_bounds__(256) spec_update_kernel(const SpecArgs a)
{
    const R *sl = (const R *)a.sl, *sr = (const R *)a.sr;
    const double dt = a.dtv ? a.dtv[0] : a.dt_arg;
    const double del[3] = {a.dx, a.dy, a.dz};
    const Grid3 G{a.nx, a.ny, a.ndim == 3 ? a.nz : 1};
    const long ncell = (long)a.nx * a.ny * (a.ndim == 3 ? a.nz : 1);
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < ncell; c += (long)gridDim.x * blockDim.x) {
        const int i = (int)(c % a.nx), j = (int)((c / a.nx) % a.ny), k = (int)(c / ((long)a.nx * a.ny));
        const double dold = a.st_old[D * a.vstride + c], dnew = a.st_new[D * a.vstride + c];
        double sum = 0.;
        for (int n = 0; n < a.ns; n++) {
            double FL[3], FR[3];
            for (int d = 0; d < a.ndim; d++) {
                const int di = d == 0, dj = d == 1, dk = d == 2;
                const R *f = (const R *)a.fd[d];
                const R *L = sl + ((long)d * a.ns + n) * a.nwmax, *Rr = sr + ((long)d * a.ns + n) * a.nwmax;
                // face between cell c - e_d and c, and between c and c + e_d
                const double fl = (double)f[G.fidx(d, i, j, k)], fr = (double)f[G.fidx(d, i + di, j + dj, k + dk)];
                FL[d] = fl < 0. ? fl * (double)L[G.widx(d, i, j, k)] : fl * (double)Rr[G.widx(d, i - di, j - dj, k - dk)];
                FR[d] = fr < 0. ? fr * (double)L[G.widx(d, i + di, j + dj, k + dk)] : fr * (double)Rr[G.widx(d, i, j, k)];
            }
            const double x0 = a.sp_in[n * a.vstride + c];
            double x;
            if (a.ndim == 2) x = (x0 * dold + dt * ((FL[0] - FR[0]) / del[0] + (FL[1] - FR[1]) / del[1])) / dnew;
            else x = (x0 * dold + dt * ((FL[0] - FR[0]) / del[0] + (FL[1] - FR[1]) / del[1] + (FL[2] - FR[2]) / del[2])) / dnew;
            a.sp_out[n * a.vstride + c] = x;
            if (n < a.nsp) sum = sum + x;
        }
        for (int n = 0; n < a.nsp; n++) a.sp_out[n * a.vstride + c] = a.sp_out[n * a.vstride + c] / sum;
    }
}

template <class R> void launch_species_t(const SpecArgs &a, cudaStream_t s)
{
    const int nb = 148 * 8;
    spec_sig_kernel<R><<<nb, 256, 0, s>>>(a);
    spec_states_kernel<R><<<nb, 256, 0, s>>>(a);
    spec_update_kernel<R><<<nb, 256, 0, s>>>(a);
}

} // namespace fxb
