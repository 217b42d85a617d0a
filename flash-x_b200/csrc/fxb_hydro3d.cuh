// fxb_hydro3d.cuh -- 3-D unsplit hydro step with full CTU corner coupling.
//
// Four kernels per step, one thread per cell or face, intermediates in HBM:
//   sig3d     sigma_d (upwind transverse flux, hy_upwindTransverseFlux) of every
//             cell of the grid padded by one layer, for d = x, y, z
//   states3d  face states of one sweep direction: PPM/WENO + characteristic
//             tracing, minus dt/2 * the other two sigmas, negativity fallback,
//             gravity half-update, then the 3-D CTU cross terms built from the
//             neighbours' sigmas (hy_getRiemannState.F90:963-1338)
//   flux3d    HLLC/HLL on every face of one direction (hy_getFaceFlux.F90)
//   update3d  conserved + aux-eint update, gravity half steps
//             (hy_unsplitUpdate.F90:1195-1250, hy_addGravity.F90), energyFix,
//             Eos, store, CFL rate
// Guard cells are resolved on load through map_axis, as in the 2-D kernel.
#pragma once
#include "fxb_device.cuh"

namespace fxb {

struct Args3D {
    const double *in;
    double *out;
    long vstride;
    int nx, ny, nz;
    int bc[6];
    double dx, dy, dz;
    double dt_arg;
    const double *dtv;
    double gam1inv, ggprodinv;
    DevParams prm;
    unsigned long long *rate_max;
    int *err;
    void *sig;      // [3][6][(nx+2)(ny+2)(nz+2)] of R
    void *wst[3];   // per direction [12][cells with that coordinate in [-1, n]]
    void *flx[3];   // per direction [8][faces]
};

// 3-D tile extents accepted by fxb_init (the unfused kernels take any size)
constexpr int T3X = 1, T3Y = 1, T3Z = 1;

struct Grid3 {
    int nx, ny, nz;
    __device__ long npad() const { return (long)(nx + 2) * (ny + 2) * (nz + 2); }
    __device__ long pidx(int i, int j, int k) const { return ((long)(k + 1) * (ny + 2) + (j + 1)) * (nx + 2) + (i + 1); }
    // state cells of direction d: coordinate d in [-1, n_d], the others interior
    __device__ long nw(int d) const {
        return d == 0 ? (long)(nx + 2) * ny * nz : d == 1 ? (long)nx * (ny + 2) * nz : (long)nx * ny * (nz + 2);
    }
    __device__ long widx(int d, int i, int j, int k) const {
        if (d == 0) return ((long)k * ny + j) * (nx + 2) + (i + 1);
        if (d == 1) return ((long)k * (ny + 2) + (j + 1)) * nx + i;
        return ((long)(k + 1) * ny + j) * nx + i;
    }
    __device__ long nf(int d) const {
        return d == 0 ? (long)(nx + 1) * ny * nz : d == 1 ? (long)nx * (ny + 1) * nz : (long)nx * ny * (nz + 1);
    }
    __device__ long fidx(int d, int i, int j, int k) const {
        if (d == 0) return ((long)k * ny + j) * (nx + 1) + i;
        if (d == 1) return ((long)k * (ny + 1) + j) * nx + i;
        return ((long)k * ny + j) * nx + i;
    }
};

// primitive 8-vector (D,VX,VY,VZ,P,GC,GE,EI) of a possibly virtual cell
template <class R>
__device__ __forceinline__ void load_cell(const Args3D &a, int i, int j, int k, R v[8])
{
    double sx = 1.0, sy = 1.0, sz = 1.0;
    int mi = map_axis(i, a.nx, a.bc[0], a.bc[1], &sx);
    int mj = map_axis(j, a.ny, a.bc[2], a.bc[3], &sy);
    int mk = map_axis(k, a.nz, a.bc[4], a.bc[5], &sz);
    long c = ((long)mk * a.ny + mj) * a.nx + mi;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        double x = __ldg(a.in + q * a.vstride + c);
        if (q == VX) x = x * sx;
        if (q == VY) x = x * sy;
        if (q == VZ) x = x * sz;
        v[q] = (R)x;
    }
}

template <class R> __device__ __forceinline__ void six(const R v[8], R g[6])
{ g[0] = v[D]; g[1] = v[VX]; g[2] = v[VY]; g[3] = v[VZ]; g[4] = v[P]; g[5] = v[EI]; }

template <class R> __device__ __forceinline__ void rot3(int dir, const R *g, R *r)
{
    r[0] = g[0]; r[4] = g[4]; r[5] = g[5];
    if (dir == 0)      { r[1] = g[1]; r[2] = g[2]; r[3] = g[3]; }
    else if (dir == 1) { r[1] = g[2]; r[2] = g[3]; r[3] = g[1]; }
    else               { r[1] = g[3]; r[2] = g[1]; r[3] = g[2]; }
}
template <class R> __device__ __forceinline__ void unrot3(int dir, const R *r, R *g)
{
    g[0] = r[0]; g[4] = r[4]; g[5] = r[5];
    if (dir == 0)      { g[1] = r[1]; g[2] = r[2]; g[3] = r[3]; }
    else if (dir == 1) { g[2] = r[1]; g[3] = r[2]; g[1] = r[3]; }
    else               { g[3] = r[1]; g[1] = r[2]; g[2] = r[3]; }
}

__device__ __forceinline__ void offs(int d, int o, int &di, int &dj, int &dk)
{ di = d == 0 ? o : 0; dj = d == 1 ? o : 0; dk = d == 2 ? o : 0; }

// ---- sigma_d of every padded cell --------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) sig3d_kernel(const Args3D a)
{
    Grid3 G{a.nx, a.ny, a.nz};
    R *sig = (R *)a.sig;
    const long np = G.npad();
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < np; idx += (long)gridDim.x * blockDim.x) {
        int i = (int)(idx % (a.nx + 2)) - 1;
        int j = (int)((idx / (a.nx + 2)) % (a.ny + 2)) - 1;
        int k = (int)(idx / ((long)(a.nx + 2) * (a.ny + 2))) - 1;
        R vc[8];
        load_cell(a, i, j, k, vc);
        R gc[6]; six(vc, gc);
        for (int d = 0; d < 3; d++) {
            int di, dj, dk;
            offs(d, 1, di, dj, dk);
            R vm[8], vp[8], g[6], m[6], c[6], p[6], sr[6], sg[6];
            load_cell(a, i - di, j - dj, k - dk, vm);
            load_cell(a, i + di, j + dj, k + dk, vp);
            six(vm, g); rot3(d, g, m);
            rot3(d, gc, c);
            six(vp, g); rot3(d, g, p);
            Eig<R> e;
            if (!eigen(c[0], c[1], c[4], vc[GC], e)) atomicOr(a.err, ERR_SOUND);
            trans_flux(e, m, c, p, a.prm.use_aux_eint != 0, sr);
            unrot3(d, sr, sg);
#pragma unroll
            for (int q = 0; q < 6; q++) sig[((long)d * 6 + q) * np + idx] = sg[q];
        }
    }
}

template <class R>
__device__ __forceinline__ void read_sig(const Args3D &a, const Grid3 &G, int d, int i, int j, int k, R s[6])
{
    const R *sig = (const R *)a.sig;
    long np = G.npad(), p = G.pidx(i, j, k);
#pragma unroll
    for (int q = 0; q < 6; q++) s[q] = sig[((long)d * 6 + q) * np + p];
}

// CTU cross term of one transverse pair: upwinding along e of sigma_s at the
// cell's e-neighbours, with the e-direction eigensystem of the cell
template <class R>
__device__ __forceinline__ void ctu_term(const Args3D &a, const Grid3 &G, const R vc[8], int e, int s,
                                        int i, int j, int k, R T[6])
{
    int di, dj, dk;
    offs(e, 1, di, dj, dk);
    R sm[6], sc[6], sp[6], m[6], c[6], p[6], gcell[6], r[6], tr[6];
    read_sig(a, G, s, i - di, j - dj, k - dk, sm);
    read_sig(a, G, s, i, j, k, sc);
    read_sig(a, G, s, i + di, j + dj, k + dk, sp);
    rot3(e, sm, m); rot3(e, sc, c); rot3(e, sp, p);
    six(vc, gcell); rot3(e, gcell, r);
    Eig<R> ev;
    if (!eigen(r[0], r[1], r[4], vc[GC], ev)) atomicOr(a.err, ERR_SOUND);
    trans_flux(ev, m, c, p, a.prm.use_aux_eint != 0, tr);
    unrot3(e, tr, T);
}

// ---- face states of direction d ------------------------------------------------
// One instantiation per reconstruction order, so the register allocation of
// the PPM path (three eigensystems and slopes) and of the WENO path (one
// eigensystem, five projected cells) do not add up.  The minimum number of
// resident 256-thread CTAs per SM bounds the registers per thread: two CTAs
// (128 registers, a few hundred bytes of spills in FP64) measured 18 % faster
// on B200 than one CTA with 244-255 registers, and three CTAs (80 registers)
// lost again to spill traffic.
#ifndef FXB_S3_MINB_FP64
#define FXB_S3_MINB_FP64 2
#endif
#ifndef FXB_S3_MINB_FP32
#define FXB_S3_MINB_FP32 2
#endif
template <class R> struct MinB3D { static constexpr int value = sizeof(R) == 8 ? FXB_S3_MINB_FP64 : FXB_S3_MINB_FP32; };
template <class R, int ORDER>
__global__ void __launch_bounds__(256, MinB3D<R>::value) states3d_kernel(const Args3D a, int d)
{
    Grid3 G{a.nx, a.ny, a.nz};
    const double dt = a.dtv ? a.dtv[0] : a.dt_arg;
    const double del[3] = {a.dx, a.dy, a.dz};
    const R dtn = R(dt / del[d]), hdtn = R(0.5 * (dt / del[d]));
    const R hdtx = R(0.5 * dt / a.dx), hdty = R(0.5 * dt / a.dy), hdtz = R(0.5 * dt / a.dz);
    R *w = (R *)a.wst[d];
    const long nw = G.nw(d);
    const int lx = a.nx + (d == 0 ? 2 : 0), ly = a.ny + (d == 1 ? 2 : 0);
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < nw; idx += (long)gridDim.x * blockDim.x) {
        int i = (int)(idx % lx), j = (int)((idx / lx) % ly), k = (int)(idx / ((long)lx * ly));
        if (d == 0) i -= 1; else if (d == 1) j -= 1; else k -= 1;
        int di, dj, dk;
        offs(d, 1, di, dj, dk);
        R S8[5][8], S[5][6], g[6];
#pragma unroll
        for (int o = -2; o <= 2; o++) {
            load_cell(a, i + o * di, j + o * dj, k + o * dk, S8[o + 2]);
            six(S8[o + 2], g); rot3(d, g, S[o + 2]);
        }
        const R *vc = S8[2];
        Eig<R> e;
        if (!eigen(S[2][0], S[2][1], S[2][4], vc[GC], e)) atomicOr(a.err, ERR_SOUND);
        R vecL[6], vecR[6];
        if constexpr (ORDER == 5) {
            weno_interfaces(a.prm, e, S, vecL, vecR);
        } else {
            Eig<R> eN, eP;
            if (!eigen(S[1][0], S[1][1], S[1][4], S8[1][GC], eN)) atomicOr(a.err, ERR_SOUND);
            if (!eigen(S[3][0], S[3][1], S[3][4], S8[3][GC], eP)) atomicOr(a.err, ERR_SOUND);
            R dbN[6], db0[6], dbP[6];
            tvd_slope(a.prm, eN, S[0], S[1], S[2], dbN);
            tvd_slope(a.prm, e, S[1], S[2], S[3], db0);
            tvd_slope(a.prm, eP, S[2], S[3], S[4], dbP);
            ppm_interfaces(S[1], S[2], S[3], dbN, db0, dbP, vecL, vecR);
        }
        R wm[6], wp[6], Wm[6], Wp[6];
        ppm_trace(e, dtn, hdtn, S[2], vecL, vecR, wm, wp);
        unrot3(d, wm, Wm); unrot3(d, wp, Wp);
        // transverse terms, hy_dataReconstOneStep.F90:931-962
        R s1[6], s2[6];
        if (d == 0) {
            read_sig(a, G, 1, i, j, k, s1); read_sig(a, G, 2, i, j, k, s2);
#pragma unroll
            for (int q = 0; q < 6; q++) {
                Wm[q] = Wm[q] - hdty * s1[q]; Wp[q] = Wp[q] - hdty * s1[q];
                Wm[q] = Wm[q] - hdtz * s2[q]; Wp[q] = Wp[q] - hdtz * s2[q];
            }
        } else if (d == 1) {
            read_sig(a, G, 0, i, j, k, s1); read_sig(a, G, 2, i, j, k, s2);
#pragma unroll
            for (int q = 0; q < 6; q++) {
                Wm[q] = Wm[q] - hdtx * s1[q]; Wp[q] = Wp[q] - hdtx * s1[q];
                Wm[q] = Wm[q] - hdtz * s2[q]; Wp[q] = Wp[q] - hdtz * s2[q];
            }
        } else {
            read_sig(a, G, 0, i, j, k, s1); read_sig(a, G, 1, i, j, k, s2);
#pragma unroll
            for (int q = 0; q < 6; q++) {
                Wm[q] = Wm[q] - hdtx * s1[q] - hdty * s2[q];
                Wp[q] = Wp[q] - hdtx * s1[q] - hdty * s2[q];
            }
        }
        R gvc[6]; six(vc, gvc);
        if (Wm[0] < R(0) || Wp[0] < R(0) || Wm[4] < R(0) || Wp[4] < R(0)) {
#pragma unroll
            for (int q = 0; q < 6; q++) { Wm[q] = gvc[q]; Wp[q] = gvc[q]; }
        }
        if (a.prm.use_gravity) {   // hy_getRiemannState.F90:843-885
            const R hdt = R(0.5 * dt);
            R gl, gr;
            gravity_faces(a.prm, R(a.prm.grav[d]), gl, gr);
#pragma unroll
            for (int q = 0; q < 3; q++) {
                R gp = q == d ? gr : R(a.prm.grav[q]);
                R gn = q == d ? gl : R(a.prm.grav[q]);
                Wp[1 + q] = Wp[1 + q] + hdt * gp;
                Wm[1 + q] = Wm[1 + q] + hdt * gn;
            }
        }
        if (a.prm.use_3d_full_ctu) {
            int e1, s1d, e2, s2d; double fac;
            if (d == 0)      { e1 = 1; s1d = 2; e2 = 2; s2d = 1; fac = dt * dt / (6. * a.dy * a.dz); }
            else if (d == 1) { e1 = 2; s1d = 0; e2 = 0; s2d = 2; fac = dt * dt / (6. * a.dz * a.dx); }
            else             { e1 = 0; s1d = 1; e2 = 1; s2d = 0; fac = dt * dt / (6. * a.dx * a.dy); }
            R T1[6], T2[6];
            ctu_term(a, G, vc, e1, s1d, i, j, k, T1);
            ctu_term(a, G, vc, e2, s2d, i, j, k, T2);
            const R f = R(fac);
#pragma unroll
            for (int q = 0; q < 6; q++) {
                Wp[q] = Wp[q] + (T1[q] + T2[q]) * f;
                Wm[q] = Wm[q] + (T1[q] + T2[q]) * f;
            }
            if (Wp[0] <= R(0) || Wm[0] <= R(0) || Wp[4] <= R(0) || Wm[4] <= R(0)) {
#pragma unroll
                for (int q = 0; q < 6; q++) { Wm[q] = gvc[q]; Wp[q] = gvc[q]; }
            }
        }
#pragma unroll
        for (int q = 0; q < 6; q++) { w[(long)q * nw + idx] = Wp[q]; w[(long)(6 + q) * nw + idx] = Wm[q]; }
    }
}

// ---- Riemann fluxes of direction d ---------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) flux3d_kernel(const Args3D a, int d)
{
    Grid3 G{a.nx, a.ny, a.nz};
    const R *w = (const R *)a.wst[d];
    R *f = (R *)a.flx[d];
    const long nf = G.nf(d), nw = G.nw(d);
    const int lx = a.nx + (d == 0 ? 1 : 0), ly = a.ny + (d == 1 ? 1 : 0);
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < nf; idx += (long)gridDim.x * blockDim.x) {
        int i = (int)(idx % lx), j = (int)((idx / lx) % ly), k = (int)(idx / ((long)lx * ly));
        int di, dj, dk;
        offs(d, 1, di, dj, dk);
        long wl = G.widx(d, i - di, j - dj, k - dk), wr = G.widx(d, i, j, k);
        R VL[6], VR[6], F[8], cl[8], cr[8];
#pragma unroll
        for (int q = 0; q < 6; q++) { VL[q] = w[(long)q * nw + wl]; VR[q] = w[(long)(6 + q) * nw + wr]; }
        load_cell(a, i - di, j - dj, k - dk, cl);
        load_cell(a, i, j, k, cr);
        int e = riemann(a.prm, d, VL, cl[GC], cl[GE], VR, cr[GC], cr[GE], F);
        if (e) atomicOr(a.err, e);
#pragma unroll
        for (int q = 0; q < NF; q++) f[(long)q * nf + idx] = F[q];
    }
}

// ---- update, energyFix, Eos, CFL rate -------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) update3d_kernel(const Args3D a)
{
    Grid3 G{a.nx, a.ny, a.nz};
    const double dt = a.dtv ? a.dtv[0] : a.dt_arg;
    const DevParams &prm = a.prm;
    const long n = (long)a.nx * a.ny * a.nz;
    const double del[3] = {a.dx, a.dy, a.dz};
    double rate = 0.;
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        int i = (int)(c % a.nx), j = (int)((c / a.nx) % a.ny), k = (int)(c / ((long)a.nx * a.ny));
        const long vs = a.vstride;
        double dens0 = a.in[D * vs + c];
        double vx0 = a.in[VX * vs + c], vy0 = a.in[VY * vs + c], vz0 = a.in[VZ * vs + c];
        double en0 = a.in[DV_ENER * vs + c], eint0 = a.in[EI * vs + c];
        double U0[5] = {dens0, vx0 * dens0, vy0 * dens0, vz0 * dens0, dens0 * en0};
        double Sph[5] = {0., 0., 0., 0., 0.};
        double A[3], B[3], pav = 0.;
        for (int d = 0; d < 3; d++) {
            const R *f = (const R *)a.flx[d];
            const R *w = (const R *)a.wst[d];
            long nf = G.nf(d), nw = G.nw(d);
            int di, dj, dk;
            offs(d, 1, di, dj, dk);
            long fl = G.fidx(d, i, j, k), fr = G.fidx(d, i + di, j + dj, k + dk);
            double dtdl = dt / del[d];
#pragma unroll
            for (int v = 0; v < 5; v++)
                U0[v] = U0[v] - dtdl * ((double)f[(long)v * nf + fr] - (double)f[(long)v * nf + fl]);
            A[d] = (double)f[(long)FEI * nf + fl] - (double)f[(long)FEI * nf + fr];
            B[d] = (double)f[(long)FVOL * nf + fl] - (double)f[(long)FVOL * nf + fr];
            Sph[1 + d] = ((double)f[(long)FP * nf + fl] - (double)f[(long)FP * nf + fr]) * (1.0 - prm.fpres) / del[d];
            long wc = G.widx(d, i, j, k);
            double sum = (double)w[(long)(6 + P) * nw + wc] + (double)w[(long)P * nw + wc];
            if (d == 0) pav = 0.5 * sum;
            else if (d == 1) pav = pav * 0.5 + sum * 0.25;
            else pav = (pav * 4.0 + sum) / 6.0;
        }
        double inten = 0.;
        if (prm.use_aux_eint) {
            inten = dens0 * eint0;
            for (int d = 0; d < 3; d++) inten = inten + dt / del[d] * (A[d] + pav * B[d]);
            inten = inten + dt * 0.0;
        }
        const double momOld[3] = {vx0 * dens0, vy0 * dens0, vz0 * dens0};
        for (int v = 0; v < 5; v++) U0[v] = U0[v] + dt * (0. + Sph[v]);
        if (prm.use_gravity) {
            for (int d = 0; d < 3; d++) U0[1 + d] = U0[1 + d] + 0.5 * dt * dens0 * prm.grav[d];
            double dp = 0.;
            for (int d = 0; d < 3; d++) dp = dp + momOld[d] * prm.grav[d];
            U0[4] = U0[4] + 0.5 * dt * dp;
        }
        double dens = fmax2(U0[0], prm.small_dens);
        double vx = U0[1] / dens, vy = U0[2] / dens, vz = U0[3] / dens;
        double ener = U0[4] / dens;
        double eint = prm.use_aux_eint ? inten / dens : eint0;
        if (prm.use_gravity) {   // hy_gravityStepBlk -> hy_addGravity: n+1 half step
            const double hdt = 0.5 * dt;
            double vn[3] = {vx + hdt * prm.grav[0], vy + hdt * prm.grav[1], vz + hdt * prm.grav[2]};
            double dp = 0.;
            for (int d = 0; d < 3; d++) dp = dp + vn[d] * prm.grav[d];
            ener = ener + hdt * dp;
            vx = vn[0]; vy = vn[1]; vz = vn[2];
        }
        double ekin = vx * vx; ekin = ekin + vy * vy; ekin = ekin + vz * vz; ekin = 0.5 * ekin;
        double ee = ener - ekin - 0.0;
        double newE = (!prm.use_aux_eint || ee > prm.eint_switch * (ekin + 0.0)) ? fmax2(prm.small_e, ee)
                                                                                : fmax2(prm.small_e, eint);
        ener = newE + ekin;
        eint = newE;
        double ek2 = 0.5 * (vx * vx + vy * vy + vz * vz);
        double eg = eint;
        if (ener - ek2 > fmax2(prm.small_e, prm.eint_switch * ek2)) eg = ener - ek2;
        double pres = dens * eg * a.gam1inv;
        double temp = eg * a.ggprodinv * prm.abar;
        double game = pres / (eg * dens) + 1;
        double *o = a.out;
        o[D * vs + c] = dens; o[VX * vs + c] = vx; o[VY * vs + c] = vy; o[VZ * vs + c] = vz;
        o[P * vs + c] = pres; o[GC * vs + c] = prm.gamma; o[GE * vs + c] = game;
        o[EI * vs + c] = eg; o[DV_ENER * vs + c] = eg + ek2; o[DV_TEMP * vs + c] = temp;
        double cs = sqrt(prm.gamma * pres / dens);
        double r = (fabs(vx - 0.) + cs) * (1.0 / a.dx);
        r = fmax2(r, (fabs(vy - 0.) + cs) * (1.0 / a.dy));
        r = fmax2(r, (fabs(vz - 0.) + cs) * (1.0 / a.dz));
        rate = fmax2(rate, r);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, off));
    if ((threadIdx.x & 31) == 0) atomicMax(a.rate_max, (unsigned long long)__double_as_longlong(rate));
}

// bytes of the 3-D intermediates for R of the given size
inline size_t sig3d_bytes(int nx, int ny, int nz, size_t rsz)
{ return rsz * 18 * (size_t)(nx + 2) * (ny + 2) * (nz + 2); }
inline size_t w3d_bytes(int d, int nx, int ny, int nz, size_t rsz)
{
    size_t n = d == 0 ? (size_t)(nx + 2) * ny * nz : d == 1 ? (size_t)nx * (ny + 2) * nz : (size_t)nx * ny * (nz + 2);
    return rsz * 12 * n;
}
inline size_t f3d_bytes(int d, int nx, int ny, int nz, size_t rsz)
{
    size_t n = d == 0 ? (size_t)(nx + 1) * ny * nz : d == 1 ? (size_t)nx * (ny + 1) * nz : (size_t)nx * ny * (nz + 1);
    return rsz * 8 * n;
}

template <class R> void launch_hydro3d_t(const Args3D &a, cudaStream_t s)
{
    const int nb = 148 * 8;
    sig3d_kernel<R><<<nb, 256, 0, s>>>(a);
    for (int d = 0; d < 3; d++) {
        if (a.prm.order == 5) states3d_kernel<R, 5><<<nb, 256, 0, s>>>(a, d);
        else states3d_kernel<R, 3><<<nb, 256, 0, s>>>(a, d);
    }
    for (int d = 0; d < 3; d++) flux3d_kernel<R><<<nb, 256, 0, s>>>(a, d);
    update3d_kernel<R><<<nb, 256, 0, s>>>(a);
}

} // namespace fxb
