// fxb_hydro2d.cuh -- fused 2-D unsplit hydro step, one CTA per 16x16 tile.
//
// Replaces, for every leaf block, UHD/hy_computeFluxes.F90:87-417 (with
// Uout => Uin, levelFlux/Hydro.F90:191-212): hy_getRiemannState,
// hy_getFaceFlux, hy_unsplitUpdate, hy_energyFix, Eos_wrapped(MODE_DENS_EI),
// and the per-cell part of Hydro_computeDt.F90:151-242.
//
// Data: one FP64 array per variable over the whole uniform grid (x fastest),
// read from `in` and written to `out` (ping-pong), so blocks need no stored
// guard cells: the load stage resolves every halo cell from the neighbouring
// tile or from the physical boundary condition (map_axis), which is what
// Grid_fillGuardCells followed by the per-block copy would have provided.
//
// Stages (s = shared memory, R = reconstruction type):
//   A  load the 22x22 window (tile + 3 halo) of D,VX,VY,VZ,P,GC,GE,EI -> s.V
//      (tiles whose window lies inside the stored grid: one TMA box
//      [8][22][24] starting one column left of the window, so that its x
//      origin is 16-byte aligned; tiles at the grid's edge: per-thread loads
//      with the boundary conditions resolved by map_axis)
//   B  x: eigensystem + limited slopes of cells i=-2..17, j=0..15      -> s.DB
//   C  x: PPM/WENO face states of i=-1..16, j=0..15, minus dt/2dy*sig_y -> s.W
//   D  x: HLLC/HLL on faces i=0..16                                     -> s.F
//   E  owner threads: x part of the conserved and aux-eint update (registers)
//   F..H the same for y
//   I  owner threads: y update, energyFix, Eos, store, CFL rate max
#pragma once
#include "fxb_device.cuh"
#include "fxb_tma.cuh"

namespace fxb {

struct alignas(64) Args2D {
    CUtensorMap tmap;        // the 8 window variables of `in` as [var][y][x] (built by the host)
    int use_tma;             // stage interior windows by TMA (else per-thread loads everywhere)
    unsigned tma_extra_tx;   // test hook: bytes the barrier expects beyond the box (0)
    long long wait_budget;   // clock cycles a CTA waits for its window before ERR_TIMEOUT
    const double *in;
    double *out;
    long vstride;            // elements between variables
    int nx, ny;
    int bc[4];
    double dx, dy;
    double dt_arg;           // used when dtv == nullptr
    const double *dtv;       // device dt (dtv[0]) for graph-captured loops
    double gam1inv, ggprodinv;
    DevParams prm;
    unsigned long long *rate_max;
    int *err;
    const void *flat;        // flattening coefficients [2][(nx+2)(ny+2)] of R, padded by one cell
    void *fd[2] = {nullptr, nullptr};   // species on: the mass flux of every x / y face, R ((nx+1) ny, nx (ny+1))
    long rate_c0 = 0, rate_c1 = 0x7fffffffffffffffL;   // cells [c0, c1) enter the CFL rate (a slab's own)
    const unsigned char *shok = nullptr;   // shock detector on: the flag of every cell [y][x]
};

constexpr int T2 = 16;             // tile edge
constexpr int WIN = T2 + 6;        // window edge
constexpr int WP = WIN + 2;        // stored row: one column left of the window (TMA x alignment) and one right
constexpr int XO = 1;              // stored column of window column 0
// Threads per CTA.  Two CTAs share an SM's 64K registers, so the count sets
// the register budget.  320 threads (10 warps, 96 registers) measured fastest
// for both precisions on B200: 288 threads (112 registers) cannot place 18
// warps evenly on the four SM sub-partitions and drops to one CTA per SM;
// 256 threads (128 registers, fewer spills) needs a second pass in every
// stage.  Every stage loops, so other counts remain valid.
#ifndef FXB_FP64_THREADS
#define FXB_FP64_THREADS 320
#endif
template <class R> struct Threads2D { static constexpr int value = sizeof(R) == 8 ? FXB_FP64_THREADS : 320; };
// registers per thread for two CTAs per SM (multiple of 8)
template <class R> struct Regs2D { static constexpr int value = (65536 / (2 * Threads2D<R>::value)) / 8 * 8; };
constexpr int NDB = (T2 + 4) * T2; // 320 slope cells
constexpr int NW = (T2 + 2) * T2;  // 288 face-state cells
constexpr int NFC = (T2 + 1) * T2; // 272 faces

// The FP32 path keeps the direction-independent part of each slope cell's
// eigensystem (the four values that cost a square root and three divisions)
// in shared memory for the state stage of the same direction, and the FP64
// update inputs of the owner cells (OWN).  The FP64 path recomputes the
// eigensystem: its 10 KB more shared memory leaves too little L1 for its
// register spills (29 % slower measured on B200).
template <class R> struct KeepOwn { static constexpr bool value = sizeof(R) == 4; };
// FP32 keeps the slope stage's sigma of the other direction in shared memory;
// FP64 recomputes it in the face-state stage from the window (the same
// operations on the same cells): the 15 KB it frees per CTA stay L1, which
// holds the FP64 kernel's register spills
template <class R> struct KeepSig { static constexpr bool value = sizeof(R) == 4; };

constexpr int NOWN = T2 * T2;      // owner cells of a tile

template <class R> struct Smem2D {
    R V[8][WIN][WP];
    R DBF[NF * NFC];               // slopes [6][NDB], then fluxes [8][NFC]
    R SG[6][KeepSig<R>::value ? NDB : 1];   // sigma of the other direction at the slope cells (global order)
    R W[12][NW];                   // Wp (D,VX,VY,VZ,P,EI), then Wm
    R EB[4][KeepOwn<R>::value ? NDB : 1];   // eigensystem base of the slope cells: cf, ahinv, lp, a2inv
    // FP64 update inputs of the owner cells that the window does not hold
    // exactly: ENER, and in the FP32 path also D, VX, VY, VZ, EINT
    double OWN[KeepOwn<R>::value ? 6 : 1][NOWN];
};

// rotate a global-order 6-vector (D,VX,VY,VZ,P,EI) into sweep order
// (D, v_normal, v2, v3, P, EI) with v2/v3 as in hy_eigenVector.F90:67-79
template <class R> __device__ __forceinline__ void rot(int dir, const R *g, R *r)
{
    r[0] = g[0]; r[4] = g[4]; r[5] = g[5];
    if (dir == 0)      { r[1] = g[1]; r[2] = g[2]; r[3] = g[3]; }
    else if (dir == 1) { r[1] = g[2]; r[2] = g[3]; r[3] = g[1]; }
    else               { r[1] = g[3]; r[2] = g[1]; r[3] = g[2]; }
}
template <class R> __device__ __forceinline__ void unrot(int dir, const R *r, R *g)
{
    g[0] = r[0]; g[4] = r[4]; g[5] = r[5];
    if (dir == 0)      { g[1] = r[1]; g[2] = r[2]; g[3] = r[3]; }
    else if (dir == 1) { g[2] = r[1]; g[3] = r[2]; g[1] = r[3]; }
    else               { g[3] = r[1]; g[1] = r[2]; g[2] = r[3]; }
}

template <class R> __device__ __forceinline__ void win6(const Smem2D<R> &s, int wx, int wy, R *g)
{
    g[0] = s.V[D][wy][wx + XO]; g[1] = s.V[VX][wy][wx + XO]; g[2] = s.V[VY][wy][wx + XO];
    g[3] = s.V[VZ][wy][wx + XO]; g[4] = s.V[P][wy][wx + XO]; g[5] = s.V[EI][wy][wx + XO];
}

__device__ __forceinline__ void set_err(int *err, int code) { atomicOr(err, code); }

// the upwind transverse flux sigma of the direction other than dir at window
// cell (wx, wy) (hy_upwindTransverseFlux), g its global-order 6-vector, eb its
// eigensystem base; global order
template <class R>
__device__ __forceinline__ void sigma_other(const Args2D &a, const Smem2D<R> &s, int dir, int wx, int wy, const R g[6],
                                            const EigBase<R> &eb, R sg[6])
{
    const int td = 1 - dir, tx = td == 0, ty = td == 1;
    R gm[6], gp[6], m[6], c[6], p[6], sr[6];
    win6(s, wx - tx, wy - ty, gm); win6(s, wx + tx, wy + ty, gp);
    rot(td, gm, m); rot(td, g, c); rot(td, gp, p);
    Eig<R> et;
    eigen_dir(eb, c[1], et);
    trans_flux(et, m, c, p, a.prm.use_aux_eint != 0, sr);
    unrot(td, sr, sg);
}

// Per-cell analysis along dir at a slope cell: the eigensystem and limited
// slopes (PPM), and the upwind transverse flux sigma of the other direction
// (hy_upwindTransverseFlux), which the state stage of dir subtracts.
template <class R>
__device__ __forceinline__ void analysis_stage(const Args2D &a, Smem2D<R> &s, int dir, int t, int wx, int wy,
                                               bool ppm)
{
    R g[6], c[6];
    win6(s, wx, wy, g);
    // one eigensystem base for the slope direction and the transverse one
    EigBase<R> eb;
    if (!eigen_base(g[0], g[4], s.V[GC][wy][wx + XO], eb)) set_err(a.err, ERR_SOUND);
    if (KeepOwn<R>::value) { s.EB[0][t] = eb.cf; s.EB[1][t] = eb.ahinv; s.EB[2][t] = eb.lp; s.EB[3][t] = eb.a2inv; }
    if (ppm) {
        const int ox = dir == 0, oy = dir == 1;
        R gm[6], gp[6], Vm[6], Vp[6], db[6];
        win6(s, wx - ox, wy - oy, gm); win6(s, wx + ox, wy + oy, gp);
        rot(dir, gm, Vm); rot(dir, g, c); rot(dir, gp, Vp);
        Eig<R> e;
        eigen_dir(eb, c[1], e);
        tvd_slope(a.prm, e, Vm, c, Vp, db);
#pragma unroll
        for (int k = 0; k < 6; k++) s.DBF[k * NDB + t] = db[k];
    }
    if (KeepSig<R>::value) {
        R sg[6];
        sigma_other(a, s, dir, wx, wy, g, eb, sg);
#pragma unroll
        for (int k = 0; k < 6; k++) s.SG[k][t] = sg[k];
    }
}

// velocity component q (VX or VY) of window cell (wx, wy); read from the
// state through the boundary map when it lies outside the window
template <class R> __device__ __forceinline__ R vel2d(const Args2D &a, const Smem2D<R> &s, int q, int wx, int wy)
{
    if (wx >= 0 && wx < WIN && wy >= 0 && wy < WIN) return s.V[q][wy][wx + XO];
    double sx = 1.0, sy = 1.0;
    const int gx = (int)(blockIdx.x * T2) + wx - 3, gy = (int)(blockIdx.y * T2) + wy - 3;
    const int mx = map_axis(gx, a.nx, a.bc[0], a.bc[1], &sx), my = map_axis(gy, a.ny, a.bc[2], a.bc[3], &sy);
    double v = __ldg(a.in + q * a.vstride + (long)my * a.nx + mx);
    if (q == VX) v = v * sx;
    if (q == VY) v = v * sy;
    return (R)v;
}
// hybrid order's undivided velocity divergence (hy_getRiemannState.F90:341-360)
template <class R> __device__ __forceinline__ R divu2d(const Args2D &a, const Smem2D<R> &s, int wx, int wy)
{
    R dv = vel2d(a, s, VX, wx + 1, wy) - vel2d(a, s, VX, wx - 1, wy);
    dv = dv + vel2d(a, s, VY, wx, wy + 1) - vel2d(a, s, VY, wx, wy - 1);
    return R(0.5) * dv;
}

// face states of one cell along dir, with the transverse correction of the
// other direction (hy_dataReconstOneStep.F90:931-936) and the negativity
// fallback (:1131-1165); stores global-order Wp/Wm into s.W[.][t].
template <class R, int EXT>
__device__ __forceinline__ void states_stage(const Args2D &a, Smem2D<R> &s, int dir, int t, int wx, int wy,
                                             int dbi, int dbstep, R dtn, R hdtn, R hdtt, R hdt)
{
    const int ox = dir == 0, oy = dir == 1;
    R g[6], Vm[6], Vc[6], Vp[6], vecL[6], vecR[6], Wm[6], Wp[6];
    win6(s, wx, wy, g); rot(dir, g, Vc);
    // the cell's eigensystem along dir (FP32: from the base the slope stage kept)
    Eig<R> e;
    if (KeepOwn<R>::value) {
        EigBase<R> eb;
        eb.cf = s.EB[0][dbi]; eb.ahinv = s.EB[1][dbi]; eb.lp = s.EB[2][dbi]; eb.a2inv = s.EB[3][dbi];
        eb.rho = Vc[0];
        eb.rp = eb.rho * (eb.cf * eb.cf);
        eigen_dir(eb, Vc[1], e);
    } else {
        EigBase<R> eb;
        if (!eigen_base(Vc[0], Vc[4], s.V[GC][wy][wx + XO], eb)) set_err(a.err, ERR_SOUND);
        eigen_dir(eb, Vc[1], e);
        if (!KeepSig<R>::value) {
            // sigma of the other direction at this cell, times dt/2 dx_t, parked
            // in this thread's face-state slots until the transverse correction
            R sgo[6];
            sigma_other(a, s, dir, wx, wy, g, eb, sgo);
#pragma unroll
            for (int k = 0; k < 6; k++) s.W[k][t] = hdtt * sgo[k];
        }
    }
    if (EXT && a.prm.order == 2) {
        // MUSCL-Hancock: the cell's own slope, flattening and tracing in one step
        win6(s, wx - ox, wy - oy, g); rot(dir, g, Vm);
        win6(s, wx + ox, wy + oy, g); rot(dir, g, Vp);
        R F = R(0.);
        if (a.prm.flattening) {
            const long gx = (long)blockIdx.x * T2 + wx - 3, gy = (long)blockIdx.y * T2 + wy - 3;
            const long np = (long)(a.nx + 2) * (a.ny + 2);
            F = ((const R *)a.flat)[dir * np + (gy + 1) * (a.nx + 2) + gx + 1];
        }
        R wm[6], wp[6];
        mh_trace(a.prm, e, dtn, hdtn, Vm, Vc, Vp, F, wm, wp);
        unrot(dir, wm, Wm); unrot(dir, wp, Wp);
    } else {
    if (a.prm.order == 5) {
        R S[5][6];
#pragma unroll
        for (int o = -2; o <= 2; o++) { win6(s, wx + o * ox, wy + o * oy, g); rot(dir, g, S[o + 2]); }
        weno_interfaces(a.prm, e, S, vecL, vecR);
#pragma unroll
        for (int k = 0; k < 6; k++) { Vm[k] = S[1][k]; Vp[k] = S[3][k]; }
    } else {
        win6(s, wx - ox, wy - oy, g); rot(dir, g, Vm);
        win6(s, wx + ox, wy + oy, g); rot(dir, g, Vp);
        R dbN[6], db0[6], dbP[6];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            dbN[k] = s.DBF[k * NDB + dbi - dbstep];
            db0[k] = s.DBF[k * NDB + dbi];
            dbP[k] = s.DBF[k * NDB + dbi + dbstep];
        }
        ppm_interfaces(Vm, Vc, Vp, dbN, db0, dbP, vecL, vecR);
        if (EXT && a.prm.steepening)
            steepen(R(a.prm.tiny), R(dir == 0 ? a.dx : a.dy), s.V[D][wy - 2 * oy][wx - 2 * ox + XO], Vm, Vc, Vp,
                    s.V[D][wy + 2 * oy][wx + 2 * ox + XO], s.V[GE][wy][wx + XO], dbN[0], dbP[0], vecL, vecR);
    }
    if (a.prm.flattening) {
        // the window origin is the tile origin minus three cells
        const long gx = (long)blockIdx.x * T2 + wx - 3, gy = (long)blockIdx.y * T2 + wy - 3;
        const long np = (long)(a.nx + 2) * (a.ny + 2);
        flatten(((const R *)a.flat)[dir * np + (gy + 1) * (a.nx + 2) + gx + 1], Vc, vecL, vecR);
    }
    R wm[6], wp[6];
    ppm_trace(e, dtn, hdtn, Vc, vecL, vecR, wm, wp);
    unrot(dir, wm, Wm); unrot(dir, wp, Wp);
    }
    if (EXT && a.prm.use_hybrid) {
        const int k4 = a.prm.order - 1 > 2 ? 2 : a.prm.order - 1;
        const R eps = hybrid_eps(a.prm, s.V[D][wy][wx + XO], s.V[P][wy][wx + XO], s.V[GC][wy][wx + XO]);
        R mn = divu2d(a, s, wx - k4, wy - k4);
        for (int jj = -k4; jj <= k4; jj++)
            for (int ii = -k4; ii <= k4; ii++) mn = fmin(mn, divu2d(a, s, wx + ii, wy + jj));
        if (mn < eps) {
            win6(s, wx, wy, g);
            hybrid_rh(2, g, g, s.V[GC][wy][wx + XO], Wm, Wp);
        }
    }
    // transverse flux of the other direction at this cell (from the analysis stage)
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const R corr = KeepSig<R>::value ? hdtt * s.SG[k][dbi] : s.W[k][t];
        Wm[k] = Wm[k] - corr;
        Wp[k] = Wp[k] - corr;
    }
    if (Wm[0] < R(0) || Wp[0] < R(0) || Wm[4] < R(0) || Wp[4] < R(0)) {
        win6(s, wx, wy, g);
#pragma unroll
        for (int k = 0; k < 6; k++) { Wm[k] = g[k]; Wp[k] = g[k]; }
    }
    if (EXT && a.prm.use_gravity) {   // hy_getRiemannState.F90:843-885, global axes after unrot
        R gl, gr;
        gravity_face_values(a.prm, dir, gl, gr);
#pragma unroll
        for (int q = 0; q < 3; q++) {
            R gp = q == dir ? gr : R(a.prm.grav[q]);
            R gn = q == dir ? gl : R(a.prm.grav[q]);
            Wp[1 + q] = Wp[1 + q] + hdt * gp;
            Wm[1 + q] = Wm[1 + q] + hdt * gn;
        }
    }
#pragma unroll
    for (int k = 0; k < 6; k++) { s.W[k][t] = Wp[k]; s.W[6 + k][t] = Wm[k]; }
}

// total energy of a window cell, read from the state (the window holds D..EI)
template <class R> __device__ __forceinline__ R ener2d(const Args2D &a, int wx, int wy)
{
    double s_ = 1.0;
    const int gx = (int)(blockIdx.x * T2) + wx - 3, gy = (int)(blockIdx.y * T2) + wy - 3;
    const int mx = map_axis(gx, a.nx, a.bc[0], a.bc[1], &s_), my = map_axis(gy, a.ny, a.bc[2], a.bc[3], &s_);
    return (R)__ldg(a.in + DV_ENER * a.vstride + (long)my * a.nx + mx);
}

template <class R, int EXT>
__device__ __forceinline__ void faces_stage(const Args2D &a, Smem2D<R> &s, int dir, int t, int wl, int wr,
                                            int wxl, int wyl, int wxr, int wyr)
{
    R VL[6], VR[6], F[8];
#pragma unroll
    for (int k = 0; k < 6; k++) { VL[k] = s.W[k][wl]; VR[k] = s.W[6 + k][wr]; }
    bool shock = false;
    if (EXT && a.shok) {       // window column/row w is grid cell tile origin + w - 3
        const int x0 = blockIdx.x * T2 - 3, y0 = blockIdx.y * T2 - 3;
        shock = shock_flag(a.shok, x0 + wxl, y0 + wyl, 0, a.nx, a.ny, 1, a.bc) +
                shock_flag(a.shok, x0 + wxr, y0 + wyr, 0, a.nx, a.ny, 1, a.bc) > 0;
    }
    int e = riemann<R, EXT>(a.prm, dir, VL, s.V[GC][wyl][wxl + XO], s.V[GE][wyl][wxl + XO],
                    VR, s.V[GC][wyr][wxr + XO], s.V[GE][wyr][wxr + XO], F, shock);
    if (e) set_err(a.err, e);
    if (EXT && a.prm.use_avisc) {
        const int td = 1 - dir, tx = td == 0, ty = td == 1, vt = td == 0 ? VX : VY, vn = dir == 0 ? VX : VY;
        const R del[2] = {R(a.dx), R(a.dy)};
        R tr[3] = {R(0.), R(0.), R(0.)};
        tr[td] = R(0.25) * (s.V[vt][wyr + ty][wxr + tx + XO] - s.V[vt][wyr - ty][wxr - tx + XO] + s.V[vt][wyl + ty][wxl + tx + XO] -
                            s.V[vt][wyl - ty][wxl - tx + XO]) * del[dir] / del[td];
        const R Ul[5] = {s.V[D][wyl][wxl + XO], s.V[VX][wyl][wxl + XO], s.V[VY][wyl][wxl + XO], s.V[VZ][wyl][wxl + XO], ener2d<R>(a, wxl, wyl)};
        const R Ur[5] = {s.V[D][wyr][wxr + XO], s.V[VX][wyr][wxr + XO], s.V[VY][wyr][wxr + XO], s.V[VZ][wyr][wxr + XO], ener2d<R>(a, wxr, wyr)};
        avisc_flux(R(a.prm.cvisc), dir, 2, s.V[vn][wyl][wxl + XO], s.V[vn][wyr][wxr + XO], tr, Ul, Ur, F);
        eint_fluxes(a.prm, VL, VR, F);
    }
#pragma unroll
    for (int k = 0; k < NF; k++) s.DBF[k * NFC + t] = F[k];
}

// dynamic shared memory of one CTA: the stages' arrays plus 128 bytes to
// align them for TMA
template <class R> constexpr int smem2d_bytes() { return (int)sizeof(Smem2D<R>) + 128; }
// bytes of one TMA window box: 8 variables x 22 rows x 24 columns of FP64
constexpr unsigned kWinBoxBytes = 8u * WIN * WP * 8u;
// the FP32 kernel stages the FP64 box in the region of its slopes, sigmas,
// face states and eigensystem bases (unused during stage A), which follows
// the window at a 128-byte aligned offset
static_assert(sizeof(float) * 8 * WIN * WP % 128 == 0, "FP32 window size keeps the staging area aligned");
static_assert(sizeof(float) * (NF * NFC + 6 * NDB + 12 * NW + 4 * NDB) >= kWinBoxBytes,
              "FP32 staging area holds the FP64 window box");

template <class R, int EXT>
__global__ void __launch_bounds__(Threads2D<R>::value) __maxnreg__(Regs2D<R>::value)
hydro2d_kernel(const __grid_constant__ Args2D a)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // 128-byte aligned base (the TMA destination); the launch adds 128 bytes
    unsigned char *base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    Smem2D<R> &s = *reinterpret_cast<Smem2D<R> *>(base);
    __shared__ __align__(8) uint64_t wbar;
    constexpr int NT2 = Threads2D<R>::value;
    const int tid = threadIdx.x;
    const int tx0 = blockIdx.x * T2, ty0 = blockIdx.y * T2;
    const double dt = a.dtv ? a.dtv[0] : a.dt_arg;

    // ---- A: window load.  Interior windows: one TMA box (columns tx0-4 ..
    // tx0+19, rows ty0-3 .. ty0+18, the 8 variables) issued by thread 0 while
    // the owner threads fetch their FP64 update inputs.  Edge windows: every
    // cell through map_axis, all of a thread's loads in flight together.
    const bool owner = tid < NOWN;
    const int oi = tid % T2, oj = tid / T2;
    const long gidx = (long)(ty0 + oj) * a.nx + (tx0 + oi);
    const bool tma = a.use_tma && tx0 >= 4 && tx0 + T2 + 4 <= a.nx && ty0 >= 3 && ty0 + T2 + 3 <= a.ny;
    bool ok = true;
    if (tma) {
        double *stage = sizeof(R) == 8 ? reinterpret_cast<double *>(&s.V[0][0][0])
                                       : reinterpret_cast<double *>(&s.DBF[0]);
        if (tid == 0) mbar_init(&wbar, 1);
        __syncthreads();
        if (tid == 0) {
            mbar_arrive_expect_tx(&wbar, kWinBoxBytes + a.tma_extra_tx);
            tma_load_3d(stage, &a.tmap, tx0 - 4, ty0 - 3, 0, &wbar);
        }
        double own0 = 0.;
        if (owner) own0 = __ldg(a.in + DV_ENER * a.vstride + gidx);
        ok = mbar_wait_bounded(&wbar, 0, a.wait_budget, a.err);
        if (owner) s.OWN[0][tid] = own0;
        if constexpr (sizeof(R) == 4) {
            // the FP64 update inputs of the owner cells come from the box exactly
            if (owner) {
                const int c = ((oj + 3) * WP) + oi + 3 + XO;
                s.OWN[KeepOwn<R>::value ? 1 : 0][tid] = stage[D * WIN * WP + c];
                s.OWN[KeepOwn<R>::value ? 2 : 0][tid] = stage[VX * WIN * WP + c];
                s.OWN[KeepOwn<R>::value ? 3 : 0][tid] = stage[VY * WIN * WP + c];
                s.OWN[KeepOwn<R>::value ? 4 : 0][tid] = stage[VZ * WIN * WP + c];
                s.OWN[KeepOwn<R>::value ? 5 : 0][tid] = stage[EI * WIN * WP + c];
            }
            // whole stored rows (the box's 24 columns, pads included) two
            // values at a time: 16-byte shared loads, 8-byte stores
            constexpr int NPR = WP / 2, NPAIR = 8 * WIN * NPR;
            static_assert(WP % 2 == 0, "stored rows hold whole pairs");
            float *vw = reinterpret_cast<float *>(&s.V[0][0][0]);
            for (int e = tid; e < NPAIR; e += NT2) {
                const int row = e / NPR, q = e - row * NPR;
                const double2 d2 = reinterpret_cast<const double2 *>(stage + row * WP)[q];
                reinterpret_cast<float2 *>(vw + row * WP)[q] = make_float2((float)d2.x, (float)d2.y);
            }
        }
    } else {
        constexpr int NEL = 8 * WIN * WIN, NLD = (NEL + NT2 - 1) / NT2;
        double buf[NLD];
#pragma unroll
        for (int q = 0; q < NLD; q++) {
            const int e = tid + q * NT2;
            buf[q] = 0.;
            if (e < NEL) {
                int v = e / (WIN * WIN), r = e - v * (WIN * WIN);
                int wy = r / WIN, wx = r - wy * WIN;
                double sx = 1.0, sy = 1.0;
                int gx = map_axis(tx0 + wx - 3, a.nx, a.bc[0], a.bc[1], &sx);
                int gy = map_axis(ty0 + wy - 3, a.ny, a.bc[2], a.bc[3], &sy);
                double val = __ldg(a.in + v * a.vstride + (long)gy * a.nx + gx);
                buf[q] = v == VX ? val * sx : (v == VY ? val * sy : val);
            }
        }
        double own[KeepOwn<R>::value ? 6 : 1];
        if (owner) {
            own[0] = __ldg(a.in + DV_ENER * a.vstride + gidx);
            if (KeepOwn<R>::value) {
                own[KeepOwn<R>::value ? 1 : 0] = __ldg(a.in + D * a.vstride + gidx);
                own[KeepOwn<R>::value ? 2 : 0] = __ldg(a.in + VX * a.vstride + gidx);
                own[KeepOwn<R>::value ? 3 : 0] = __ldg(a.in + VY * a.vstride + gidx);
                own[KeepOwn<R>::value ? 4 : 0] = __ldg(a.in + VZ * a.vstride + gidx);
                own[KeepOwn<R>::value ? 5 : 0] = __ldg(a.in + EI * a.vstride + gidx);
            }
        }
#pragma unroll
        for (int q = 0; q < NLD; q++) {
            const int e = tid + q * NT2;
            if (e < NEL) {
                int v = e / (WIN * WIN), r = e - v * (WIN * WIN);
                int wy = r / WIN, wx = r - wy * WIN;
                s.V[v][wy][wx + XO] = (R)buf[q];
            }
        }
        if (owner) {
#pragma unroll
            for (int q = 0; q < (KeepOwn<R>::value ? 6 : 1); q++) s.OWN[q][tid] = own[q];
        }
    }
    // the step's quotients of dt and the cell sizes, one FP64 division per
    // thread of the first six instead of all six in every thread
    __shared__ double uq[6];
    if (tid < 6) {
        const double num = tid < 2 ? dt : (tid < 4 ? 0.5 * dt : 1.0);
        uq[tid] = num / ((tid & 1) ? a.dy : a.dx);
    }
    // a window that did not arrive in time ends the tile (ERR_TIMEOUT is set)
    if (__syncthreads_or(!ok)) return;

    const double dt_dx = uq[0], dt_dy = uq[1];
    const R dtnx = R(dt_dx), hdtnx = R(0.5 * dt_dx);
    const R dtny = R(dt_dy), hdtny = R(0.5 * dt_dy);
    const R hdtx = R(uq[2]), hdty = R(uq[3]);
    const bool ppm = a.prm.order == 3;     // PPM reads the slopes of its neighbours

    // ---- B: x slopes and sigma_y
    for (int t = tid; t < NDB; t += NT2) {
        int ii = t % (T2 + 4) - 2, jj = t / (T2 + 4);
        analysis_stage(a, s, 0, t, ii + 3, jj + 3, ppm);
    }
    __syncthreads();
    // ---- C: x face states
    for (int t = tid; t < NW; t += NT2) {
        int ii = t % (T2 + 2) - 1, jj = t / (T2 + 2);
        states_stage<R, EXT>(a, s, 0, t, ii + 3, jj + 3, jj * (T2 + 4) + ii + 2, 1, dtnx, hdtnx, hdty, R(0.5 * dt));
    }
    __syncthreads();
    // ---- D: x faces
    for (int t = tid; t < NFC; t += NT2) {
        int fi = t % (T2 + 1), jj = t / (T2 + 1);
        faces_stage<R, EXT>(a, s, 0, t, jj * (T2 + 2) + fi, jj * (T2 + 2) + fi + 1, fi + 2, jj + 3, fi + 3, jj + 3);
        if (EXT && a.fd[0] && (fi < T2 || tx0 + T2 == a.nx))   // the species' mass fluxes
            ((R *)a.fd[0])[(long)(ty0 + jj) * (a.nx + 1) + tx0 + fi] = s.DBF[FD * NFC + t];
    }
    __syncthreads();

    // ---- E: owner threads, x part of the update
    double U0[5], dens0 = 0., Ax = 0., Bx = 0., pav = 0., SphX = 0., eint0 = 0.;
    const double dtdx = dt_dx, dtdy = dt_dy;
    if (owner) {
        double vx, vy, vz, en = s.OWN[0][tid];
        if (KeepOwn<R>::value) {
            dens0 = s.OWN[KeepOwn<R>::value ? 1 : 0][tid]; vx = s.OWN[KeepOwn<R>::value ? 2 : 0][tid];
            vy = s.OWN[KeepOwn<R>::value ? 3 : 0][tid]; vz = s.OWN[KeepOwn<R>::value ? 4 : 0][tid];
            eint0 = s.OWN[KeepOwn<R>::value ? 5 : 0][tid];
        } else {   // the FP64 window holds these values exactly
            dens0 = (double)s.V[D][oj + 3][oi + 3 + XO]; vx = (double)s.V[VX][oj + 3][oi + 3 + XO];
            vy = (double)s.V[VY][oj + 3][oi + 3 + XO]; vz = (double)s.V[VZ][oj + 3][oi + 3 + XO];
            eint0 = (double)s.V[EI][oj + 3][oi + 3 + XO];
        }
        U0[0] = dens0; U0[1] = vx * dens0; U0[2] = vy * dens0; U0[3] = vz * dens0; U0[4] = dens0 * en;
        int fl = oj * (T2 + 1) + oi, fr = fl + 1;
#pragma unroll
        for (int v = 0; v < 5; v++)
            U0[v] = U0[v] - dtdx * ((double)s.DBF[v * NFC + fr] - (double)s.DBF[v * NFC + fl]);
        Ax = (double)s.DBF[FEI * NFC + fl] - (double)s.DBF[FEI * NFC + fr];
        Bx = (double)s.DBF[FVOL * NFC + fl] - (double)s.DBF[FVOL * NFC + fr];
        SphX = ((double)s.DBF[FP * NFC + fl] - (double)s.DBF[FP * NFC + fr]) * (1.0 - a.prm.fpres) / a.dx;
        int w = oj * (T2 + 2) + oi + 1;
        pav = 0.5 * ((double)s.W[6 + P][w] + (double)s.W[P][w]);
    }
    __syncthreads();

    // ---- F: y slopes and sigma_x
    for (int t = tid; t < NDB; t += NT2) {
        int ii = t % T2, jj = t / T2 - 2;
        analysis_stage(a, s, 1, t, ii + 3, jj + 3, ppm);
    }
    __syncthreads();
    // ---- G: y face states
    for (int t = tid; t < NW; t += NT2) {
        int ii = t % T2, jj = t / T2 - 1;
        states_stage<R, EXT>(a, s, 1, t, ii + 3, jj + 3, (jj + 2) * T2 + ii, T2, dtny, hdtny, hdtx, R(0.5 * dt));
    }
    __syncthreads();
    // ---- H: y faces
    for (int t = tid; t < NFC; t += NT2) {
        int ii = t % T2, fj = t / T2;
        faces_stage<R, EXT>(a, s, 1, t, fj * T2 + ii, (fj + 1) * T2 + ii, ii + 3, fj + 2, ii + 3, fj + 3);
        if (EXT && a.fd[1] && (fj < T2 || ty0 + T2 == a.ny))
            ((R *)a.fd[1])[(long)(ty0 + fj) * a.nx + tx0 + ii] = s.DBF[FD * NFC + t];
    }
    __syncthreads();

    // ---- I: finish the update, energyFix, Eos, store, CFL rate
    double rate = 0.;
    if (owner) {
        const DevParams &prm = a.prm;
        int fl = oj * T2 + oi, fr = fl + T2;
#pragma unroll
        for (int v = 0; v < 5; v++)
            U0[v] = U0[v] - dtdy * ((double)s.DBF[v * NFC + fr] - (double)s.DBF[v * NFC + fl]);
        double Ay = (double)s.DBF[FEI * NFC + fl] - (double)s.DBF[FEI * NFC + fr];
        double By = (double)s.DBF[FVOL * NFC + fl] - (double)s.DBF[FVOL * NFC + fr];
        double SphY = ((double)s.DBF[FP * NFC + fl] - (double)s.DBF[FP * NFC + fr]) * (1.0 - prm.fpres) / a.dy;
        int w = (oj + 1) * T2 + oi;
        pav = pav * 0.5 + ((double)s.W[6 + P][w] + (double)s.W[P][w]) * 0.25;
        double inten = 0.;
        if (prm.use_aux_eint) {
            inten = dens0 * eint0;
            inten = inten + dtdx * (Ax + pav * Bx);
            inten = inten + dtdy * (Ay + pav * By);
            inten = inten + dt * 0.0;
        }
        const double Sph[5] = {0., SphX, SphY, 0., 0.};
#pragma unroll
        for (int v = 0; v < 5; v++) U0[v] = U0[v] + dt * (0. + Sph[v]);
        if (EXT && prm.use_gravity) {   // hy_unsplitUpdate.F90:1234-1245, from the step's old momentum
            double vold[3];
#pragma unroll
            for (int q = 0; q < 3; q++)
                vold[q] = KeepOwn<R>::value ? s.OWN[KeepOwn<R>::value ? 2 + q : 0][tid]
                                            : (double)s.V[VX + q][oj + 3][oi + 3 + XO];
            const double momOld[3] = {vold[0] * dens0, vold[1] * dens0, vold[2] * dens0};
            for (int q = 0; q < 3; q++) U0[1 + q] = U0[1 + q] + 0.5 * dt * dens0 * prm.grav[q];
            double dp = 0.;
            for (int q = 0; q < 3; q++) dp = dp + momOld[q] * prm.grav[q];
            U0[4] = U0[4] + 0.5 * dt * dp;
        }
        double dens = fmax2(U0[0], prm.small_dens);
        const double rdens = 1.0 / dens;   // one division for the five quotients by dens
        double vx = rdiv_y(U0[1], dens, rdens), vy = rdiv_y(U0[2], dens, rdens), vz = rdiv_y(U0[3], dens, rdens);
        double ener = rdiv_y(U0[4], dens, rdens);
        double eint = prm.use_aux_eint ? rdiv_y(inten, dens, rdens) : eint0;
        if (EXT && prm.use_gravity) {   // hy_gravityStepBlk -> hy_addGravity: the n+1 half step
            const double hdt = 0.5 * dt;
            double vn[3] = {vx + hdt * prm.grav[0], vy + hdt * prm.grav[1], vz + hdt * prm.grav[2]};
            double dp = 0.;
            for (int q = 0; q < 3; q++) dp = dp + vn[q] * prm.grav[q];
            ener = ener + hdt * dp;
            vx = vn[0]; vy = vn[1]; vz = vn[2];
        }
        // hy_energyFix.F90:240-260
        double ekin = vx * vx; ekin = ekin + vy * vy; ekin = ekin + vz * vz; ekin = 0.5 * ekin;
        double ee = ener - ekin - 0.0;
        double newE = (!prm.use_aux_eint || ee > prm.eint_switch * (ekin + 0.0)) ? fmax2(prm.small_e, ee)
                                                                                : fmax2(prm.small_e, eint);
        ener = newE + ekin;
        eint = newE;
        // Eos_wrapped(MODE_DENS_EI)
        double ek2 = 0.5 * (vx * vx + vy * vy + vz * vz);
        double eg = eint;
        if (ener - ek2 > fmax2(prm.small_e, prm.eint_switch * ek2)) eg = ener - ek2;
        double pres = dens * eg * a.gam1inv;
        double temp = eg * a.ggprodinv * prm.abar;
        double game = pres / (eg * dens) + 1;
        double* o = a.out;
        const long vs = a.vstride;
        o[D * vs + gidx] = dens; o[VX * vs + gidx] = vx; o[VY * vs + gidx] = vy; o[VZ * vs + gidx] = vz;
        o[P * vs + gidx] = pres; o[GC * vs + gidx] = prm.gamma; o[GE * vs + gidx] = game;
        o[EI * vs + gidx] = eg; o[DV_ENER * vs + gidx] = eg + ek2; o[DV_TEMP * vs + gidx] = temp;
        // Hydro_computeDt.F90:215-222 rate, in FP64
        double cs = sqrt(rdiv_y(prm.gamma * pres, dens, rdens));
        rate = (fabs(vx - 0.) + cs) * uq[4];
        rate = fmax2(rate, (fabs(vy - 0.) + cs) * uq[5]);
        if (gidx < a.rate_c0 || gidx >= a.rate_c1) rate = 0.;
    }
    // CTA max, then one atomic per CTA (positive doubles order like their bits)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, off));
    __shared__ double red[NT2 / 32];
    if ((tid & 31) == 0) red[tid >> 5] = rate;
    __syncthreads();
    if (tid == 0) {
        double m = red[0];
        for (int w = 1; w < NT2 / 32; w++) m = fmax(m, red[w]);
        atomicMax(a.rate_max, (unsigned long long)__double_as_longlong(m));
    }
}

// flattening coefficients of every cell of the grid padded by one layer, both
// directions (hy_getRiemannState.F90:367-465); neighbours through map_axis
template <class R>
__global__ void __launch_bounds__(256) flat2d_kernel(const Args2D a, R *flat)
{
    const long np = (long)(a.nx + 2) * (a.ny + 2);
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < np; idx += (long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % (a.nx + 2)) - 1, j = (int)(idx / (a.nx + 2)) - 1;
        for (int d = 0; d < 2; d++) {
            R p[7], v[5];
#pragma unroll
            for (int o = -3; o <= 3; o++) {
                double sx = 1.0, sy = 1.0;
                int gx = map_axis(i + (d == 0 ? o : 0), a.nx, a.bc[0], a.bc[1], &sx);
                int gy = map_axis(j + (d == 1 ? o : 0), a.ny, a.bc[2], a.bc[3], &sy);
                long c = (long)gy * a.nx + gx;
                p[o + 3] = (R)__ldg(a.in + P * a.vstride + c);
                if (o >= -2 && o <= 2)
                    v[o + 2] = (R)(d == 0 ? __ldg(a.in + VX * a.vstride + c) * sx : __ldg(a.in + VY * a.vstride + c) * sy);
            }
            R ftm = flat_tilde(p[0], p[1], p[3], p[4], v[0], v[2]);
            R ft0 = flat_tilde(p[1], p[2], p[4], p[5], v[1], v[3]);
            R ftp = flat_tilde(p[2], p[3], p[5], p[6], v[2], v[4]);
            flat[d * np + idx] = flat_coeff(p[4] - p[2], ftm, ft0, ftp);
        }
    }
}

} // namespace fxb
