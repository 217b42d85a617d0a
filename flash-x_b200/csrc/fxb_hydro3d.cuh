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
//
// The same kernels run in AMR batch mode (template flag AMR): blockIdx.y
// selects one leaf block of a batch whose guard cells were filled by the
// AMR guard-cell kernels; every block is then a small grid of nx*ny*nz
// cells with its own cell size (its refinement level) and its own slice of
// the intermediates, and the update writes the leaf's interior store.
#pragma once
#include "fxb_device.cuh"

namespace fxb {

// one entry of an AMR batch
struct AmrEntry3 {
    int out_blk;    // block index of the leaf in the interior store
    int level;      // refinement level, 1-based
    int leaf;       // leaf slot (UNK block index)
    int flags;      // AMR_SKIP_UPDATE: the update waits for corrected fluxes
};
enum { AMR_SKIP_UPDATE = 1 };

// Division by a launch-invariant divisor d as a multiply-high, an add and a
// shift (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): with 2^s >= d and m = floor(2^32 (2^s - d) / d) + 1,
// x / d = (umulhi(x, m) + x) >> s for every x below 2^31.
struct FastDiv {
    unsigned d, m, s;
};
inline FastDiv make_fastdiv(unsigned d)
{
    unsigned s = 0;
    while ((1ull << s) < d) s++;
    return FastDiv{d, (unsigned)((((1ull << 32) * ((1ull << s) - d)) / d) + 1), s};
}

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
    void *wst[3];   // per direction [2][cells with that coordinate in [-1, n]]: Wp, Wm pressures
    void *flx[3];   // per direction [8][faces]
    void *slp;      // PPM: characteristic-limited slopes of the current direction [6][Grid3::ns(d)]
    long slp_bstride;           // AMR: elements of R per batch entry
    void *flat;     // flattening coefficients [3][(nx+2)(ny+2)(nz+2)] of R
    long flat_bstride;          // AMR: elements of R per batch entry
    // AMR batch mode
    const void *gcb;            // guard-filled blocks [entry][var][nz+2g][ny+2g][nx+2g] of R
    long gcb_vstride, gcb_bstride;
    const double *istore;       // interior store holding the step's input state (FP64)
    int ng;
    const AmrEntry3 *batch;
    const double *dxl;          // cell sizes [level-1][3]
    double *odata;              // interior store [block][var][cell]
    long o_vstride, o_bstride;
    long sig_bstride, w_bstride[3], f_bstride[3];   // elements of R per batch entry
    int cta[4];                 // AMR: CTAs per batch entry (sig3d, slope3d, flux3d, update3d); uniform
                                // grid: CTAs of sig3d (+ flattening, hybrid), states3d (+ slopes), flux3d, update3d
    FastDiv fdx[5], fdy[5];     // divisors nx + e and ny + e (e = 0, 1, 2, 4), set by the launchers
    int sf_len[3], sf_lines[3]; // face-state tiles per direction (cells along d, lines), set by the launchers
    int sf_t1[3] = {0, 0, 0};   // lines per face-state tile chosen by the tuner (0: the launchers' choice)
    const unsigned char *hyb;   // hybrid order: 1 where min DivU over the cell's box < eps, padded box (AMR: per entry)
    long hyb_bstride = 0;       // AMR: flags per batch entry
    void *divu = nullptr;       // AMR: DivU scratch per batch entry, box [-3, n+2]^3 of R
    long divu_bstride = 0;
    long rate_c0 = 0, rate_c1 = 0x7fffffffffffffffL;   // cells [c0, c1) enter the CFL rate (a slab's own)
    unsigned char *ctufb[3] = {nullptr, nullptr, nullptr};   // species on: 1 where the CTU fallback fired (Grid3::widx)
    const unsigned char *shok = nullptr;   // shock detector on (uniform grid): the flag of every cell
};
// Face-state tile of direction d (N cells along d, N1 along the t1 axis):
// the fewest warp lanes in total (the N + 1 faces split into segments of
// Ls - 1, each needing Ls cells, on lines grouped T1 at a time, CTAs rounded
// up to whole warps), then the largest CTA; lines along y or z group at least
// 8 x-neighbours (coalescing).
#ifndef FXB_SF_MAXT
#define FXB_SF_MAXT 288
#endif
// force_t1 > 0 takes that line count (when it fits) and only picks Ls.
inline void sflux_tile(int d, int N, int N1, int halo, int &Ls, int &T1, int force_t1 = 0)
{
    long best = -1;
    Ls = 3; T1 = 1;
    const int cand[5] = {16, 8, 4, 2, 1};
    const bool forced = force_t1 > 0 && force_t1 <= N1;
    for (int t1 : cand) {
        if (t1 > N1) continue;
        if (forced ? t1 != force_t1 : (d != 0 && t1 < (N1 < 8 ? N1 : 8))) continue;
        for (int ls = 3; (ls + halo) * t1 <= FXB_SF_MAXT; ls++) {
            const long nseg = (N + ls - 1) / (ls - 1);
            const long work = nseg * (long)((N1 + t1 - 1) / t1) * (((ls + halo) * t1 + 31) / 32 * 32);
            if (best < 0 || work < best || (work == best && (ls + halo) * t1 > (Ls + halo) * T1)) {
                best = work; Ls = ls; T1 = t1;
            }
        }
    }
}

// the launchers' copy of the arguments with the index divisors and the
// face-state tiles filled in (halo: extra slope cells per line segment)
inline Args3D with_divisors(const Args3D &a, int halo = 0)
{
    Args3D b = a;
    for (int e = 0; e <= 4; e++) { b.fdx[e] = make_fastdiv((unsigned)a.nx + e); b.fdy[e] = make_fastdiv((unsigned)a.ny + e); }
    const int n[3] = {a.nx, a.ny, a.nz};
    for (int d = 0; d < 3; d++) sflux_tile(d, n[d], d == 0 ? a.ny : a.nx, halo, b.sf_len[d], b.sf_lines[d], a.sf_t1[d]);
    return b;
}
enum { AMR_SIG = 1, AMR_STATES = 2 };   // sigma (+ flattening); slopes, face states and fluxes

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
    // slope cells of direction d: coordinate d in [-2, n_d + 1], the others interior
    __device__ long ns(int d) const {
        return d == 0 ? (long)(nx + 4) * ny * nz : d == 1 ? (long)nx * (ny + 4) * nz : (long)nx * ny * (nz + 4);
    }
    __device__ long sidx(int d, int i, int j, int k) const {
        if (d == 0) return ((long)k * ny + j) * (nx + 4) + (i + 2);
        if (d == 1) return ((long)k * (ny + 4) + (j + 2)) * nx + i;
        return ((long)(k + 2) * ny + j) * nx + i;
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

// The block coordinates a stage body works with: CTA x of nx CTAs sharing
// one batch entry y.  A kernel launch passes (blockIdx.x, blockIdx.y,
// gridDim.x); the persistent AMR kernel passes (0, its scratch slot, 1), so
// one CTA runs a whole leaf through every stage.
struct VB {
    int x, y, nx;
};
__device__ __forceinline__ VB hw_block() { return VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x}; }

// Geometry, source and intermediates of one kernel invocation: the whole
// uniform grid, or (AMR) the batch entry `by`.
template <class R, bool AMR> struct Ctx3 {
    Grid3 G;
    const double *src;          // uniform grid: the FP64 state
    const R *srcR;              // AMR: the guard-filled block in the reconstruction type
    long svs;
    int sx, sy, so;
    R *sig, *wst[3], *flx[3], *slp, *flat;
    double dx, dy, dz;
    AmrEntry3 m;
    const unsigned char *hyb;   // hybrid-order flags of the padded box
    __device__ Ctx3(const Args3D &a, int by)
    {
        G = Grid3{a.nx, a.ny, a.nz};
        if constexpr (AMR) {
            const int bb = by;
            m = a.batch[bb];
            hyb = a.hyb ? a.hyb + (long)bb * a.hyb_bstride : nullptr;
            src = nullptr;
            srcR = (const R *)a.gcb + (long)bb * a.gcb_bstride;
            svs = a.gcb_vstride;
            so = a.ng; sx = a.nx + 2 * a.ng; sy = a.ny + 2 * a.ng;
            sig = (R *)a.sig + (long)bb * a.sig_bstride;
            slp = (R *)a.slp + (long)bb * a.slp_bstride;
            flat = (R *)a.flat + (long)bb * a.flat_bstride;
            for (int d = 0; d < 3; d++) {
                wst[d] = (R *)a.wst[d] + (long)bb * a.w_bstride[d];
                flx[d] = (R *)a.flx[d] + (long)bb * a.f_bstride[d];
            }
            dx = a.dxl[3 * (m.level - 1)]; dy = a.dxl[3 * (m.level - 1) + 1]; dz = a.dxl[3 * (m.level - 1) + 2];
        } else {
            m = AmrEntry3{0, 1, 0, 0};
            hyb = a.hyb;
            src = a.in; srcR = nullptr; svs = a.vstride; so = 0; sx = a.nx; sy = a.ny;
            sig = (R *)a.sig;
            slp = (R *)a.slp;
            flat = (R *)a.flat;
            for (int d = 0; d < 3; d++) { wst[d] = (R *)a.wst[d]; flx[d] = (R *)a.flx[d]; }
            dx = a.dx; dy = a.dy; dz = a.dz;
        }
    }
    // primitive 8-vector of cell (i,j,k); AMR blocks hold their guard cells
    __device__ __forceinline__ void load(const Args3D &a, int i, int j, int k, R v[8]) const
    {
        if constexpr (AMR) {
            long c = ((long)(k + so) * sy + (j + so)) * sx + (i + so);
#pragma unroll
            for (int q = 0; q < 8; q++) v[q] = __ldg(srcR + q * svs + c);
        } else {
            load_cell(a, i, j, k, v);
        }
    }
    // the two Eos gammas of cell (i,j,k), all the Riemann solver needs of it
    __device__ __forceinline__ void load_gammas(const Args3D &a, int i, int j, int k, R &gc, R &ge) const
    {
        long c;
        if constexpr (AMR) {
            c = ((long)(k + so) * sy + (j + so)) * sx + (i + so);
        } else {
            double s_ = 1.0;
            int mi = map_axis(i, a.nx, a.bc[0], a.bc[1], &s_);
            int mj = map_axis(j, a.ny, a.bc[2], a.bc[3], &s_);
            int mk = map_axis(k, a.nz, a.bc[4], a.bc[5], &s_);
            c = ((long)mk * a.ny + mj) * a.nx + mi;
        }
        if constexpr (AMR) {
            gc = __ldg(srcR + GC * svs + c);
            ge = __ldg(srcR + GE * svs + c);
        } else {
            gc = (R)__ldg(src + GC * svs + c);
            ge = (R)__ldg(src + GE * svs + c);
        }
    }
    // offset of interior cell (i,j,k) in the source arrays
    __device__ __forceinline__ long cell(int i, int j, int k) const
    { return ((long)(k + so) * sy + (j + so)) * sx + (i + so); }
    // variable q of cell (i,j,k): the uniform grid's state (boundaries
    // mapped, rounded to R), or the AMR leaf's guard-filled block
    __device__ __forceinline__ R var(const Args3D &a, int q, int i, int j, int k) const;
};

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

// one state variable of a possibly virtual cell of the uniform grid
template <class R>
__device__ __forceinline__ R state_var(const Args3D &a, int q, int i, int j, int k)
{
    double sx = 1.0, sy = 1.0, sz = 1.0;
    int mi = map_axis(i, a.nx, a.bc[0], a.bc[1], &sx);
    int mj = map_axis(j, a.ny, a.bc[2], a.bc[3], &sy);
    int mk = map_axis(k, a.nz, a.bc[4], a.bc[5], &sz);
    double x = __ldg(a.in + q * a.vstride + ((long)mk * a.ny + mj) * a.nx + mi);
    if (q == VX) x = x * sx;
    if (q == VY) x = x * sy;
    if (q == VZ) x = x * sz;
    return (R)x;
}

template <class R, bool AMR>
__device__ __forceinline__ R Ctx3<R, AMR>::var(const Args3D &a, int q, int i, int j, int k) const
{
    if constexpr (AMR) return __ldg(srcR + q * svs + cell(i, j, k));
    else return state_var<R>(a, q, i, j, k);
}

// artificial viscosity of the direction-d face between cells (i,j,k) - e_d
// and (i,j,k), on the uniform grid or an AMR leaf (whose guard-filled block
// then carries the total energy)
template <class R, bool AMR>
__device__ __forceinline__ void avisc3d(const Args3D &a, const Ctx3<R, AMR> &X, int d, int i, int j, int k, R F[])
{
    int di, dj, dk;
    offs(d, 1, di, dj, dk);
    const int im = i - di, jm = j - dj, km = k - dk;
    const R del[3] = {R(X.dx), R(X.dy), R(X.dz)};
    R tr[3] = {R(0.), R(0.), R(0.)};
#pragma unroll
    for (int e = 0; e < 3; e++) {
        if (e == d) continue;
        int ie, je, ke;
        offs(e, 1, ie, je, ke);
        const int v = VX + e;
        tr[e] = R(0.25) * (X.var(a, v, i + ie, j + je, k + ke) - X.var(a, v, i - ie, j - je, k - ke) +
                           X.var(a, v, im + ie, jm + je, km + ke) - X.var(a, v, im - ie, jm - je, km - ke)) *
                del[d] / del[e];
    }
    const R Ul[5] = {X.var(a, D, im, jm, km), X.var(a, VX, im, jm, km), X.var(a, VY, im, jm, km),
                     X.var(a, VZ, im, jm, km), X.var(a, DV_ENER, im, jm, km)};
    const R Ur[5] = {X.var(a, D, i, j, k), X.var(a, VX, i, j, k), X.var(a, VY, i, j, k), X.var(a, VZ, i, j, k),
                     X.var(a, DV_ENER, i, j, k)};
    avisc_flux(R(a.prm.cvisc), d, 3, Ul[1 + d], Ur[1 + d], tr, Ul, Ur, F);
}

// (i, j, k) of the linear index of an lx * ly * lz box, in 32-bit arithmetic:
// every box a kernel walks holds fewer than 2^30 cells (checked by fxb_init)
__device__ __forceinline__ void unflatten(unsigned idx, unsigned lx, unsigned ly, int &i, int &j, int &k)
{
    const unsigned q = idx / lx, r = q / ly;
    i = (int)(idx - q * lx); j = (int)(q - r * ly); k = (int)r;
}
__device__ __forceinline__ unsigned fast_div(unsigned x, const FastDiv &f) { return (__umulhi(x, f.m) + x) >> f.s; }
__device__ __forceinline__ void unflatten(unsigned idx, const FastDiv &fx, const FastDiv &fy, int &i, int &j, int &k)
{
    const unsigned q = fast_div(idx, fx), r = fast_div(q, fy);
    i = (int)(idx - q * fx.d); j = (int)(q - r * fy.d); k = (int)r;
}
// grid-stride loop bounds of one launch in 32-bit arithmetic
#define FXB_GRID_LOOP(idx, count) \
    for (int idx = (int)(blockIdx.x * blockDim.x + threadIdx.x); idx < (int)(count); idx += (int)(gridDim.x * blockDim.x))
// the same loop over the CTAs of a virtual block
#define FXB_VB_LOOP(idx, count, vb) \
    for (int idx = (int)((vb).x * blockDim.x + threadIdx.x); idx < (int)(count); idx += (int)((vb).nx * blockDim.x))

// ---- sigma_d of every padded cell --------------------------------------------
template <class R, bool AMR>
__device__ __forceinline__ void sig3d_kernel_body(const Args3D &a, const VB vb)
{
    const Ctx3<R, AMR> X(a, vb.y);
    const Grid3 &G = X.G;
    R *sig = X.sig;
    const long np = G.npad();
    FXB_VB_LOOP(idx, np, vb) {
        int i, j, k;
        unflatten(idx, a.fdx[2], a.fdy[2], i, j, k);
        i -= 1; j -= 1; k -= 1;
        R vc[8];
        X.load(a, i, j, k, vc);
        R gc[6]; six(vc, gc);
        EigBase<R> eb;
        const bool eok = eigen_base(vc[D], vc[P], vc[GC], eb);
        if (!eok) atomicOr(a.err, ERR_SOUND);
        for (int d = 0; d < 3; d++) {
            int di, dj, dk;
            offs(d, 1, di, dj, dk);
            R vm[8], vp[8], g[6], m[6], c[6], p[6], sr[6], sg[6];
            X.load(a, i - di, j - dj, k - dk, vm);
            X.load(a, i + di, j + dj, k + dk, vp);
            six(vm, g); rot3(d, g, m);
            rot3(d, gc, c);
            six(vp, g); rot3(d, g, p);
            Eig<R> e;
            eigen_dir(eb, c[1], e);
            trans_flux(e, m, c, p, a.prm.use_aux_eint != 0, sr);
            unrot3(d, sr, sg);
#pragma unroll
            for (int q = 0; q < 6; q++) sig[((long)d * 6 + q) * np + idx] = sg[q];
        }
    }
}
template <class R, bool AMR>
__global__ void __launch_bounds__(256) sig3d_kernel(const Args3D a)
{
    sig3d_kernel_body<R, AMR>(a, hw_block());
}

// ---- flattening coefficients of every padded cell, three directions ----------
// (hy_getRiemannState.F90:367-465; FlatTilde of the cell and its two
// neighbours along d from pressures three cells either side)
template <class R, bool AMR>
__device__ __forceinline__ void flat3d_kernel_body(const Args3D &a, const VB vb)
{
    const Ctx3<R, AMR> X(a, vb.y);
    const Grid3 &G = X.G;
    const long np = G.npad();
    FXB_VB_LOOP(idx, np, vb) {
        int i, j, k;
        unflatten(idx, a.fdx[2], a.fdy[2], i, j, k);
        i -= 1; j -= 1; k -= 1;
        for (int d = 0; d < 3; d++) {
            int di, dj, dk;
            offs(d, 1, di, dj, dk);
            R p[7], v[5];
#pragma unroll
            for (int o = -3; o <= 3; o++) {
                R c[8];
                X.load(a, i + o * di, j + o * dj, k + o * dk, c);
                p[o + 3] = c[P];
                if (o >= -2 && o <= 2) v[o + 2] = c[VX + d];
            }
            R ftm = flat_tilde(p[0], p[1], p[3], p[4], v[0], v[2]);
            R ft0 = flat_tilde(p[1], p[2], p[4], p[5], v[1], v[3]);
            R ftp = flat_tilde(p[2], p[3], p[5], p[6], v[2], v[4]);
            X.flat[(long)d * np + idx] = flat_coeff(p[4] - p[2], ftm, ft0, ftp);
        }
    }
}
template <class R, bool AMR>
__global__ void __launch_bounds__(256) flat3d_kernel(const Args3D a)
{
    flat3d_kernel_body<R, AMR>(a, hw_block());
}

template <class R>
__device__ __forceinline__ void read_sig(const R *sig, const Grid3 &G, int d, int i, int j, int k, R s[6])
{
    long np = G.npad(), p = G.pidx(i, j, k);
#pragma unroll
    for (int q = 0; q < 6; q++) s[q] = sig[((long)d * 6 + q) * np + p];
}

// CTU cross term of one transverse pair: upwinding along e of sigma_s at the
// cell's e-neighbours, with the e-direction eigensystem of the cell
template <class R>
__device__ __forceinline__ void ctu_term(const Args3D &a, const R *sigp, const Grid3 &G, const R vc[8],
                                        const EigBase<R> &eb, int e, int s, int i, int j, int k, R T[6])
{
    int di, dj, dk;
    offs(e, 1, di, dj, dk);
    R sm[6], sc[6], sp[6], m[6], c[6], p[6], gcell[6], r[6], tr[6];
    read_sig(sigp, G, s, i - di, j - dj, k - dk, sm);
    read_sig(sigp, G, s, i, j, k, sc);
    read_sig(sigp, G, s, i + di, j + dj, k + dk, sp);
    rot3(e, sm, m); rot3(e, sc, c); rot3(e, sp, p);
    six(vc, gcell); rot3(e, gcell, r);
    Eig<R> ev;
    eigen_dir(eb, r[1], ev);
    trans_flux(ev, m, c, p, a.prm.use_aux_eint != 0, tr);
    unrot3(e, tr, T);
}

// ---- PPM slopes of direction d ----------------------------------------------
// hy_TVDslope of every cell once (eigensystem of the cell, characteristic or
// primitive limiting over its two neighbours along d), in the rotated frame
// of direction d; each face-state cell then reads the slopes of itself and of
// its two neighbours instead of recomputing them.
template <class R, bool AMR>
__device__ __forceinline__ void slope3d_kernel_body(const Args3D &a, const VB vb, int d)
{
    const Ctx3<R, AMR> X(a, vb.y);
    const Grid3 &G = X.G;
    const long ns = G.ns(d);
    int di, dj, dk;
    offs(d, 1, di, dj, dk);
    FXB_VB_LOOP(idx, ns, vb) {
        int i, j, k;
        unflatten(idx, a.fdx[d == 0 ? 4 : 0], a.fdy[d == 1 ? 4 : 0], i, j, k);
        if (d == 0) i -= 2; else if (d == 1) j -= 2; else k -= 2;
        R S8[3][8], S[3][6], g[6];
#pragma unroll
        for (int o = -1; o <= 1; o++) {
            X.load(a, i + o * di, j + o * dj, k + o * dk, S8[o + 1]);
            six(S8[o + 1], g); rot3(d, g, S[o + 1]);
        }
        Eig<R> e;
        if (!eigen(S[1][0], S[1][1], S[1][4], S8[1][GC], e)) atomicOr(a.err, ERR_SOUND);
        R db[6];
        tvd_slope(a.prm, e, S[0], S[1], S[2], db);
#pragma unroll
        for (int q = 0; q < 6; q++) X.slp[(long)q * ns + idx] = db[q];
    }
}
template <class R, bool AMR>
__global__ void __launch_bounds__(256) slope3d_kernel(const Args3D a, int d)
{
    slope3d_kernel_body<R, AMR>(a, hw_block(), d);
}

// The face states of one cell from its traced states wm, wp (sweep frame):
// transverse terms, negativity fallback, gravity and the 3-D full-CTU terms.
// vc: the cell's 8-vector.
template <class R, bool AMR, int DIR, int EXT>
__device__ __forceinline__ void face_states_finish(const Args3D &a, const Ctx3<R, AMR> &X, const double dt,
                                                   const R hdtx, const R hdty, const R hdtz, int i, int j, int k,
                                                   const R vc[8], const EigBase<R> &eb, const R wm[6], const R wp[6],
                                                   R Wm_out[6], R Wp_out[6])
{
    constexpr int d = DIR;
    const Grid3 &G = X.G;
    R Wm[6], Wp[6];
    unrot3(d, wm, Wm); unrot3(d, wp, Wp);
    // transverse terms, hy_dataReconstOneStep.F90:931-962
    R s1[6], s2[6];
    if (d == 0) {
        read_sig(X.sig, G, 1, i, j, k, s1); read_sig(X.sig, G, 2, i, j, k, s2);
#pragma unroll
        for (int q = 0; q < 6; q++) {
            Wm[q] = Wm[q] - hdty * s1[q]; Wp[q] = Wp[q] - hdty * s1[q];
            Wm[q] = Wm[q] - hdtz * s2[q]; Wp[q] = Wp[q] - hdtz * s2[q];
        }
    } else if (d == 1) {
        read_sig(X.sig, G, 0, i, j, k, s1); read_sig(X.sig, G, 2, i, j, k, s2);
#pragma unroll
        for (int q = 0; q < 6; q++) {
            Wm[q] = Wm[q] - hdtx * s1[q]; Wp[q] = Wp[q] - hdtx * s1[q];
            Wm[q] = Wm[q] - hdtz * s2[q]; Wp[q] = Wp[q] - hdtz * s2[q];
        }
    } else {
        read_sig(X.sig, G, 0, i, j, k, s1); read_sig(X.sig, G, 1, i, j, k, s2);
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
        gravity_face_values(a.prm, d, gl, gr);
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
        if (d == 0)      { e1 = 1; s1d = 2; e2 = 2; s2d = 1; fac = dt * dt / (6. * X.dy * X.dz); }
        else if (d == 1) { e1 = 2; s1d = 0; e2 = 0; s2d = 2; fac = dt * dt / (6. * X.dz * X.dx); }
        else             { e1 = 0; s1d = 1; e2 = 1; s2d = 0; fac = dt * dt / (6. * X.dx * X.dy); }
        R T1[6], T2[6];
        ctu_term(a, X.sig, G, vc, eb, e1, s1d, i, j, k, T1);
        ctu_term(a, X.sig, G, vc, eb, e2, s2d, i, j, k, T2);
        const R f = R(fac);
#pragma unroll
        for (int q = 0; q < 6; q++) {
            Wp[q] = Wp[q] + (T1[q] + T2[q]) * f;
            Wm[q] = Wm[q] + (T1[q] + T2[q]) * f;
        }
        if (Wp[0] <= R(0) || Wm[0] <= R(0) || Wp[4] <= R(0) || Wm[4] <= R(0)) {
#pragma unroll
            for (int q = 0; q < 6; q++) { Wm[q] = gvc[q]; Wp[q] = gvc[q]; }
            if constexpr (EXT && !AMR) {   // species (extended-option kernels) fall back too
                if (a.ctufb[d]) a.ctufb[d][G.widx(d, i, j, k)] = 1;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) { Wm_out[q] = Wm[q]; Wp_out[q] = Wp[q]; }
}

// hybrid order on the traced states wm, wp (sweep frame) of a uniform-grid
// cell whose flag (hyb3d_kernel) is set
template <class R, bool AMR>
__device__ __forceinline__ void hybrid3d(const Args3D &a, const Ctx3<R, AMR> &X, int i, int j, int k, const R vc[8],
                                         const R Sc[6], R wm[6], R wp[6])
{
    if (a.prm.use_hybrid && X.hyb[X.G.pidx(i, j, k)]) {
        R g[6];
        six(vc, g);
        hybrid_rh(3, g, Sc, vc[GC], wm, wp);
    }
}

// The face states of one cell from its interface values: flattening and
// characteristic tracing (PPM, WENO), then face_states_finish.  Sc: the
// cell's rotated primitives, vc its 8-vector.
template <class R, bool AMR, int DIR, int EXT = 0>
__device__ __forceinline__ void face_states_tail(const Args3D &a, const Ctx3<R, AMR> &X, const double dt, const R dtn,
                                                 const R hdtn, const R hdtx, const R hdty, const R hdtz, int i, int j,
                                                 int k, const R Sc[6], const R vc[8], const EigBase<R> &eb,
                                                 const Eig<R> &e, R vecL[6], R vecR[6], R Wm_out[6], R Wp_out[6])
{
    constexpr int d = DIR;
    const Grid3 &G = X.G;
    if (a.prm.flattening) flatten(X.flat[(long)d * G.npad() + G.pidx(i, j, k)], Sc, vecL, vecR);
    R wm[6], wp[6];
    ppm_trace(e, dtn, hdtn, Sc, vecL, vecR, wm, wp);
    if constexpr (EXT) hybrid3d<R, AMR>(a, X, i, j, k, vc, Sc, wm, wp);
    face_states_finish<R, AMR, DIR, EXT>(a, X, dt, hdtx, hdty, hdtz, i, j, k, vc, eb, wm, wp, Wm_out, Wp_out);
}

// ---- face states of one cell in direction d ------------------------------------
// One instantiation per reconstruction order, so the register allocation of
// the PPM path (three eigensystems and slopes), of the WENO path (one
// eigensystem, five projected cells) and of MUSCL-Hancock (ORDER 2, only in
// the extended-option kernels) do not add up.
template <class R, int ORDER, bool AMR, int DIR, int EXT>
__device__ __forceinline__ void face_states(const Args3D &a, const Ctx3<R, AMR> &X, const double dt, const R dtn,
                                            const R hdtn, const R hdtx, const R hdty, const R hdtz, int i, int j,
                                            int k, R Wm_out[6], R Wp_out[6], R &gc_out, R &ge_out)
{
    constexpr int d = DIR;
    const Grid3 &G = X.G;
    int di, dj, dk;
    offs(d, 1, di, dj, dk);
    R S8[5][8], S[5][6], g[6];
#pragma unroll
    for (int o = -2; o <= 2; o++) {
        if (ORDER != 5 && (o == -2 || o == 2)) continue;   // PPM reads its neighbours' slopes; MH needs none
        X.load(a, i + o * di, j + o * dj, k + o * dk, S8[o + 2]);
        six(S8[o + 2], g); rot3(d, g, S[o + 2]);
    }
    const R *vc = S8[2];
    // the cell's eigensystem along d, and (CTU) along the two other directions
    EigBase<R> eb;
    if (!eigen_base(S[2][0], S[2][4], vc[GC], eb)) atomicOr(a.err, ERR_SOUND);
    Eig<R> e;
    eigen_dir(eb, S[2][1], e);
    if constexpr (ORDER == 2) {
        const R F = a.prm.flattening ? X.flat[(long)d * G.npad() + G.pidx(i, j, k)] : R(0.);
        R wm[6], wp[6];
        mh_trace(a.prm, e, dtn, hdtn, S[1], S[2], S[3], F, wm, wp);
        hybrid3d<R, AMR>(a, X, i, j, k, vc, S[2], wm, wp);
        face_states_finish<R, AMR, DIR, EXT>(a, X, dt, hdtx, hdty, hdtz, i, j, k, vc, eb, wm, wp, Wm_out, Wp_out);
        gc_out = vc[GC]; ge_out = vc[GE];
        return;
    }
    R vecL[6], vecR[6];
    if constexpr (ORDER == 5) {
        weno_interfaces(a.prm, e, S, vecL, vecR);
    } else {
        // slopes of the cell and its two neighbours from slope3d_kernel
        const long ns = G.ns(d);
        const long sN = G.sidx(d, i - di, j - dj, k - dk), s0 = G.sidx(d, i, j, k), sP = G.sidx(d, i + di, j + dj, k + dk);
        R dbN[6], db0[6], dbP[6];
#pragma unroll
        for (int q = 0; q < 6; q++) {
            dbN[q] = X.slp[(long)q * ns + sN];
            db0[q] = X.slp[(long)q * ns + s0];
            dbP[q] = X.slp[(long)q * ns + sP];
        }
        ppm_interfaces(S[1], S[2], S[3], dbN, db0, dbP, vecL, vecR);
        if (EXT && a.prm.steepening) {   // densities two cells out along d
            R Smm[8], Spp[8];
            X.load(a, i - 2 * di, j - 2 * dj, k - 2 * dk, Smm);
            X.load(a, i + 2 * di, j + 2 * dj, k + 2 * dk, Spp);
            steepen(R(a.prm.tiny), R(d == 0 ? X.dx : d == 1 ? X.dy : X.dz), Smm[D], S[1], S[2], S[3], Spp[D], vc[GE],
                    dbN[0], dbP[0], vecL, vecR);
        }
    }
    face_states_tail<R, AMR, DIR, EXT>(a, X, dt, dtn, hdtn, hdtx, hdty, hdtz, i, j, k, S[2], vc, eb, e, vecL, vecR,
                                       Wm_out, Wp_out);
    gc_out = vc[GC]; ge_out = vc[GE];
}


// ---- face states and Riemann fluxes as two kernels (FP64) --------------------------
// In FP64 the fused kernel below measured slower on B200 (its barrier between
// the face states and the fluxes idles two CTAs of long FP64 warps), so the
// FP64 path stores all twelve face-state values and solves the Riemann
// problems in a second kernel.  FP32 fuses them.
#ifndef FXB_FUSE_FP64
#define FXB_FUSE_FP64 0
#endif
template <class R> struct FusedFaces { static constexpr bool value = sizeof(R) == 4 || FXB_FUSE_FP64; };
// slots of the Wp and Wm pressures in the face-state arrays
template <class R> struct PwSlots {
    static constexpr int wp = FusedFaces<R>::value ? 0 : P, wm = FusedFaces<R>::value ? 1 : 6 + P;
};

// The minimum number of resident 256-thread CTAs per SM bounds the registers
// per thread: two CTAs (128 registers, a few hundred bytes of spills)
// measured 18 % faster on B200 than one CTA with 244-255 registers, and three
// CTAs (80 registers) lost again to spill traffic.
#ifndef FXB_S3_MINB_FP64
#define FXB_S3_MINB_FP64 2
#endif
template <class R, int ORDER, bool AMR, int DIR, int EXT>
__device__ __forceinline__ void states3d_kernel_body(const Args3D &a, const VB vb)
{
    constexpr int d = DIR;
    const Ctx3<R, AMR> X(a, vb.y);
    const Grid3 &G = X.G;
    const double dt = a.dtv ? a.dtv[0] : a.dt_arg;
    const double del[3] = {X.dx, X.dy, X.dz};
    const R dtn = R(dt / del[d]), hdtn = R(0.5 * (dt / del[d]));
    const R hdtx = R(0.5 * dt / X.dx), hdty = R(0.5 * dt / X.dy), hdtz = R(0.5 * dt / X.dz);
    R *w = X.wst[d];
    const long nw = G.nw(d);
    FXB_VB_LOOP(idx, nw, vb) {
        int i, j, k;
        unflatten(idx, a.fdx[d == 0 ? 2 : 0], a.fdy[d == 1 ? 2 : 0], i, j, k);
        if (d == 0) i -= 1; else if (d == 1) j -= 1; else k -= 1;
        R Wm[6], Wp[6], gc, ge;
        face_states<R, ORDER, AMR, DIR, EXT>(a, X, dt, dtn, hdtn, hdtx, hdty, hdtz, i, j, k, Wm, Wp, gc, ge);
#pragma unroll
        for (int q = 0; q < 6; q++) { w[(long)q * nw + idx] = Wp[q]; w[(long)(6 + q) * nw + idx] = Wm[q]; }
    }
}
template <class R, int ORDER, bool AMR, int DIR, int EXT>
__global__ void __launch_bounds__(256, FXB_S3_MINB_FP64) states3d_kernel(const Args3D a)
{
    states3d_kernel_body<R, ORDER, AMR, DIR, EXT>(a, hw_block());
}

// ---- Riemann fluxes of direction d ---------------------------------------------
// the direction is a template parameter so that the solver's per-direction
// indexing of the state vectors resolves at compile time (no local memory)
template <class R, bool AMR, int DIR, int EXT>
__device__ __forceinline__ void flux3d_kernel_body(const Args3D &a, const VB vb)
{
    constexpr int d = DIR;
    const Ctx3<R, AMR> X(a, vb.y);
    const Grid3 &G = X.G;
    const R *w = X.wst[d];
    R *f = X.flx[d];
    const long nf = G.nf(d), nw = G.nw(d);
    FXB_VB_LOOP(idx, nf, vb) {
        int i, j, k;
        unflatten(idx, a.fdx[d == 0 ? 1 : 0], a.fdy[d == 1 ? 1 : 0], i, j, k);
        int di, dj, dk;
        offs(d, 1, di, dj, dk);
        long wl = G.widx(d, i - di, j - dj, k - dk), wr = G.widx(d, i, j, k);
        R VL[6], VR[6], F[8], gcl, gel, gcr, ger;
#pragma unroll
        for (int q = 0; q < 6; q++) { VL[q] = w[(long)q * nw + wl]; VR[q] = w[(long)(6 + q) * nw + wr]; }
        X.load_gammas(a, i - di, j - dj, k - dk, gcl, gel);
        X.load_gammas(a, i, j, k, gcr, ger);
        bool shock = false;
        if (EXT && !AMR && a.shok)
            shock = shock_flag(a.shok, i - di, j - dj, k - dk, a.nx, a.ny, a.nz, a.bc) +
                    shock_flag(a.shok, i, j, k, a.nx, a.ny, a.nz, a.bc) > 0;
        int e = riemann<R, EXT>(a.prm, d, VL, gcl, gel, VR, gcr, ger, F, shock);
        if (e) atomicOr(a.err, e);
        if constexpr (EXT) {
            if (a.prm.use_avisc) { avisc3d<R, AMR>(a, X, d, i, j, k, F); eint_fluxes(a.prm, VL, VR, F); }
        }
#pragma unroll
        for (int q = 0; q < NF; q++) f[(long)q * nf + idx] = F[q];
    }
}
template <class R, bool AMR, int DIR, int EXT>
__global__ void __launch_bounds__(256) flux3d_kernel(const Args3D a)
{
    flux3d_kernel_body<R, AMR, DIR, EXT>(a, hw_block());
}

// ---- face states and Riemann fluxes of direction d --------------------------------
// A CTA takes Ls consecutive cells (a segment seg: cells seg*S - 1 ..
// seg*S + S - 1 along d, S = Ls - 1) of T1 neighbouring lines, computes their
// face states, keeps the right-face states in shared memory and solves the
// Riemann problems of the S faces seg*S .. seg*S + S - 1 (the left face of
// each of its cells but the first), so the face states never leave the SM;
// only the pressures of the interior cells' two face states are stored, for
// the update's pressure average.  Threads run along d for d = 0 and along x
// otherwise, so the loads of neighbouring threads are coalesced.  The
// register cap keeps three CTAs of up to 288 threads per SM in FP32 and two
// in FP64.
template <class R> struct SfluxRegs {
    static constexpr int value = (65536 / ((sizeof(R) == 8 ? 2 : 3) * FXB_SF_MAXT)) / 8 * 8;
};
template <class R, int ORDER, bool AMR, int DIR, int EXT>
__device__ __forceinline__ void sflux3d_kernel_body(const Args3D &a, const VB vb, unsigned char *sflux_smem, int nt)
{
    constexpr int d = DIR;
    constexpr int H = ORDER == 3 ? 1 : 0;          // PPM: one slope cell either side of the face-state cells
    R *sW = reinterpret_cast<R *>(sflux_smem);     // [8][threads]: right-face state, then gamc, game
    R *sD = sW + 8 * nt;                           // PPM: [6][threads] limited slopes
    const Ctx3<R, AMR> X(a, vb.y);
    const Grid3 &G = X.G;
    const double dt = a.dtv ? a.dtv[0] : a.dt_arg;
    const double del[3] = {X.dx, X.dy, X.dz};
    const R dtn = R(dt / del[d]), hdtn = R(0.5 * (dt / del[d]));
    const R hdtx = R(0.5 * dt / X.dx), hdty = R(0.5 * dt / X.dy), hdtz = R(0.5 * dt / X.dz);
    const int N = d == 0 ? a.nx : d == 1 ? a.ny : a.nz;
    const int N1 = d == 0 ? a.ny : a.nx, N2 = d == 2 ? a.ny : a.nz;
    const int Ls = a.sf_len[d], T1 = a.sf_lines[d], S = Ls - 1, Lt = Ls + 2 * H;
    const int nseg = (N + S) / S, nt1 = (N1 + T1 - 1) / T1;
    const int t = threadIdx.x;
    const int ld = d == 0 ? t % Lt : t / T1;
    const int l1 = d == 0 ? t / Lt : t % T1;
    const int step = d == 0 ? 1 : T1;              // the neighbour along d, in threads
    int b = vb.x;
    const int seg = b % nseg;
    b /= nseg;
    const int t1 = (b % nt1) * T1 + l1, t2 = b / nt1;
    const int c = seg * S - 1 - H + ld;
    const bool line = t < nt && t1 < N1 && t2 < N2;   // threads beyond the tile only meet the barriers
    const bool st = line && ld >= H && ld < Lt - H && c <= N;   // a face-state cell
    const int i = d == 0 ? c : t1, j = d == 0 ? t1 : d == 1 ? c : t2, k = d == 2 ? c : t2;
    R Wm[6], Wp[6], gc = R(0), ge = R(0);
    if constexpr (ORDER == 3) {
        // the slope of every cell of the segment and its two neighbours (cells
        // -2 .. N+1), then the face states from the slopes in shared memory;
        // a face-state cell reuses its slope's loads and eigensystem
        R S8[3][8], Sr[3][6];
        EigBase<R> eb;
        Eig<R> e;
        if (line && c <= N + 1) {
            int di, dj, dk;
            offs(d, 1, di, dj, dk);
            R g[6];
#pragma unroll
            for (int o = -1; o <= 1; o++) {
                X.load(a, i + o * di, j + o * dj, k + o * dk, S8[o + 1]);
                six(S8[o + 1], g); rot3(d, g, Sr[o + 1]);
            }
            if (!eigen_base(Sr[1][0], Sr[1][4], S8[1][GC], eb)) atomicOr(a.err, ERR_SOUND);
            eigen_dir(eb, Sr[1][1], e);
            R db[6];
            tvd_slope(a.prm, e, Sr[0], Sr[1], Sr[2], db);
#pragma unroll
            for (int q = 0; q < 6; q++) sD[q * nt + t] = db[q];
        }
        __syncthreads();
        if (st) {
            R dbN[6], db0[6], dbP[6], vecL[6], vecR[6];
#pragma unroll
            for (int q = 0; q < 6; q++) {
                dbN[q] = sD[q * nt + t - step];
                db0[q] = sD[q * nt + t];
                dbP[q] = sD[q * nt + t + step];
            }
            ppm_interfaces(Sr[0], Sr[1], Sr[2], dbN, db0, dbP, vecL, vecR);
            if (EXT && a.prm.steepening) {   // densities two cells out along d
                int di, dj, dk;
                offs(d, 1, di, dj, dk);
                R Smm[8], Spp[8];
                X.load(a, i - 2 * di, j - 2 * dj, k - 2 * dk, Smm);
                X.load(a, i + 2 * di, j + 2 * dj, k + 2 * dk, Spp);
                steepen(R(a.prm.tiny), R(d == 0 ? X.dx : d == 1 ? X.dy : X.dz), Smm[D], Sr[0], Sr[1], Sr[2], Spp[D],
                        S8[1][GE], dbN[0], dbP[0], vecL, vecR);
            }
            face_states_tail<R, AMR, DIR, EXT>(a, X, dt, dtn, hdtn, hdtx, hdty, hdtz, i, j, k, Sr[1], S8[1], eb, e,
                                               vecL, vecR, Wm, Wp);
            gc = S8[1][GC];
            ge = S8[1][GE];
        }
    } else {
        if (st) face_states<R, ORDER, AMR, DIR, EXT>(a, X, dt, dtn, hdtn, hdtx, hdty, hdtz, i, j, k, Wm, Wp, gc, ge);
    }
    if (st) {
#pragma unroll
        for (int q = 0; q < 6; q++) sW[q * nt + t] = Wp[q];
        sW[6 * nt + t] = gc;
        sW[7 * nt + t] = ge;
        if (c >= 0 && c < N) {
            R *pw = X.wst[d];
            const long nw = G.nw(d), wc = G.widx(d, i, j, k);
            pw[PwSlots<R>::wp * nw + wc] = Wp[P];
            pw[PwSlots<R>::wm * nw + wc] = Wm[P];
        }
    }
    __syncthreads();
    if (st && ld >= H + 1) {
        const int tl = t - step;
        R VL[6], F[NF];
#pragma unroll
        for (int q = 0; q < 6; q++) VL[q] = sW[q * nt + tl];
        bool shock = false;      // the face between cell (i, j, k) - e_d and (i, j, k)
        if (EXT && !AMR && a.shok) {
            int di, dj, dk;
            offs(d, 1, di, dj, dk);
            shock = shock_flag(a.shok, i - di, j - dj, k - dk, a.nx, a.ny, a.nz, a.bc) +
                    shock_flag(a.shok, i, j, k, a.nx, a.ny, a.nz, a.bc) > 0;
        }
        const int e = riemann<R, EXT>(a.prm, d, VL, sW[6 * nt + tl], sW[7 * nt + tl], Wm, gc, ge, F, shock);
        if (e) atomicOr(a.err, e);
        if constexpr (EXT) {
            if (a.prm.use_avisc) { avisc3d<R, AMR>(a, X, d, i, j, k, F); eint_fluxes(a.prm, VL, Wm, F); }
        }
        R *f = X.flx[d];
        const long nf = G.nf(d), fi = G.fidx(d, i, j, k);
#pragma unroll
        for (int q = 0; q < NF; q++) f[q * nf + fi] = F[q];
    }
}
template <class R, int ORDER, bool AMR, int DIR, int EXT>
__global__ void __launch_bounds__(FXB_SF_MAXT) __maxnreg__(SfluxRegs<R>::value) sflux3d_kernel(const Args3D a)
{
    extern __shared__ __align__(16) unsigned char sflux_smem[];
    sflux3d_kernel_body<R, ORDER, AMR, DIR, EXT>(a, hw_block(), sflux_smem, (int)blockDim.x);
}

// ---- update, energyFix, Eos, CFL rate -------------------------------------------
// four resident CTAs per SM (64 registers, ~200 bytes of spills) measured
// faster on B200 than three (80 registers) and 10-20 % faster than two (128)
#ifndef FXB_UPD_MINB
#define FXB_UPD_MINB 4
#endif
template <class R, bool AMR>
__device__ __forceinline__ void update3d_kernel_body(const Args3D &a, const VB vb)
{
    const Ctx3<R, AMR> X(a, vb.y);
    const Grid3 &G = X.G;
    if (AMR && (X.m.flags & AMR_SKIP_UPDATE)) return;
    const double dt = a.dtv ? a.dtv[0] : a.dt_arg;
    const DevParams &prm = a.prm;
    const long n = (long)a.nx * a.ny * a.nz;
    const double del[3] = {X.dx, X.dy, X.dz};
    double *out = AMR ? a.odata + (long)X.m.out_blk * a.o_bstride : a.out;
    const long ovs = AMR ? a.o_vstride : a.vstride;
    double rate = 0.;
    FXB_VB_LOOP(c, n, vb) {
        int i, j, k;
        unflatten(c, a.fdx[0], a.fdy[0], i, j, k);
        // the update starts from the FP64 state: the grid, or the leaf's interior store
        const long vs = AMR ? a.o_vstride : X.svs;
        const double *in = AMR ? a.istore + (long)X.m.out_blk * a.o_bstride + c : X.src + X.cell(i, j, k);
        double dens0 = in[D * vs];
        double vx0 = in[VX * vs], vy0 = in[VY * vs], vz0 = in[VZ * vs];
        double en0 = in[DV_ENER * vs], eint0 = in[EI * vs];
        double U0[5] = {dens0, vx0 * dens0, vy0 * dens0, vz0 * dens0, dens0 * en0};
        double Sph[5] = {0., 0., 0., 0., 0.};
        double A[3], B[3], pav = 0.;
        for (int d = 0; d < 3; d++) {
            const R *f = X.flx[d];
            const R *w = X.wst[d];
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
            double sum = (double)w[(long)PwSlots<R>::wm * nw + wc] + (double)w[(long)PwSlots<R>::wp * nw + wc];
            if (d == 0) pav = 0.5 * sum;
            else if (d == 1) pav = pav * 0.5 + sum * 0.25;
            else pav = divk<6>(pav * 4.0 + sum);
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
        const double rdens = 1.0 / dens;   // one division for the five quotients by dens
        double vx = rdiv_y(U0[1], dens, rdens), vy = rdiv_y(U0[2], dens, rdens), vz = rdiv_y(U0[3], dens, rdens);
        double ener = rdiv_y(U0[4], dens, rdens);
        double eint = prm.use_aux_eint ? rdiv_y(inten, dens, rdens) : eint0;
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
        double *o = out + c;
        o[D * ovs] = dens; o[VX * ovs] = vx; o[VY * ovs] = vy; o[VZ * ovs] = vz;
        o[P * ovs] = pres; o[GC * ovs] = prm.gamma; o[GE * ovs] = game;
        o[EI * ovs] = eg; o[DV_ENER * ovs] = eg + ek2; o[DV_TEMP * ovs] = temp;
        double cs = sqrt(rdiv_y(prm.gamma * pres, dens, rdens));
        double r = (fabs(vx - 0.) + cs) * (1.0 / X.dx);
        r = fmax2(r, (fabs(vy - 0.) + cs) * (1.0 / X.dy));
        r = fmax2(r, (fabs(vz - 0.) + cs) * (1.0 / X.dz));
        if (c >= a.rate_c0 && c < a.rate_c1) rate = fmax2(rate, r);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, off));
    if ((threadIdx.x & 31) == 0) atomicMax(a.rate_max, (unsigned long long)__double_as_longlong(rate));
}
template <class R, bool AMR>
__global__ void __launch_bounds__(256, FXB_UPD_MINB) update3d_kernel(const Args3D a)
{
    update3d_kernel_body<R, AMR>(a, hw_block());
}

// bytes of the 3-D intermediates for R of the given size
inline size_t sig3d_bytes(int nx, int ny, int nz, size_t rsz)
{ return rsz * 18 * (size_t)(nx + 2) * (ny + 2) * (nz + 2); }
// face states of every cell of direction d: all twelve values (FP64), or the
// pressures of the two (FP32, fused with the fluxes)
inline size_t w3d_bytes(int d, int nx, int ny, int nz, size_t rsz)
{
    size_t n = d == 0 ? (size_t)(nx + 2) * ny * nz : d == 1 ? (size_t)nx * (ny + 2) * nz : (size_t)nx * ny * (nz + 2);
    return rsz * (rsz == 4 ? 2 : 12) * n;
}
// the PPM slope buffer, sized for the largest direction
inline size_t slp3d_bytes(int nx, int ny, int nz, size_t rsz)
{
    size_t m = (size_t)(nx + 4) * ny * nz;
    m = m > (size_t)nx * (ny + 4) * nz ? m : (size_t)nx * (ny + 4) * nz;
    m = m > (size_t)nx * ny * (nz + 4) ? m : (size_t)nx * ny * (nz + 4);
    return rsz * 6 * m;
}
inline size_t f3d_bytes(int d, int nx, int ny, int nz, size_t rsz)
{
    size_t n = d == 0 ? (size_t)(nx + 1) * ny * nz : d == 1 ? (size_t)nx * (ny + 1) * nz : (size_t)nx * ny * (nz + 1);
    return rsz * 8 * n;
}

// face states and fluxes of one direction (PPM: slopes first); g.x CTAs per
// block for the grid-stride kernels, g.y batch entries
template <class R, bool AMR, int DIR, int EXT> void launch_states3d_rs(const Args3D &a, dim3 g, cudaStream_t s)
{
    if constexpr (EXT) {
        if (a.prm.order == 2) {   // MUSCL-Hancock: three cells per face state, no slope pass
            if constexpr (!FusedFaces<R>::value) {
                states3d_kernel<R, 2, AMR, DIR, 1><<<g, 256, 0, s>>>(a);
                flux3d_kernel<R, AMR, DIR, EXT><<<dim3(a.cta[2], g.y), 256, 0, s>>>(a);
            } else {
                const int N = DIR == 0 ? a.nx : DIR == 1 ? a.ny : a.nz;
                const int N1 = DIR == 0 ? a.ny : a.nx, N2 = DIR == 2 ? a.ny : a.nz;
                const int Ls = a.sf_len[DIR], T1 = a.sf_lines[DIR];
                const int nseg = (N + Ls - 1) / (Ls - 1), nt1 = (N1 + T1 - 1) / T1;
                const dim3 gs((unsigned)(nseg * nt1 * N2), g.y);
                sflux3d_kernel<R, 2, AMR, DIR, EXT><<<gs, Ls * T1, 8 * sizeof(R) * (size_t)(Ls * T1), s>>>(a);
            }
            return;
        }
    }
    if constexpr (!FusedFaces<R>::value) {
        // the face states hold no Riemann solve: EXT = 2 runs the EXT = 1 ones
        constexpr int SX = EXT ? 1 : 0;
        if (a.prm.order == 5) {
            states3d_kernel<R, 5, AMR, DIR, SX><<<g, 256, 0, s>>>(a);
        } else {
            slope3d_kernel<R, AMR><<<g, 256, 0, s>>>(a, DIR);
            states3d_kernel<R, 3, AMR, DIR, SX><<<g, 256, 0, s>>>(a);
        }
        flux3d_kernel<R, AMR, DIR, EXT><<<dim3(a.cta[2], g.y), 256, 0, s>>>(a);
    } else {
        const int N = DIR == 0 ? a.nx : DIR == 1 ? a.ny : a.nz;
        const int N1 = DIR == 0 ? a.ny : a.nx, N2 = DIR == 2 ? a.ny : a.nz;
        const int Ls = a.sf_len[DIR], T1 = a.sf_lines[DIR];
        const int nseg = (N + Ls - 1) / (Ls - 1), nt1 = (N1 + T1 - 1) / T1;
        const dim3 gs((unsigned)(nseg * nt1 * N2), g.y);
        if (a.prm.order == 5) {
            sflux3d_kernel<R, 5, AMR, DIR, EXT><<<gs, Ls * T1, 8 * sizeof(R) * (size_t)(Ls * T1), s>>>(a);
        } else {   // the slopes are computed in the kernel: two more cells per line
            const int nt = (Ls + 2) * T1;
            sflux3d_kernel<R, 3, AMR, DIR, EXT><<<gs, nt, 14 * sizeof(R) * (size_t)nt, s>>>(a);
        }
    }
}
// the rarely used options (Roe, contact steepening, MUSCL-Hancock) have kernel instantiations of their own
template <class R, bool AMR, int DIR> void launch_states3d(const Args3D &a, dim3 g, cudaStream_t s)
{
    if (marquina_solver(a.prm)) launch_states3d_rs<R, AMR, DIR, 2>(a, g, s);
    else if (extended_options(a.prm)) launch_states3d_rs<R, AMR, DIR, 1>(a, g, s);
    else launch_states3d_rs<R, AMR, DIR, 0>(a, g, s);
}

// slope cells a face-state tile adds per line: two when the FP32 kernel computes the PPM slopes itself
template <class R> int sflux_halo(const Args3D &a) { return (FusedFaces<R>::value && a.prm.order == 3) ? 2 : 0; }

// hybrid order: DivU (hy_getRiemannState.F90:341-360) on [-3, n+2]^3,
// stored with offset 3 (AMR: per batch entry y, from the guard-filled block)
template <class R, bool AMR>
__global__ void __launch_bounds__(256) divu3d_kernel(const Args3D a, R *divu_base)
{
    const VB vb = hw_block();
    const Ctx3<R, AMR> X(a, vb.y);
    R *divu = divu_base + (AMR ? (long)vb.y * a.divu_bstride : 0L);
    const long ex = a.nx + 6, ey = a.ny + 6, n = ex * ey * (a.nz + 6);
    for (long idx = (long)vb.x * blockDim.x + threadIdx.x; idx < n; idx += (long)vb.nx * blockDim.x) {
        const int i = (int)(idx % ex) - 3, j = (int)((idx / ex) % ey) - 3, k = (int)(idx / (ex * ey)) - 3;
        R dv = X.var(a, VX, i + 1, j, k) - X.var(a, VX, i - 1, j, k);
        dv = dv + X.var(a, VY, i, j + 1, k) - X.var(a, VY, i, j - 1, k);
        dv = dv + X.var(a, VZ, i, j, k + 1) - X.var(a, VZ, i, j, k - 1);
        divu[idx] = R(0.5) * dv;
    }
}
// the flag of every cell of the padded box [-1, n]^3: min DivU over the
// cell's (2 k4 + 1)^3 box below hybridOrderKappa times its sound speed
template <class R, bool AMR>
__global__ void __launch_bounds__(256) hyb3d_kernel(const Args3D a, const R *divu_base, unsigned char *flag_base)
{
    const VB vb = hw_block();
    const Ctx3<R, AMR> X(a, vb.y);
    const R *divu = divu_base + (AMR ? (long)vb.y * a.divu_bstride : 0L);
    unsigned char *flag = flag_base + (AMR ? (long)vb.y * a.hyb_bstride : 0L);
    const Grid3 G{a.nx, a.ny, a.nz};
    const long ex = a.nx + 6, ey = a.ny + 6, np = G.npad();
    const int k4 = a.prm.order - 1 > 2 ? 2 : a.prm.order - 1;
    for (long idx = (long)vb.x * blockDim.x + threadIdx.x; idx < np; idx += (long)vb.nx * blockDim.x) {
        const int i = (int)(idx % (a.nx + 2)) - 1, j = (int)((idx / (a.nx + 2)) % (a.ny + 2)) - 1,
                  k = (int)(idx / ((long)(a.nx + 2) * (a.ny + 2))) - 1;
        const R eps = hybrid_eps(a.prm, X.var(a, D, i, j, k), X.var(a, P, i, j, k), X.var(a, GC, i, j, k));
        R mn = divu[((long)(k - k4 + 3) * ey + (j - k4 + 3)) * ex + (i - k4 + 3)];
        for (int kk = -k4; kk <= k4; kk++)
            for (int jj = -k4; jj <= k4; jj++)
                for (int ii = -k4; ii <= k4; ii++)
                    mn = fmin(mn, divu[((long)(k + kk + 3) * ey + (j + jj + 3)) * ex + (i + ii + 3)]);
        flag[idx] = mn < eps ? 1 : 0;
    }
}
// bytes of the hybrid-order scratch of a uniform grid: DivU in R, then the flags
inline size_t hyb3d_bytes(int nx, int ny, int nz, size_t rsz)
{
    return rsz * (size_t)(nx + 6) * (ny + 6) * (nz + 6) + (size_t)(nx + 2) * (ny + 2) * (nz + 2);
}

// a.cta: the CTAs of each stage (grid-stride kernels of 256 threads)
template <class R> void launch_hydro3d_t(const Args3D &a0, cudaStream_t s)
{
    const Args3D a = with_divisors(a0, sflux_halo<R>(a0));
    const int nsig = a.cta[0], nst = a.cta[1], nupd = a.cta[3];
    if (a.prm.use_hybrid) {
        R *divu = (R *)a.hyb;
        unsigned char *flag = (unsigned char *)a.hyb + sizeof(R) * (size_t)(a.nx + 6) * (a.ny + 6) * (a.nz + 6);
        divu3d_kernel<R, false><<<nsig, 256, 0, s>>>(a, divu);
        hyb3d_kernel<R, false><<<nsig, 256, 0, s>>>(a, divu, flag);
        Args3D b = a;
        b.hyb = flag;
        if (a.prm.flattening) flat3d_kernel<R, false><<<nsig, 256, 0, s>>>(b);
        sig3d_kernel<R, false><<<nsig, 256, 0, s>>>(b);
        launch_states3d<R, false, 0>(b, dim3(nst), s);
        launch_states3d<R, false, 1>(b, dim3(nst), s);
        launch_states3d<R, false, 2>(b, dim3(nst), s);
        update3d_kernel<R, false><<<nupd, 256, 0, s>>>(b);
        return;
    }
    if (a.prm.flattening) flat3d_kernel<R, false><<<nsig, 256, 0, s>>>(a);
    sig3d_kernel<R, false><<<nsig, 256, 0, s>>>(a);
    launch_states3d<R, false, 0>(a, dim3(nst), s);
    launch_states3d<R, false, 1>(a, dim3(nst), s);
    launch_states3d<R, false, 2>(a, dim3(nst), s);
    update3d_kernel<R, false><<<nupd, 256, 0, s>>>(a);
}

// ---- AMR batch: boundary fluxes for flux correction ------------------------------
// Grid_putFluxData: the fluxes on the six boundary faces of every entry,
// [leaf][face][slot][t2 * n1 + t1] with (t1, t2) the face's transverse cell
// (x faces: (y, z); y faces: (x, z); z faces: (x, y)).
template <class R>
__device__ __forceinline__ void amr_emit_flux_kernel_body(const Args3D &a, const VB vb, R *bflux, long nfc)
{
    const Ctx3<R, true> X(a, vb.y);
    const Grid3 &G = X.G;
    const int n[3] = {a.nx, a.ny, a.nz};
    R *dst = bflux + (long)X.m.leaf * 6 * NF * nfc;
    for (int f = 0; f < 6; f++) {
        const int d = f >> 1, side = f & 1;
        const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
        const long nface = (long)n[a1] * n[a2];
        const long nfd = G.nf(d);
        for (long t = vb.x * (long)blockDim.x + threadIdx.x; t < nface * NF; t += (long)vb.nx * blockDim.x) {
            const int v = (int)(t / nface);
            const long tt = t - v * nface;
            const int t1 = (int)(tt % n[a1]), t2 = (int)(tt / n[a1]);
            int c[3];
            c[d] = side ? n[d] : 0; c[a1] = t1; c[a2] = t2;
            dst[((long)f * NF + v) * nfc + tt] = X.flx[d][(long)v * nfd + G.fidx(d, c[0], c[1], c[2])];
        }
    }
}
template <class R>
__global__ void __launch_bounds__(256) amr_emit_flux_kernel(const Args3D a, R *bflux, long nfc)
{
    amr_emit_flux_kernel_body<R>(a, hw_block(), bflux, nfc);
}

// Grid_conserveFluxes: on a face whose same-level neighbour is refined, the
// fluxes become the fine fluxes restricted as amr_restrict_red does:
// (((f(a) + f(a+e1)) + f(a+e2)) + f(a+e1+e2)) * 0.25.  fine[leaf*24 + face*4 + q]
// is the fine leaf across the face at transverse child position q = o1 + 2*o2.
template <class R>
__device__ __forceinline__ void amr_correct_flux_kernel_body(const Args3D &a, const VB vb, const R *bflux, long nfc, const int *fine, const int *finer_mask)
{
    const Ctx3<R, true> X(a, vb.y);
    const Grid3 &G = X.G;
    // leaves whose update waits, or that are never updated (flux ghosts of a split mesh), skip it
    const int mask = (X.m.flags & AMR_SKIP_UPDATE) ? 0 : finer_mask[X.m.leaf];
    if (!mask) return;
    const int n[3] = {a.nx, a.ny, a.nz};
    for (int f = 0; f < 6; f++) {
        if (!((mask >> f) & 1)) continue;
        const int d = f >> 1, side = f & 1;
        const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
        const long nface = (long)n[a1] * n[a2];
        const long nfd = G.nf(d);
        const int ff = f ^ 1;      // the fine leaves' face toward this block
        for (long t = vb.x * (long)blockDim.x + threadIdx.x; t < nface * NF; t += (long)vb.nx * blockDim.x) {
            const int v = (int)(t / nface);
            const long tt = t - v * nface;
            const int t1 = (int)(tt % n[a1]), t2 = (int)(tt / n[a1]);
            const int o1 = (2 * t1) / n[a1], o2 = (2 * t2) / n[a2];
            const int f1 = 2 * t1 - o1 * n[a1], f2 = 2 * t2 - o2 * n[a2];
            const int fl = fine[(long)X.m.leaf * 24 + f * 4 + o1 + 2 * o2];
            const R *src = bflux + (((long)fl * 6 + ff) * NF + v) * nfc;
            // L2 loads: in the persistent AMR kernel another SM stored these this step
            const R fa = __ldcg(src + (long)f2 * n[a1] + f1), fb = __ldcg(src + (long)f2 * n[a1] + f1 + 1);
            const R fc = __ldcg(src + (long)(f2 + 1) * n[a1] + f1), fd = __ldcg(src + (long)(f2 + 1) * n[a1] + f1 + 1);
            int c[3];
            c[d] = side ? n[d] : 0; c[a1] = t1; c[a2] = t2;
            X.flx[d][(long)v * nfd + G.fidx(d, c[0], c[1], c[2])] = (((fa + fb) + fc) + fd) * R(0.25);
        }
    }
}
template <class R>
__global__ void __launch_bounds__(256) amr_correct_flux_kernel(const Args3D a, const R *bflux, long nfc,
                                                               const int *fine, const int *finer_mask)
{
    amr_correct_flux_kernel_body<R>(a, hw_block(), bflux, nfc, fine, finer_mask);
}

// The 3-D pipeline over one AMR batch of `entries` guard-filled blocks; `which`
// selects the stages (AMR_SIG | AMR_STATES), a.cta[] the CTAs per block of the
// grid-stride kernels (the face-state kernel has its own tiles).
template <class R> void launch_amr3d_fluxes_t(const Args3D &a0, int entries, int which, cudaStream_t s)
{
    const Args3D a = with_divisors(a0, sflux_halo<R>(a0));
    if ((which & AMR_SIG) && a.prm.use_hybrid) {
        divu3d_kernel<R, true><<<dim3(a.cta[0], entries), 256, 0, s>>>(a, (R *)a.divu);
        hyb3d_kernel<R, true><<<dim3(a.cta[0], entries), 256, 0, s>>>(a, (const R *)a.divu,
                                                                       const_cast<unsigned char *>(a.hyb));
    }
    if ((which & AMR_SIG) && a.prm.flattening) flat3d_kernel<R, true><<<dim3(a.cta[0], entries), 256, 0, s>>>(a);
    if (which & AMR_SIG) sig3d_kernel<R, true><<<dim3(a.cta[0], entries), 256, 0, s>>>(a);
    if (which & AMR_STATES) {
        launch_states3d<R, true, 0>(a, dim3(a.cta[1], entries), s);
        launch_states3d<R, true, 1>(a, dim3(a.cta[1], entries), s);
        launch_states3d<R, true, 2>(a, dim3(a.cta[1], entries), s);
    }
}
template <class R> void launch_amr3d_emit_t(const Args3D &a, int entries, void *bflux, long nfc, cudaStream_t s)
{
    amr_emit_flux_kernel<R><<<dim3(2, entries), 256, 0, s>>>(a, (R *)bflux, nfc);
}
template <class R> void launch_amr3d_correct_t(const Args3D &a, int entries, const void *bflux, long nfc,
                                               const int *fine, const int *finer_mask, cudaStream_t s)
{
    amr_correct_flux_kernel<R><<<dim3(2, entries), 256, 0, s>>>(a, (const R *)bflux, nfc, fine, finer_mask);
}
template <class R> void launch_amr3d_update_t(const Args3D &a0, int entries, cudaStream_t s)
{
    const Args3D a = with_divisors(a0);
    update3d_kernel<R, true><<<dim3(a.cta[3], entries), 256, 0, s>>>(a);
}

} // namespace fxb
