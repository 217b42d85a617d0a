// fxb_amr_dev.cuh -- device-side description of a block-structured AMR mesh
// and the guard-cell arithmetic shared by the AMR kernels: same-level
// copies, PARAMESH's multilinear prolongation in conserved form
// (amr_1blk_cc_prol_linear), Eos on guard regions, and the restriction of
// parent cells (amr_restrict_unk_genorder).  Included by the AMR host code
// and by the precision translation units that instantiate the persistent
// AMR kernel.
#pragma once
#include "../../include/flashx_b200.h"
#include "fxb_device.cuh"
#include "fxb_hydro3d.cuh"

namespace fxb {

struct DevBlk {
    int level, c0, c1, c2, parent;
};

// device-side description of the mesh for the guard-fill kernels
struct MeshArgs {
    const DevBlk *blk;
    const int *ntab;            // [block][27] same-level neighbour, -1 none, -2 boundary
    const double *store;        // interior store [block][var][cell]
    long vstride, bstride;      // cells per block, NV_DEV * cells
    int n, ng;                  // cells per block side, guard layers
    int nb1[3];                 // root blocks per axis
    int bc[6];
    int *err;
};

constexpr int ERR_AMR = 16;
// variables of the guard-filled blocks: D..EI, all the 3-D pipeline reads
// (ENER feeds the guard cells' Eos, TEMP nothing); artificial viscosity adds
// ENER, the next variable
constexpr int NV_GCB = EI + 1;
static_assert(DV_ENER == NV_GCB, "total energy follows the guard-filled variables");     // guard cell without a covering block (device error word)


// ------------------------------------------------------------------ device
__device__ __forceinline__ int fdiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// PER_MASS variables of UNK (velx vely velz ener eint) in device order
__device__ __forceinline__ bool per_mass(int v) { return v == VX || v == VY || v == VZ || v == DV_ENER || v == EI; }

// Eos_wrapped(MODE_DENS_EI) of one cell (Gamma/Eos.F90:238-250)
__device__ inline void eos_cell_dev(double u[NV_DEV], const DevParams &prm, double gam1inv, double ggprodinv)
{
    double ekin = 0.5 * (u[VX] * u[VX] + u[VY] * u[VY] + u[VZ] * u[VZ]);
    double eint = u[EI];
    if (u[DV_ENER] - ekin > fmax2(prm.small_e, prm.eint_switch * ekin)) eint = u[DV_ENER] - ekin;
    double dens = u[D];
    double pres = dens * eint * gam1inv;
    u[P] = pres;
    u[DV_TEMP] = eint * ggprodinv * prm.abar;
    u[GC] = prm.gamma;
    u[EI] = eint;
    u[DV_ENER] = eint + ekin;
    u[GE] = pres / (eint * dens) + 1;
}

// non-periodic boundary map of one level-l cell index along axis a
__device__ __forceinline__ int bc_map(const MeshArgs &m, int lev, int a, int x, double *sg)
{
    const int N = (m.nb1[a] << (lev - 1)) * m.n;
    if (x < 0) {
        int bc = m.bc[2 * a];
        if (bc == FXB_BC_OUTFLOW) return 0;
        if (bc == FXB_BC_REFLECTING) { *sg = -*sg; return -1 - x; }
    } else if (x >= N) {
        int bc = m.bc[2 * a + 1];
        if (bc == FXB_BC_OUTFLOW) return N - 1;
        if (bc == FXB_BC_REFLECTING) { *sg = -*sg; return 2 * N - 1 - x; }
    }
    return x;   // inside, or periodic (left unwrapped: the neighbour table wraps)
}

// store offset (variable 0) of the level-lev cell x (unwrapped along periodic
// axes, inside along the others) in the block holding it among block b's 27
// neighbours, or -1
__device__ __forceinline__ long same_level_off(const MeshArgs &m, int b, const DevBlk &B, const int x[3])
{
    int r[3], loc[3];
    const int bc[3] = {B.c0, B.c1, B.c2};
    for (int a = 0; a < 3; a++) {
        r[a] = fdiv(x[a] - bc[a] * m.n, m.n);
        if (r[a] < -1 || r[a] > 1) return -1;
        loc[a] = x[a] - (bc[a] + r[a]) * m.n;
    }
    int nb = m.ntab[(long)b * 27 + (r[2] + 1) * 9 + (r[1] + 1) * 3 + (r[0] + 1)];
    if (nb < 0) return -1;
    return (long)nb * m.bstride + ((long)loc[2] * m.n + loc[1]) * m.n + loc[0];
}

// Where the guard value of one cell of a leaf comes from: a same-level cell
// (a leaf or a restricted parent), or the eight parent-level cells of the
// prolongation stencil, as store offsets of variable 0, with the sign flips
// of reflecting boundaries (bit a: the velocity along axis a changes sign).
enum { GS_SAME = 0, GS_PROL = 1, GS_NONE = 2 };
struct GuardSrc {
    int kind;
    unsigned own;       // flips of the cell's own boundary map
    unsigned parity;    // prolongation weights: bit a = x[a] & 1
    unsigned flips;     // prolongation: three flip bits per stencil cell
    long off[8];
};

// the prolongation stencil of the level-lev cell x (mapped into the domain) of
// block B: amr_1blk_cc_prol_linear from the eight parent-level cells
// floor((x+1)/2)-1 and +1 per axis, found among the parent's neighbours
__device__ __forceinline__ void prol_resolve(const MeshArgs &m, const DevBlk &B, const int x[3], GuardSrc &gs)
{
    gs.kind = GS_NONE;
    if (B.parent < 0) return;
    const int pb = B.parent;
    const DevBlk PB = m.blk[pb];
    int p1[3];
    for (int a = 0; a < 3; a++) {
        p1[a] = fdiv(x[a] + 1, 2) - 1;
        gs.parity |= (unsigned)(x[a] & 1) << a;
    }
#pragma unroll
    for (int s8 = 0; s8 < 8; s8++) {
        const int ii = s8 & 1, jj = (s8 >> 1) & 1, kk = s8 >> 2;
        int q[3] = {p1[0] + ii, p1[1] + jj, p1[2] + kk};
        double sq[3] = {1., 1., 1.};
        for (int a = 0; a < 3; a++) q[a] = bc_map(m, PB.level, a, q[a], &sq[a]);
        gs.off[s8] = same_level_off(m, pb, PB, q);
        if (gs.off[s8] < 0) return;
        gs.flips |= ((sq[0] < 0. ? 1u : 0u) | (sq[1] < 0. ? 2u : 0u) | (sq[2] < 0. ? 4u : 0u)) << (3 * s8);
    }
    gs.kind = GS_PROL;
}

__device__ __forceinline__ void guard_resolve(const MeshArgs &m, int b, const int xin[3], GuardSrc &gs)
{
    const DevBlk B = m.blk[b];
    int x[3];
    double sg[3] = {1., 1., 1.};
    for (int a = 0; a < 3; a++) x[a] = bc_map(m, B.level, a, xin[a], &sg[a]);
    gs.own = (sg[0] < 0. ? 1u : 0u) | (sg[1] < 0. ? 2u : 0u) | (sg[2] < 0. ? 4u : 0u);
    gs.parity = 0; gs.flips = 0;
    gs.off[0] = same_level_off(m, b, B, x);
    if (gs.off[0] >= 0) { gs.kind = GS_SAME; return; }
    prol_resolve(m, B, x, gs);
}

// same-level guard value: the cell's first NV variables, velocities flipped at reflecting boundaries
template <int NV = NV_DEV>
__device__ __forceinline__ void guard_eval_same(const double *store, long vstride, long off, unsigned own,
                                                double out[NV_DEV])
{
    const double *s = store + off;
#pragma unroll
    for (int v = 0; v < NV; v++) out[v] = s[v * vstride];
#pragma unroll
    for (int a = 0; a < 3; a++)
        if ((own >> a) & 1u) out[VX + a] = out[VX + a] * -1.;
}

// prolonged guard value (amr_1blk_cc_prol_linear, conserved form): weights
// 0.25 / 0.75 by the cell's parity per axis, per-mass variables times the
// stencil cells' densities, divided by the interpolated density after
__device__ __forceinline__ void guard_eval_prol(const double *store, long vstride, const long off[8], unsigned flips,
                                                unsigned parity, unsigned own, double out[NV_DEV])
{
    double dn[8];
#pragma unroll
    for (int s8 = 0; s8 < 8; s8++) dn[s8] = store[off[s8] + D * vstride];
    const double wx = (parity & 1u) ? 0.75 : 0.25, wy = ((parity >> 1) & 1u) ? 0.75 : 0.25,
                 wz = ((parity >> 2) & 1u) ? 0.75 : 0.25;
    const double dx = wx, cx = 1. - wx, dy = wy, cy = 1. - wy, dz = wz, cz = 1. - wz;
#pragma unroll
    for (int v = 0; v < NV_DEV; v++) {
        double S[8];
#pragma unroll
        for (int s8 = 0; s8 < 8; s8++) {
            double x8 = store[off[s8] + v * vstride];
            if (v >= VX && v <= VZ && ((flips >> (3 * s8 + v - VX)) & 1u)) x8 = x8 * -1.;
            S[s8] = per_mass(v) ? dn[s8] * x8 : x8;
        }
        // S[(kk*2 + jj)*2 + ii]
        out[v] = dz * (dy * (dx * S[0] + cx * S[1]) + cy * (dx * S[2] + cx * S[3])) +
                 cz * (dy * (dx * S[4] + cx * S[5]) + cy * (dx * S[6] + cx * S[7]));
    }
    double dinv = out[D] == 0.0 ? 0.0 : 1. / out[D];
#pragma unroll
    for (int v = 0; v < NV_DEV; v++)
        if (per_mass(v)) out[v] = dinv * out[v];
#pragma unroll
    for (int a = 0; a < 3; a++)
        if ((own >> a) & 1u) out[VX + a] = out[VX + a] * -1.;
}

// guard value of leaf block b at level-lev cell x
__device__ __forceinline__ bool guard_value(const MeshArgs &m, int b, const int xin[3], double out[NV_DEV])
{
    GuardSrc gs;
    guard_resolve(m, b, xin, gs);
    if (gs.kind == GS_SAME) guard_eval_same(m.store, m.vstride, gs.off[0], gs.own, out);
    else if (gs.kind == GS_PROL) guard_eval_prol(m.store, m.vstride, gs.off, gs.flips, gs.parity, gs.own, out);
    return gs.kind != GS_NONE;
}


struct GuardPlan {
    unsigned off;       // same-level source: store offset of variable 0
    unsigned flags;     // bits 0-2 own flips, bit 3 Eos, bits 4-5 kind
};
struct __align__(16) ProlRec {
    unsigned idx;       // extended-block offset of the guard cell
    unsigned flags;     // bits 0-2 parity, 3-5 own flips, 6 Eos, 8-31 stencil flips
    unsigned off[8];    // stencil cells' store offsets (variable 0)
    unsigned pad[2];
};

__device__ __forceinline__ void ext_coords(long idx, int ne, int g, int &i, int &j, int &k)
{
    i = (int)(idx % ne) - g; j = (int)((idx / ne) % ne) - g; k = (int)(idx / ((long)ne * ne)) - g;
}


// interior cells and same-level guard cells of a batch from the plan
template <class T>
__device__ __forceinline__ void amr_copy_kernel_body(const VB vb, MeshArgs m, const AmrEntry3 *entries, const int *leaf_blk, const GuardPlan *plan, const int *glist, int nglist, T *out, long gvs, long gbs, DevParams prm, double gam1inv, double ggprodinv)
{
    const AmrEntry3 e = entries[vb.y];
    const int b = leaf_blk[e.leaf];
    const int n = m.n, g = m.ng, ne = n + 2 * g;
    const long nint = (long)n * n * n;
    const long ncell = nint + nglist;
    T *dst = out + (long)vb.y * gbs;
    const GuardPlan *pl = plan + (long)e.leaf * nglist;
    const bool wide = gbs > NV_GCB * gvs;   // blocks with total energy (artificial viscosity)
    for (int t = (int)(vb.x * blockDim.x + threadIdx.x); t < (int)ncell; t += (int)(vb.nx * blockDim.x)) {
        double u[NV_DEV];
        int idx;
        if (t < nint) {
            int i, j, k;
            unflatten(t, n, n, i, j, k);
            idx = ((k + g) * ne + j + g) * ne + i + g;
            const double *s = m.store + (long)b * m.bstride + t;
#pragma unroll
            for (int v = 0; v < NV_GCB; v++) u[v] = s[v * m.vstride];
            if (wide) u[DV_ENER] = s[DV_ENER * m.vstride];
        } else {
            const GuardPlan gp = pl[t - nint];
            const unsigned kind = (gp.flags >> 4) & 3u;
            if (kind == GS_PROL) continue;
            idx = glist[t - nint];
            if (kind == GS_NONE) {
                atomicOr(m.err, ERR_AMR);
#pragma unroll
                for (int v = 0; v < NV_DEV; v++) u[v] = 0.;
            } else if ((gp.flags >> 3) & 1u) {
                guard_eval_same<NV_DEV>(m.store, m.vstride, gp.off, gp.flags & 7u, u);
                eos_cell_dev(u, prm, gam1inv, ggprodinv);
            } else {
                guard_eval_same<NV_GCB>(m.store, m.vstride, gp.off, gp.flags & 7u, u);
                if (wide) u[DV_ENER] = m.store[gp.off + DV_ENER * m.vstride];
            }
        }
#pragma unroll
        for (int v = 0; v < NV_GCB; v++) dst[v * gvs + idx] = (T)u[v];
        if (wide) dst[DV_ENER * gvs + idx] = (T)u[DV_ENER];
    }
}
template <class T>
__device__ __forceinline__ void amr_prolong_kernel_body(const VB vb, MeshArgs m, const AmrEntry3 *entries, const ProlRec *prol, const int *poff, T *out, long gvs, long gbs, DevParams prm, double gam1inv, double ggprodinv)
{
    const AmrEntry3 e = entries[vb.y];
    const int r0 = poff[e.leaf], r1 = poff[e.leaf + 1];
    T *dst = out + (long)vb.y * gbs;
    for (int r = r0 + vb.x * blockDim.x + threadIdx.x; r < r1; r += vb.nx * blockDim.x) {
        const uint4 *q = reinterpret_cast<const uint4 *>(prol + r);
        const uint4 a = q[0], bq = q[1], c = q[2];
        const long off[8] = {(long)a.z, (long)a.w, (long)bq.x, (long)bq.y, (long)bq.z, (long)bq.w, (long)c.x, (long)c.y};
        const unsigned fl = a.y;
        double u[NV_DEV];
        guard_eval_prol(m.store, m.vstride, off, fl >> 8, fl & 7u, (fl >> 3) & 7u, u);
        if ((fl >> 6) & 1u) eos_cell_dev(u, prm, gam1inv, ggprodinv);
        const long idx = a.x;
#pragma unroll
        for (int v = 0; v < NV_GCB; v++) dst[v * gvs + idx] = (T)u[v];
        if (gbs > NV_GCB * gvs) dst[DV_ENER * gvs + idx] = (T)u[DV_ENER];
    }
}

// restriction of parent cell c of block p from its eight children cells
// (amr_restrict_unk_genorder, order 1): conserved form, weights 1/8 in k, j, i order
__device__ __forceinline__ void restrict_cell(double *store, long vstride, long bstride, int n, int p, int c,
                                              const int *child)
{
    const int h = n / 2;
    const int pi = c % n, pj = (c / n) % n, pk = c / (n * n);
    const int q = (pi >= h) | ((pj >= h) << 1) | ((pk >= h) << 2);
    const int ch = child[(long)p * 8 + q];
    const int i0 = 2 * (pi - (q & 1) * h), j0 = 2 * (pj - ((q >> 1) & 1) * h), k0 = 2 * (pk - ((q >> 2) & 1) * h);
    const double *cs = store + (long)ch * bstride;
    double s[NV_DEV];
#pragma unroll
    for (int v = 0; v < NV_DEV; v++) s[v] = 0.;
    const double w = 0.5 * 0.5 * 0.5;
    for (int kk = 0; kk < 2; kk++) for (int jj = 0; jj < 2; jj++) for (int ii = 0; ii < 2; ii++) {
        const long cc = ((long)(k0 + kk) * n + (j0 + jj)) * n + (i0 + ii);
        const double dens = cs[D * vstride + cc];
#pragma unroll
        for (int v = 0; v < NV_DEV; v++) {
            double x = cs[v * vstride + cc];
            if (per_mass(v)) x = dens * x;
            s[v] = s[v] + w * x;
        }
    }
    double dinv = s[D] == 0.0 ? 0.0 : 1. / s[D];
    double *ps = store + (long)p * bstride + c;
#pragma unroll
    for (int v = 0; v < NV_DEV; v++) ps[v * vstride] = per_mass(v) ? dinv * s[v] : s[v];
}


} // namespace fxb
