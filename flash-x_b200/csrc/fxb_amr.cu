// fxb_amr.cu -- block-structured AMR (PARAMESH layout) for the 3-D hydro path.
//
// One Hydro() step on a frozen mesh of leaf blocks at several refinement
// levels, as levelFlux/Hydro.F90:161-270 does it with PARAMESH:
//   1. restriction of every parent from its children, deepest level first,
//      in conserved form (mpi_amr_1blk_restrict.F90:303-325,813 with the
//      order-1 weights of amr_restrict_unk_genorder.F90)
//   2. guard cells of every leaf: copied from the same-level block (leaf, or
//      parent holding restricted data) or, where the neighbour is coarser,
//      interpolated multilinearly from the parent level in conserved form
//      (amr_1blk_cc_prol_linear.F90 with the index map of
//      amr_prolong_cc_fun_init.F90, PER_MASS variables multiplied by dens
//      before and divided after: flash_(un)convert_cc_hook.F90); boundary
//      conditions map positions into the domain first; Eos(MODE_DENS_EI) on
//      the guard regions whose neighbour is at another level
//      (Eos_guardCells.F90 with corners and skipSrl)
//   3. fluxes of every leaf with the 3-D pipeline of fxb_hydro3d.cuh,
//      boundary fluxes saved (Grid_putFluxData), fluxes on faces next to
//      finer leaves replaced by the restricted fine fluxes
//      (Grid_conserveFluxes, amr_restrict_red.F90), then the update,
//      energyFix, Eos and the CFL rate of every leaf.
// The leaves' interiors live in two stores swapped every step; guard-filled
// blocks and the pipeline intermediates exist for one batch of leaves at a
// time, sized to the free device memory.
#include "fxb_amr.h"
#include "fxb_launch.h"
#include "fxb_amr_dev.cuh"
#include "fxb_amr_persist.cuh"

#include <algorithm>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <type_traits>
#include <unordered_map>
#include <vector>

namespace fxb {
namespace {

struct HBlock {
    int level;
    int c[3];
    int parent;
    int child[8];
    int leaf;        // leaf slot or -1
    int nodetype;    // 1 leaf, 2 parent with a leaf child, 3 other parent
};

struct State {
    bool active = false;
    AmrCommon C{};
    int n = 0, ng = 0, nleaf = 0, nblk = 0, maxlev = 1;
    std::vector<HBlock> blk;
    std::vector<int> leaf_blk;
    std::vector<std::vector<int>> parents_at;     // per level (1-based index)
    // device
    double *store[2] = {nullptr, nullptr};
    int cur = 0;
    long vstride = 0, bstride = 0;
    DevBlk *d_blk = nullptr;
    int *d_ntab = nullptr, *d_child = nullptr, *d_plist = nullptr;
    std::vector<long> plist_off;                  // per level offset into d_plist
    unsigned *d_eosmask = nullptr;
    int *d_finer = nullptr, *d_fine = nullptr;
    double *d_dxl = nullptr;
    AmrEntry3 *d_entries = nullptr;               // [all][all, finer ones skipped][finer ones]
    int batch = 0;
    void *gcb = nullptr;                          // guard-filled blocks in the reconstruction type
    int ngcb = NV_GCB;                            // their variables (NV_GCB, + total energy with avisc)
    void *hyb = nullptr;                          // hybrid order: DivU [batch][(n+6)^3] of R, then flags [batch][(n+2)^3]
    void *sig = nullptr, *w[3] = {nullptr, nullptr, nullptr}, *f[3] = {nullptr, nullptr, nullptr};
    void *slp = nullptr;                          // PPM slopes of one direction per batch entry
    void *flat = nullptr;                         // flattening coefficients per batch entry
    void *bflux = nullptr;
    long nfc = 0;
    double *stage = nullptr;                      // UNK staging for attach / sync
    int stage_leaves = 0;
    int *leaf_blk_dev = nullptr, *d_dmap = nullptr;
    int *d_pmap = nullptr;                        // device variable -> place in a packed guard fill
    int nfiner = 0;
    int *d_glist = nullptr;                       // guard cells the pipeline reads (extended-block offsets)
    int nglist = 0;
    void *d_plan = nullptr;                       // GuardPlan [leaf][nglist]
    void *d_prol = nullptr;                       // ProlRec, per leaf from d_poff[leaf]
    int *d_poff = nullptr;
    long nprol = 0;
    int2 *d_rlist = nullptr;                      // parent cells the plan needs, per level (restriction order)
    std::vector<int> act_blk;                     // leaves and parents with a leaf child (refinement marking)
    int *d_active = nullptr;
    unsigned *d_act_eos = nullptr, *d_act_bnd = nullptr;
    double *d_ext = nullptr, *d_err = nullptr;    // marking scratch, allocated at the first marking
    std::vector<long> rlist_off;                  // per level offset into d_rlist, size maxlev + 1
    int cta[4] = {4, 4, 4, 4};                    // CTAs per block: sig, slopes, (unused), update
    int fill_cta = 8;
    bool tuned = false;                           // launch shapes chosen (first attach of the mesh)
    char tune_log[512] = "";
    std::unordered_map<uint64_t, int> map;
    // one rank's share of a mesh split over ranks (fxb_amr_set_roles): per leaf
    // 1 owned, 2 flux ghost, 0 not stepped; the step's entry lists over the
    // active leaves (same three parts as d_entries)
    std::vector<unsigned char> roles;
    std::vector<int> finer_h;                     // per leaf: faces toward finer leaves (d_finer)
    unsigned char *d_roles = nullptr;
    AmrEntry3 *d_step_entries = nullptr;
    AmrEntry3 *d_leaf_entry = nullptr;            // entry of every leaf with its role's flags
    int nstep = 0, nstep_finer = 0;
    int *d_xlist = nullptr;                       // leaf list of the last exchange message
    int xcap = 0;
    // a split mesh's host UNK holds the own leaves only (in leaf order)
    int nown = 0;
    int *d_own_blk = nullptr;                     // their blocks in the interior store
    AmrEntry3 *d_own_entries = nullptr;           // their fill entries
    // the step as one persistent kernel over the leaf list (fxb_amr_persist.cuh)
    bool persist = false;
    bool persist_ok = false;                      // the mesh and options allow the persistent kernel
    int pK = 4;                                   // CTAs per cluster (one leaf per cluster)
    int pclusters = 0;                            // resident clusters, one scratch slot each
    int pslots = 0;                               // slots allocated (the most clusters of any K)
    int *d_order = nullptr;                       // leaves in queue order, finest level first
    int *d_ctl = nullptr;                         // queue head, completion counters, abort flag
    int *d_emitted = nullptr;                     // per leaf: boundary fluxes stored
    int4 *d_ritems = nullptr;                     // restriction items (level, first, last+1)
    AmrEntry3 *d_slots = nullptr;                 // the leaf each CTA runs
    int nritem = 0;
    int rlev_items[32] = {};
    long long wait_budget = kTmaWaitBudget;
    int test_stall = 0;                           // test hook (FXB_TEST_WAIT_TIMEOUT)
};
State S;

uint64_t key(int lev, const int c[3])
{
    return ((uint64_t)lev << 60) | ((uint64_t)(uint32_t)c[0] << 40) | ((uint64_t)(uint32_t)c[1] << 20) |
           (uint64_t)(uint32_t)c[2];
}

int find(int lev, const int c[3])
{
    auto it = S.map.find(key(lev, c));
    return it == S.map.end() ? -1 : it->second;
}

int nb_at(int lev, int d)
{
    const fxb_domain &D = S.C.dom;
    int n0 = d == 0 ? D.nblockx : d == 1 ? D.nblocky : D.nblockz;
    return n0 << (lev - 1);
}

int new_block(int lev, const int c[3])
{
    HBlock b;
    b.level = lev;
    for (int d = 0; d < 3; d++) b.c[d] = c[d];
    b.parent = -1;
    for (int q = 0; q < 8; q++) b.child[q] = -1;
    b.leaf = -1;
    b.nodetype = 3;
    S.blk.push_back(b);
    int id = (int)S.blk.size() - 1;
    S.map[key(lev, c)] = id;
    return id;
}

// same-level neighbour: block, -1 none at that level, -2 outside a non-periodic boundary
int neigh(int b, int di, int dj, int dk)
{
    const HBlock &B = S.blk[b];
    int off[3] = {di, dj, dk}, c[3];
    for (int d = 0; d < 3; d++) {
        c[d] = B.c[d] + off[d];
        int nb = nb_at(B.level, d);
        if (c[d] < 0 || c[d] >= nb) {
            if (S.C.dom.bc[2 * d + (c[d] >= nb)] != FXB_BC_PERIODIC) return -2;
            c[d] = (c[d] + nb) % nb;
        }
    }
    return find(B.level, c);
}

// Grid_getBlkNeighLevels(trackBdry) + Eos_guardCells(corners, skipSrl): bit r
// set for every guard region r = (rk+1)*9 + (rj+1)*3 + (ri+1) whose
// neighbour level differs from the block's own
unsigned eos_regions(int b)
{
    const int me = S.blk[b].level;
    int lev[3][3][3], bnd[3][3][3];
    for (int k = -1; k <= 1; k++) for (int j = -1; j <= 1; j++) for (int i = -1; i <= 1; i++) {
        int nb = (i | j | k) ? neigh(b, i, j, k) : b;
        bnd[i + 1][j + 1][k + 1] = nb == -2;
        if (nb == -1) lev[i + 1][j + 1][k + 1] = me - 1;
        else if (nb >= 0 && S.blk[nb].nodetype == 2) lev[i + 1][j + 1][k + 1] = me + 1;
        else lev[i + 1][j + 1][k + 1] = me;
    }
    for (int pass = 2; pass <= 3; pass++) {
        for (int k = -1; k <= 1; k++) for (int j = -1; j <= 1; j++) for (int i = -1; i <= 1; i++) {
            if (abs(i) + abs(j) + abs(k) != pass) continue;
            if (lev[i + 1][j + 1][k + 1] != me || !bnd[i + 1][j + 1][k + 1]) continue;
            // the k range of the reference ends at min(1, j+1)
            int klo = std::max(-1, k - 1), khi = std::min(1, j + 1);
            int ilo = std::max(-1, i - 1), ihi = std::min(1, i + 1);
            int jlo = std::max(-1, j - 1), jhi = std::min(1, j + 1);
            int mn = INT32_MAX, mx = INT32_MIN;
            for (int kk = klo; kk <= khi; kk++) for (int jj = jlo; jj <= jhi; jj++) for (int ii = ilo; ii <= ihi; ii++) {
                mn = std::min(mn, lev[ii + 1][jj + 1][kk + 1]);
                mx = std::max(mx, lev[ii + 1][jj + 1][kk + 1]);
            }
            lev[i + 1][j + 1][k + 1] = mn < me ? mn : mx;
        }
    }
    unsigned mask = 0;
    for (int k = -1; k <= 1; k++) for (int j = -1; j <= 1; j++) for (int i = -1; i <= 1; i++)
        if ((i | j | k) && lev[i + 1][j + 1][k + 1] != me) mask |= 1u << ((k + 1) * 9 + (j + 1) * 3 + (i + 1));
    return mask;
}

int build_tree(const fxb_block_desc *leaves, int nleaf, std::vector<int> &finer, std::vector<int> &fine)
{
    S.blk.clear();
    S.map.clear();
    S.blk.reserve(2 * (size_t)nleaf + 64);
    S.leaf_blk.assign(nleaf, -1);
    S.maxlev = 1;
    for (int l = 0; l < nleaf; l++) {
        int lev = leaves[l].level;
        int c[3] = {leaves[l].bcoord[0], leaves[l].bcoord[1], leaves[l].bcoord[2]};
        if (lev < 1 || lev > 15) return record_error(FXB_EARG, "fxb_register_blocks: refinement level out of range");
        for (int d = 0; d < 3; d++)
            if (c[d] < 0 || c[d] >= nb_at(lev, d))
                return record_error(FXB_EARG, "fxb_register_blocks: block coordinate out of range");
        if (find(lev, c) >= 0) return record_error(FXB_EARG, "fxb_register_blocks: duplicate leaf");
        int id = new_block(lev, c);
        S.blk[id].leaf = l;
        S.blk[id].nodetype = 1;
        S.leaf_blk[l] = id;
        S.maxlev = std::max(S.maxlev, lev);
    }
    for (int l = 0; l < nleaf; l++) {
        int id = S.leaf_blk[l];
        while (S.blk[id].level > 1) {
            int pc[3] = {S.blk[id].c[0] / 2, S.blk[id].c[1] / 2, S.blk[id].c[2] / 2};
            int plev = S.blk[id].level - 1;
            int pid = find(plev, pc);
            if (pid < 0) pid = new_block(plev, pc);
            else if (S.blk[pid].leaf >= 0)
                return record_error(FXB_EARG, "fxb_register_blocks: a leaf overlaps another leaf's parent");
            int q = (S.blk[id].c[0] & 1) | ((S.blk[id].c[1] & 1) << 1) | ((S.blk[id].c[2] & 1) << 2);
            S.blk[pid].child[q] = id;
            S.blk[id].parent = pid;
            id = pid;
        }
    }
    long roots = 0, nroot = (long)nb_at(1, 0) * nb_at(1, 1) * nb_at(1, 2);
    for (auto &B : S.blk) {
        if (B.level == 1) roots++;
        if (B.leaf >= 0) continue;
        bool any_leaf = false;
        for (int q = 0; q < 8; q++) {
            if (B.child[q] < 0) return record_error(FXB_EARG, "fxb_register_blocks: the leaves do not tile the domain");
            if (S.blk[B.child[q]].leaf >= 0) any_leaf = true;
        }
        B.nodetype = any_leaf ? 2 : 3;
    }
    if (roots != nroot) return record_error(FXB_EARG, "fxb_register_blocks: the leaves do not tile the domain");
    S.nblk = (int)S.blk.size();
    // 2:1 balance across faces, edges and corners
    for (int l = 0; l < nleaf; l++) {
        int b = S.leaf_blk[l];
        for (int k = -1; k <= 1; k++) for (int j = -1; j <= 1; j++) for (int i = -1; i <= 1; i++) {
            if (!(i | j | k)) continue;
            int nb = neigh(b, i, j, k);
            if (nb >= 0 && S.blk[nb].nodetype == 3)
                return record_error(FXB_EARG, "fxb_register_blocks: neighbouring leaves differ by more than one level");
            if (nb == -1) {
                int off[3] = {i, j, k}, c[3];
                for (int d = 0; d < 3; d++) {
                    int nbd = nb_at(S.blk[b].level, d);
                    c[d] = ((S.blk[b].c[d] + off[d]) % nbd + nbd) % nbd / 2;
                }
                int cov = find(S.blk[b].level - 1, c);
                if (cov < 0 || S.blk[cov].leaf < 0)
                    return record_error(FXB_EARG, "fxb_register_blocks: neighbouring leaves differ by more than one level");
            }
        }
    }
    // faces next to refined regions and the fine leaves across them
    finer.assign(nleaf, 0);
    fine.assign((size_t)nleaf * 24, -1);
    for (int l = 0; l < nleaf; l++) {
        int b = S.leaf_blk[l];
        for (int f = 0; f < 6; f++) {
            int d = f >> 1, side = f & 1;
            int off[3] = {0, 0, 0};
            off[d] = side ? 1 : -1;
            int nb = neigh(b, off[0], off[1], off[2]);
            if (nb < 0 || S.blk[nb].nodetype != 2) continue;
            finer[l] |= 1 << f;
            int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
            for (int q = 0; q < 4; q++) {
                int cc[3];
                cc[d] = S.blk[nb].c[d] * 2 + (side ? 0 : 1);
                cc[a1] = 2 * S.blk[nb].c[a1] + (q & 1);
                cc[a2] = 2 * S.blk[nb].c[a2] + (q >> 1);
                int fb = find(S.blk[b].level + 1, cc);
                if (fb < 0 || S.blk[fb].leaf < 0)
                    return record_error(FXB_EARG, "fxb_register_blocks: neighbouring leaves differ by more than one level");
                fine[(size_t)l * 24 + f * 4 + q] = S.blk[fb].leaf;
            }
        }
    }
    return FXB_OK;
}

// guard-filled copies of a batch of leaves, in the reconstruction type T:
// out[entry][var][nz+2g][ny+2g][nx+2g]; with TO_UNK the FP64 values go into
// UNK staging instead, out[leaf][k][j][i][nunk] at the variables' UNK slots.
// Three resident 256-thread CTAs per SM (80 registers) measured faster on
// B200 than two (96) or four (64, with spills).
#ifndef FXB_FILL_MINB
#define FXB_FILL_MINB 3
#endif
// With a guard list (glist != nullptr) only the interior and the listed guard
// cells (linear offsets in the extended block) are filled: the cells the
// pipeline kernels read; without one every cell of the extended block is.
template <class T, bool TO_UNK>
__global__ void __launch_bounds__(256, FXB_FILL_MINB) amr_fill_kernel(MeshArgs m, const AmrEntry3 *entries, const int *leaf_blk,
                                                       const unsigned *eosmask, T *out, long gvs, long gbs,
                                                       int nunk, const int *dmap, const int *glist, int nlist,
                                                       DevParams prm, double gam1inv, double ggprodinv)
{
    const AmrEntry3 e = entries[blockIdx.y];
    const int b = leaf_blk[e.leaf];
    const DevBlk B = m.blk[b];
    const unsigned mask = eosmask ? eosmask[e.leaf] : 0u;     // no mask: no Eos on guard cells
    const int n = m.n, g = m.ng, ne = n + 2 * g;
    const long nint = (long)n * n * n;
    const long ncell = glist ? nint + nlist : (long)ne * ne * ne;
    T *dst = out + (long)blockIdx.y * gbs;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < ncell; t += (long)gridDim.x * blockDim.x) {
        long idx;
        if (!glist) {
            idx = t;
        } else if (t < nint) {
            idx = ((t / ((long)n * n) + g) * ne + (t / n) % n + g) * ne + t % n + g;
        } else {
            idx = glist[t - nint];
        }
        int i = (int)(idx % ne) - g, j = (int)((idx / ne) % ne) - g, k = (int)(idx / ((long)ne * ne)) - g;
        double u[NV_DEV];
        int ri = i < 0 ? -1 : i >= n ? 1 : 0, rj = j < 0 ? -1 : j >= n ? 1 : 0, rk = k < 0 ? -1 : k >= n ? 1 : 0;
        if (!(ri | rj | rk)) {
            const double *s = m.store + (long)b * m.bstride + ((long)k * n + j) * n + i;
#pragma unroll
            for (int v = 0; v < NV_DEV; v++) u[v] = s[v * m.vstride];
        } else {
            int x[3] = {B.c0 * n + i, B.c1 * n + j, B.c2 * n + k};
            if (!guard_value(m, b, x, u)) {
                atomicOr(m.err, ERR_AMR);
#pragma unroll
                for (int v = 0; v < NV_DEV; v++) u[v] = 0.;
            } else if ((mask >> ((rk + 1) * 9 + (rj + 1) * 3 + (ri + 1))) & 1u) {
                eos_cell_dev(u, prm, gam1inv, ggprodinv);
            }
        }
        if constexpr (TO_UNK) {
#pragma unroll
            for (int v = 0; v < NV_DEV; v++)
                if (dmap[v] >= 0) dst[idx * nunk + dmap[v]] = (T)u[v];   // < 0: not selected by a mask
        } else {
#pragma unroll
            for (int v = 0; v < NV_GCB; v++) dst[v * gvs + idx] = (T)u[v];
            if (gbs > NV_GCB * gvs) dst[DV_ENER * gvs + idx] = (T)u[DV_ENER];   // blocks with total energy
        }
    }
}

// ---- guard-fill plan ----------------------------------------------------------
// The mesh does not change between steps, so where every guard cell the
// pipeline reads comes from is resolved once: per leaf and guard-list entry a
// GuardPlan (same-level source, or a prolongation record), and per leaf the
// prolongation records in guard-list order.  The step's fill then copies the
// same-level cells in one light kernel and interpolates the prolonged ones
// in another, with the arithmetic of the direct path.
// one CTA per leaf; pass 0 writes the plan and counts the prolonged cells,
// pass 1 writes the prolongation records at poff[leaf] in guard-list order
__global__ void __launch_bounds__(256) amr_plan_kernel(MeshArgs m, const int *leaf_blk, const unsigned *eosmask,
                                                       const int *glist, int nglist, GuardPlan *plan, int *pcount,
                                                       ProlRec *prol, const int *poff, int pass)
{
    __shared__ int wsum[8];
    const int leaf = blockIdx.x;
    const int b = leaf_blk[leaf];
    const DevBlk B = m.blk[b];
    const unsigned mask = eosmask[leaf];
    const int n = m.n, g = m.ng, ne = n + 2 * g;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int base = pass ? poff[leaf] : 0;
    for (int g0 = 0; g0 < nglist; g0 += blockDim.x) {
        const int t = g0 + threadIdx.x;
        GuardSrc gs;
        gs.kind = GS_NONE;
        unsigned eos = 0, idx = 0;
        if (t < nglist) {
            idx = (unsigned)glist[t];
            int i, j, k;
            ext_coords(idx, ne, g, i, j, k);
            const int x[3] = {B.c0 * n + i, B.c1 * n + j, B.c2 * n + k};
            guard_resolve(m, b, x, gs);
            const int ri = i < 0 ? -1 : i >= n ? 1 : 0, rj = j < 0 ? -1 : j >= n ? 1 : 0,
                      rk = k < 0 ? -1 : k >= n ? 1 : 0;
            eos = (mask >> ((rk + 1) * 9 + (rj + 1) * 3 + (ri + 1))) & 1u;
            if (!pass) {
                GuardPlan gp;
                gp.off = gs.kind == GS_SAME ? (unsigned)gs.off[0] : 0u;
                gp.flags = gs.own | (eos << 3) | ((unsigned)gs.kind << 4);
                plan[(long)leaf * nglist + t] = gp;
            }
        }
        const bool pr = t < nglist && gs.kind == GS_PROL;
        const unsigned bal = __ballot_sync(0xffffffffu, pr);
        if (lane == 0) wsum[w] = __popc(bal);
        __syncthreads();
        int before = 0, total = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) { if (q < w) before += wsum[q]; total += wsum[q]; }
        if (pass && pr) {
            ProlRec r;
            r.idx = idx;
            r.flags = gs.parity | (gs.own << 3) | (eos << 6) | (gs.flips << 8);
#pragma unroll
            for (int s8 = 0; s8 < 8; s8++) r.off[s8] = (unsigned)gs.off[s8];
            r.pad[0] = r.pad[1] = 0;
            prol[base + before + __popc(bal & ((1u << lane) - 1u))] = r;
        }
        base += total;
        __syncthreads();
    }
    if (!pass && threadIdx.x == 0) pcount[leaf] = base;
}

template <class T>
__global__ void __launch_bounds__(256) amr_copy_kernel(MeshArgs m, const AmrEntry3 *entries, const int *leaf_blk,
                                                       const GuardPlan *plan, const int *glist, int nglist, T *out,
                                                       long gvs, long gbs, DevParams prm, double gam1inv,
                                                       double ggprodinv)
{
    amr_copy_kernel_body<T>(hw_block(), m, entries, leaf_blk, plan, glist, nglist, out, gvs, gbs, prm, gam1inv, ggprodinv);
}

// prolonged guard cells of a batch from the plan's records
template <class T>
__global__ void __launch_bounds__(256, FXB_FILL_MINB) amr_prolong_kernel(MeshArgs m, const AmrEntry3 *entries,
                                                                         const ProlRec *prol, const int *poff, T *out,
                                                                         long gvs, long gbs, DevParams prm,
                                                                         double gam1inv, double ggprodinv)
{
    amr_prolong_kernel_body<T>(hw_block(), m, entries, prol, poff, out, gvs, gbs, prm, gam1inv, ggprodinv);
}

// ---- refinement marking (Grid_markRefineDerefine) -------------------------------
// guard-filled copy of one variable of every active block (leaves and parents
// with a leaf child), all 4 guard layers, Eos on the guard regions of the
// block's Eos mask when need_eos (the variable is an Eos output)
__global__ void __launch_bounds__(256) amr_ext_fill_kernel(MeshArgs m, const int *active, const unsigned *act_eos,
                                                           int dv, int need_eos, double *ext, DevParams prm,
                                                           double gam1inv, double ggprodinv)
{
    const int sb = blockIdx.y;
    const int b = active[sb];
    const DevBlk B = m.blk[b];
    const unsigned mask = act_eos[sb];
    const int n = m.n, g = m.ng, ne = n + 2 * g;
    const int ncell = ne * ne * ne;
    double *E = ext + (long)sb * ncell;
    for (int idx = (int)(blockIdx.x * blockDim.x + threadIdx.x); idx < ncell; idx += (int)(gridDim.x * blockDim.x)) {
        int i, j, k;
        unflatten(idx, ne, ne, i, j, k);
        i -= g; j -= g; k -= g;
        const int ri = i < 0 ? -1 : i >= n ? 1 : 0, rj = j < 0 ? -1 : j >= n ? 1 : 0, rk = k < 0 ? -1 : k >= n ? 1 : 0;
        double u[NV_DEV];
        if (!(ri | rj | rk)) {
            const double *s = m.store + (long)b * m.bstride + ((long)k * n + j) * n + i;
#pragma unroll
            for (int v = 0; v < NV_DEV; v++) u[v] = s[v * m.vstride];
        } else {
            const int x[3] = {B.c0 * n + i, B.c1 * n + j, B.c2 * n + k};
            if (!guard_value(m, b, x, u)) {
                atomicOr(m.err, ERR_AMR);
#pragma unroll
                for (int v = 0; v < NV_DEV; v++) u[v] = 0.;
            } else if (need_eos && ((mask >> ((rk + 1) * 9 + (rj + 1) * 3 + (ri + 1))) & 1u)) {
                eos_cell_dev(u, prm, gam1inv, ggprodinv);
            }
        }
        double val = u[0];
#pragma unroll
        for (int v = 1; v < NV_DEV; v++) if (v == dv) val = u[v];
        E[idx] = val;
    }
}

// ---- regridding (Grid_updateRefinement's data movement) ------------------------
// blocks kept by a regrid: pairs (new block, old block), whole interiors
__global__ void amr_copy_blocks_kernel(const double *__restrict__ src, double *__restrict__ dst,
                                       const int2 *__restrict__ pairs, int np, long bstride)
{
    const long n = (long)np * bstride;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        const int p = (int)(idx / bstride);
        const long off = idx - (long)p * bstride;
        const int2 q = pairs[p];
        dst[(long)q.x * bstride + off] = src[(long)q.y * bstride + off];
    }
}

// new children of a regrid, all at one level: every interior cell
// interpolated from the parent level in conserved form (amr_prolong ->
// amr_1blk_cc_prol_gen_unk_fun with the convert hooks), reading the parent
// and its same-level neighbours, which hold their final data when the levels
// are processed coarse to fine
__global__ void __launch_bounds__(256) amr_newchild_kernel(MeshArgs m, const int *__restrict__ blocks, int nb)
{
    const int n = m.n;
    const long nc = (long)n * n * n;
    double *store = const_cast<double *>(m.store);
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)nb * nc;
         idx += (long)gridDim.x * blockDim.x) {
        const int b = blocks[idx / nc];
        const int c = (int)(idx % nc);
        const int i = c % n, j = (c / n) % n, k = c / (n * n);
        const DevBlk B = m.blk[b];
        const int x[3] = {B.c0 * n + i, B.c1 * n + j, B.c2 * n + k};
        GuardSrc gs;
        gs.parity = 0; gs.flips = 0; gs.own = 0;
        prol_resolve(m, B, x, gs);
        double u[NV_DEV];
        if (gs.kind == GS_PROL) {
            guard_eval_prol(m.store, m.vstride, gs.off, gs.flips, gs.parity, 0u, u);
        } else {
            atomicOr(m.err, ERR_AMR);
#pragma unroll
            for (int v = 0; v < NV_DEV; v++) u[v] = 0.;
        }
        double *o = store + (long)b * m.bstride + c;
#pragma unroll
        for (int v = 0; v < NV_DEV; v++) o[v * m.vstride] = u[v];
    }
}

// gr_estimateBlkError (GridMain/AMR/gr_estimateBlkError.F90, Cartesian) of
// every active block: the largest ratio of second differences to first
// differences plus filter times magnitudes over the cells grd = max(NGUARD-2, 2)
// layers in from the guard-cell edge (not past the interior at a non-periodic
// domain boundary); the first differences are recomputed per use with the
// same operations.  One CTA per block.  A cell with zero denominator and
// nonzero numerator makes the error HUGE, as the reference's assignment does
// whenever the other ratios are finite.
__global__ void __launch_bounds__(256) amr_error_kernel(const double *ext, const unsigned *act_bnd, const int *active,
                                                        const DevBlk *blk, const double *dxl, int n, int g,
                                                        double filter, double *err)
{
    __shared__ double smax[8];
    __shared__ int shuge[8];
    const int sb = blockIdx.x;
    const int ne = n + 2 * g;
    const double *E = ext + (long)sb * ne * ne * ne;
    const int lev = blk[active[sb]].level;
    const double del[3] = {0.5e0 / dxl[3 * (lev - 1)], 0.5e0 / dxl[3 * (lev - 1) + 1], 0.5e0 / dxl[3 * (lev - 1) + 2]};
    const unsigned bnd = act_bnd[sb];
    const int grd = g - 2 > 2 ? g - 2 : 2;
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        lo[a] = ((bnd >> a) & 1u) ? (grd > g ? grd : g) : grd;
        hi[a] = ((bnd >> (3 + a)) & 1u) ? (ne - 1 - grd < g + n - 1 ? ne - 1 - grd : g + n - 1) : ne - 1 - grd;
    }
    const int lx = hi[0] - lo[0] + 1, ly = hi[1] - lo[1] + 1, lz = hi[2] - lo[2] + 1;
    const int st[3] = {1, ne, ne * ne};
    double m = 0.;
    int huge = 0;
    for (int t = threadIdx.x; t < lx * ly * lz; t += blockDim.x) {
        const int i = lo[0] + t % lx, j = lo[1] + (t / lx) % ly, k = lo[2] + t / (lx * ly);
        const int p = (k * ne + j) * ne + i;
        // (1,x) (1,y) (2,x) (2,y) (1,z) (2,z) (3,x) (3,y) (3,z)
        const int comp[9] = {0, 0, 1, 1, 0, 1, 2, 2, 2}, axis[9] = {0, 1, 0, 1, 2, 2, 0, 1, 2};
        double num = 0., denom = 0.;
#pragma unroll
        for (int q = 0; q < 9; q++) {
            const int c = comp[q], ax = axis[q];
            const int pp = p + st[ax], pm = p - st[ax];
            const double dup = (E[pp + st[c]] - E[pp - st[c]]) * del[c];
            const double dum = (E[pm + st[c]] - E[pm - st[c]]) * del[c];
            const double duap = (fabs(E[pp + st[c]]) + fabs(E[pp - st[c]])) * del[c];
            const double duam = (fabs(E[pm + st[c]]) + fabs(E[pm - st[c]])) * del[c];
            const double d2 = (dup - dum) * del[ax];
            const double d3 = (fabs(dup) + fabs(dum)) * del[ax];
            const double d4 = (duap + duam) * del[ax];
            num = num + d2 * d2;
            const double s2 = d3 + (filter * d4);
            denom = denom + s2 * s2;
        }
        if (denom == 0.0 && num != 0.0) huge = 1;
        else if (denom != 0.0) m = fmax2(m, num / denom);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        m = fmax2(m, __shfl_xor_sync(0xffffffffu, m, off));
        huge |= __shfl_xor_sync(0xffffffffu, huge, off);
    }
    if ((threadIdx.x & 31) == 0) { smax[threadIdx.x >> 5] = m; shuge[threadIdx.x >> 5] = huge; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.;
        int h = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { r = fmax2(r, smax[w]); h |= shuge[w]; }
        if (h) r = fmax2(0x1.fffffffffffffp+1023, r);
        err[sb] = sqrt(r);
    }
}

// every cell of the parents of one level
__global__ void __launch_bounds__(256) amr_restrict_kernel(double *store, long vstride, long bstride, int n,
                                                           const int *plist, int np, const int *child)
{
    const long per = (long)n * n * n;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)np * per; idx += (long)gridDim.x * blockDim.x)
        restrict_cell(store, vstride, bstride, n, plist[idx / per], (int)(idx % per), child);
}

// the listed (parent, cell) pairs of one level
__global__ void __launch_bounds__(256) amr_restrict_list_kernel(double *store, long vstride, long bstride, int n,
                                                                const int2 *list, int cnt, const int *child)
{
    for (int t = (int)(blockIdx.x * blockDim.x + threadIdx.x); t < cnt; t += (int)(gridDim.x * blockDim.x)) {
        const int2 pc = list[t];
        restrict_cell(store, vstride, bstride, n, pc.x, pc.y, child);
    }
}

// parent-block cells the guard-fill plan reads (same-level copies and prolongation stencils)
// roles (nullptr: every leaf): only the plans of leaves with a nonzero role
__global__ void __launch_bounds__(256) amr_need_kernel(const GuardPlan *plan, long nplan, int nglist,
                                                       const ProlRec *prol, long nprol, const int *poff, int nleaf,
                                                       const unsigned char *roles, long vstride, long bstride,
                                                       unsigned char *need)
{
    const long stride = (long)gridDim.x * blockDim.x;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nplan; t += stride) {
        if (roles && !roles[t / nglist]) continue;
        const GuardPlan gp = plan[t];
        if (((gp.flags >> 4) & 3u) == GS_SAME) need[(gp.off / bstride) * vstride + gp.off % bstride] = 1;
    }
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nprol; t += stride) {
        if (roles) {
            // the leaf whose records hold t: poff[l] <= t < poff[l + 1]
            int lo = 0, hi = nleaf;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (poff[mid] <= t) lo = mid; else hi = mid;
            }
            if (!roles[lo]) continue;
        }
#pragma unroll
        for (int s8 = 0; s8 < 8; s8++) {
            const unsigned off = prol[t].off[s8];
            need[(off / bstride) * vstride + off % bstride] = 1;
        }
    }
}

// UNK staging (leaf, k, j, i, var with guard cells) <-> interior store / guard-filled blocks
__global__ void amr_unk_to_store_kernel(const double *unk, int l0, int nl, const int *leaf_blk, double *store,
                                        long vstride, long bstride, int n, int ng, int nunk, const int *dmap)
{
    const long per = (long)n * n * n;
    const int ne = n + 2 * ng;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)nl * per; idx += (long)gridDim.x * blockDim.x) {
        const int l = (int)(idx / per);
        const long c = idx % per;
        const int i = (int)(c % n), j = (int)((c / n) % n), k = (int)(c / ((long)n * n));
        const double *u = unk + ((((long)l * ne + k + ng) * ne + j + ng) * ne + i + ng) * nunk;
        double *s = store + (long)leaf_blk[l0 + l] * bstride + c;
        for (int v = 0; v < NV_DEV; v++) s[v * vstride] = u[dmap[v]];
    }
}

// Eos, CFL rate and volume integrals over the leaves' interiors
__global__ void amr_eos_kernel(double *store, long vstride, long bstride, int n, const int *leaf_blk, int nleaf,
                               DevParams prm, double gam1inv, double ggprodinv)
{
    const long per = (long)n * n * n;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)nleaf * per; idx += (long)gridDim.x * blockDim.x) {
        double *s = store + (long)leaf_blk[idx / per] * bstride + idx % per;
        double u[NV_DEV];
        for (int v = 0; v < NV_DEV; v++) u[v] = s[v * vstride];
        eos_cell_dev(u, prm, gam1inv, ggprodinv);
        for (int v = 0; v < NV_DEV; v++) s[v * vstride] = u[v];
    }
}

__global__ void amr_rate_kernel(const double *store, long vstride, long bstride, int n, const int *leaf_blk,
                                const DevBlk *blk, const double *dxl, int nleaf, unsigned long long *rate_max,
                                const unsigned char *role)
{
    const long per = (long)n * n * n;
    double r = 0.;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)nleaf * per; idx += (long)gridDim.x * blockDim.x) {
        if (role && role[idx / per] != 1) continue;     // a split mesh: the rank's own leaves
        const int b = leaf_blk[idx / per];
        const double *s = store + (long)b * bstride + idx % per;
        const double *dl = dxl + 3 * (blk[b].level - 1);
        double cs = sqrt(s[GC * vstride] * s[P * vstride] / s[D * vstride]);
        double t = (fabs(s[VX * vstride] - 0.) + cs) * (1.0 / dl[0]);
        t = fmax2(t, (fabs(s[VY * vstride] - 0.) + cs) * (1.0 / dl[1]));
        t = fmax2(t, (fabs(s[VZ * vstride] - 0.) + cs) * (1.0 / dl[2]));
        r = fmax2(r, t);
    }
    for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, off));
    if ((threadIdx.x & 31) == 0) atomicMax(rate_max, (unsigned long long)__double_as_longlong(r));
}

// limiting cell of the leaves: first (leaf, k, j, i) whose rate equals the maximum
__global__ void amr_locate_kernel(const double *store, long vstride, long bstride, int n, const int *leaf_blk,
                                  const DevBlk *blk, const double *dxl, int nleaf, const unsigned long long *rate_max,
                                  unsigned long long *key, const unsigned char *role)
{
    const long per = (long)n * n * n;
    const unsigned long long rm = *rate_max;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)nleaf * per; idx += (long)gridDim.x * blockDim.x) {
        if (role && role[idx / per] != 1) continue;
        const int b = leaf_blk[idx / per];
        const double *s = store + (long)b * bstride + idx % per;
        const double *dl = dxl + 3 * (blk[b].level - 1);
        double cs = sqrt(s[GC * vstride] * s[P * vstride] / s[D * vstride]);
        double t = (fabs(s[VX * vstride] - 0.) + cs) * (1.0 / dl[0]);
        t = fmax2(t, (fabs(s[VY * vstride] - 0.) + cs) * (1.0 / dl[1]));
        t = fmax2(t, (fabs(s[VZ * vstride] - 0.) + cs) * (1.0 / dl[2]));
        if ((unsigned long long)__double_as_longlong(t) == rm) atomicMin(key, (unsigned long long)idx);
    }
}

// one exchange message: y = listed leaf, x = chunk of its interior; the
// message holds one interior per leaf (mstride = bstride), or one for all
// (mstride = 0, unpack only)
__global__ void __launch_bounds__(256) amr_leaf_copy_kernel(double *store, long bstride, const int *leaf_blk,
                                                            const int *list, double *msg, long mstride, int pack)
{
    const int q = blockIdx.y;
    double2 *blk = reinterpret_cast<double2 *>(store + (long)leaf_blk[list[q]] * bstride);
    double2 *m = reinterpret_cast<double2 *>(msg + (long)q * mstride);
    const long n2 = bstride / 2;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += (long)gridDim.x * blockDim.x) {
        if (pack) m[i] = __ldcg(blk + i);
        else blk[i] = __ldcg(m + i);
    }
}

__global__ void amr_integrals_kernel(const double *store, long vstride, long bstride, int n, const int *leaf_blk,
                                     const DevBlk *blk, const double *dxl, int nleaf, double *partials,
                                     const unsigned char *role)
{
    const long per = (long)n * n * n;
    double s[7] = {0., 0., 0., 0., 0., 0., 0.};
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)nleaf * per; idx += (long)gridDim.x * blockDim.x) {
        if (role && role[idx / per] != 1) continue;
        const int b = leaf_blk[idx / per];
        const double *c = store + (long)b * bstride + idx % per;
        const double *dl = dxl + 3 * (blk[b].level - 1);
        const double dv = dl[0] * dl[1] * dl[2];
        double rho = c[D * vstride], vx = c[VX * vstride], vy = c[VY * vstride], vz = c[VZ * vstride];
        s[0] += rho * dv; s[1] += rho * vx * dv; s[2] += rho * vy * dv; s[3] += rho * vz * dv;
        s[4] += rho * c[DV_ENER * vstride] * dv; s[5] += rho * c[EI * vstride] * dv;
        s[6] += 0.5 * rho * (vx * vx + vy * vy + vz * vz) * dv;
    }
    __shared__ double sh[7][256];
    for (int q = 0; q < 7; q++) sh[q][threadIdx.x] = s[q];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 7; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 7; q++) partials[blockIdx.x * 7 + q] = sh[q][0];
}

__global__ void amr_integrals_final_kernel(const double *partials, int np, double *out)
{
    if (threadIdx.x < 7) {
        double t = 0.;
        for (int b = 0; b < np; b++) t += partials[b * 7 + threadIdx.x];
        out[threadIdx.x] = t;
    }
}

// ------------------------------------------------------------------ host
#define CKA(call)                                                                          \
    do {                                                                                   \
        cudaError_t _e = (call);                                                           \
        if (_e != cudaSuccess) {                                                           \
            char _b[256];                                                                  \
            snprintf(_b, sizeof(_b), "%s: %s", #call, cudaGetErrorString(_e));             \
            return record_error(FXB_ECUDA, _b);                                            \
        }                                                                                  \
    } while (0)

template <class T> void dfree(T *&p)
{
    if (p) cudaFree((void *)p);
    p = nullptr;
}

MeshArgs mesh_args(int which)
{
    MeshArgs m;
    m.blk = S.d_blk; m.ntab = S.d_ntab; m.store = S.store[which];
    m.vstride = S.vstride; m.bstride = S.bstride; m.n = S.n; m.ng = S.ng;
    m.nb1[0] = S.C.dom.nblockx; m.nb1[1] = S.C.dom.nblocky; m.nb1[2] = S.C.dom.nblockz;
    for (int i = 0; i < 6; i++) m.bc[i] = S.C.dom.bc[i];
    m.err = S.C.err;
    return m;
}

size_t rsize() { return S.C.prm.precision == FXB_MIXED ? sizeof(float) : sizeof(double); }
long ne3() { long e = S.n + 2 * S.ng; return e * e * e; }

Args3D batch_args(const double *dtv, double dt)
{
    Args3D a;
    memset((void *)&a, 0, sizeof(a));
    a.rate_c0 = 0;
    a.rate_c1 = 0x7fffffffffffffffL;     // every leaf cell enters the CFL rate
    a.nx = a.ny = a.nz = S.n;
    for (int i = 0; i < 6; i++) a.bc[i] = S.C.dom.bc[i];
    a.dt_arg = dt; a.dtv = dtv;
    a.gam1inv = S.C.gam1inv; a.ggprodinv = S.C.ggprodinv;
    a.prm = S.C.dprm; a.rate_max = S.C.rate_max; a.err = S.C.err;
    a.sig = S.sig;
    a.slp = S.slp;
    a.flat = S.flat;
    for (int d = 0; d < 3; d++) { a.wst[d] = S.w[d]; a.flx[d] = S.f[d]; }
    a.gcb = S.gcb; a.gcb_vstride = ne3(); a.gcb_bstride = ne3() * S.ngcb; a.ng = S.ng;
    a.istore = S.store[S.cur];
    a.dxl = S.d_dxl;
    for (int q = 0; q < 4; q++) a.cta[q] = S.cta[q];
    a.odata = S.store[1 - S.cur]; a.o_vstride = S.vstride; a.o_bstride = S.bstride;
    const size_t r = rsize();
    a.sig_bstride = (long)(sig3d_bytes(S.n, S.n, S.n, r) / r);
    a.slp_bstride = (long)(slp3d_bytes(S.n, S.n, S.n, r) / r);
    a.flat_bstride = 3L * (S.n + 2) * (S.n + 2) * (S.n + 2);
    for (int d = 0; d < 3; d++) {
        a.w_bstride[d] = (long)(w3d_bytes(d, S.n, S.n, S.n, r) / r);
        a.f_bstride[d] = (long)(f3d_bytes(d, S.n, S.n, S.n, r) / r);
    }
    if (S.hyb) {
        const long nd = (long)(S.n + 6) * (S.n + 6) * (S.n + 6);
        a.divu = S.hyb;
        a.divu_bstride = nd;
        a.hyb = (const unsigned char *)S.hyb + r * nd * S.batch;
        a.hyb_bstride = (long)(S.n + 2) * (S.n + 2) * (S.n + 2);
    }
    return a;
}

void restrict_all(int which)
{
    for (int lev = S.maxlev - 1; lev >= 1; lev--) {
        int np = (int)S.parents_at[lev].size();
        if (!np) continue;
        long work = (long)np * S.n * S.n * S.n;
        int grid = (int)std::min<long>((work + 255) / 256, 148L * 16);
        amr_restrict_kernel<<<grid, 256, 0, S.C.stream>>>(S.store[which], S.vstride, S.bstride, S.n,
                                                          S.d_plist + S.plist_off[lev], np, S.d_child);
    }
}

template <class T> void fill_planned(const AmrEntry3 *entries, int cnt, int which)
{
    const dim3 g(S.fill_cta, cnt);
    amr_copy_kernel<T><<<g, 256, 0, S.C.stream>>>(mesh_args(which), entries, S.leaf_blk_dev, (const GuardPlan *)S.d_plan,
                                                  S.d_glist, S.nglist, (T *)S.gcb, ne3(), ne3() * S.ngcb, S.C.dprm,
                                                  S.C.gam1inv, S.C.ggprodinv);
    if (S.nprol)
        amr_prolong_kernel<T><<<g, 256, 0, S.C.stream>>>(mesh_args(which), entries, (const ProlRec *)S.d_prol, S.d_poff,
                                                         (T *)S.gcb, ne3(), ne3() * S.ngcb, S.C.dprm, S.C.gam1inv,
                                                         S.C.ggprodinv);
}

// restriction of only the parent cells the guard-fill plan reads (every cell
// without a plan); returns the number of launches
int restrict_needed(int which)
{
    if (!S.d_rlist) { restrict_all(which); return S.maxlev - 1; }
    int nl = 0;
    for (int lev = S.maxlev - 1; lev >= 1; lev--) {
        const long cnt = S.rlist_off[lev + 1] - S.rlist_off[lev];
        if (!cnt) continue;
        nl++;
        int grid = (int)std::min<long>((cnt + 255) / 256, 148L * 16);
        amr_restrict_list_kernel<<<grid, 256, 0, S.C.stream>>>(S.store[which], S.vstride, S.bstride, S.n,
                                                               S.d_rlist + S.rlist_off[lev], (int)cnt, S.d_child);
    }
    return nl;
}

// guard fill of one batch; returns the number of launches
int fill_batch(const AmrEntry3 *entries, int cnt, int which)
{
    const dim3 g(S.fill_cta, cnt);
    if (S.d_plan) {
        if (S.C.prm.precision == FXB_MIXED) fill_planned<float>(entries, cnt, which);
        else fill_planned<double>(entries, cnt, which);
        return S.nprol ? 2 : 1;
    }
    if (S.C.prm.precision == FXB_MIXED)
        amr_fill_kernel<float, false><<<g, 256, 0, S.C.stream>>>(mesh_args(which), entries, S.leaf_blk_dev, S.d_eosmask,
                                                                (float *)S.gcb, ne3(), ne3() * S.ngcb, 0, nullptr,
                                                                S.d_glist, S.nglist, S.C.dprm, S.C.gam1inv,
                                                                S.C.ggprodinv);
    else
        amr_fill_kernel<double, false><<<g, 256, 0, S.C.stream>>>(mesh_args(which), entries, S.leaf_blk_dev, S.d_eosmask,
                                                                 (double *)S.gcb, ne3(), ne3() * S.ngcb, 0, nullptr,
                                                                 S.d_glist, S.nglist, S.C.dprm, S.C.gam1inv,
                                                                 S.C.ggprodinv);
    return 1;
}

template <class T> cudaError_t upload(T *&dst, const std::vector<T> &v)
{
    cudaError_t e = cudaMalloc((void **)&dst, sizeof(T) * std::max<size_t>(1, v.size()));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync((void *)dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, S.C.stream);
}

int persist_upload();

// parent cells the guard-fill plans of the stepped leaves read (every leaf,
// or with roles set the active ones), and below them the parent cells their
// restriction reads (coarse to fine); listed per level for the step
static cudaError_t build_rlist()
{
#define CKR(call) do { cudaError_t _e = (call); if (_e != cudaSuccess) return _e; } while (0)
    cudaStream_t st = S.C.stream;
    const size_t ncb = (size_t)S.nblk * S.vstride;
    unsigned char *d_need = nullptr;
    CKR(cudaMalloc(&d_need, ncb));
    CKR(cudaMemsetAsync(d_need, 0, ncb, st));
    const long nplan = (long)S.nleaf * S.nglist;
    const int grid = (int)std::min<long>((std::max(nplan, S.nprol) + 255) / 256, 148L * 16);
    amr_need_kernel<<<grid, 256, 0, st>>>((const GuardPlan *)S.d_plan, nplan, S.nglist, (const ProlRec *)S.d_prol,
                                           S.nprol, S.d_poff, S.nleaf, S.roles.empty() ? nullptr : S.d_roles,
                                           S.vstride, S.bstride, d_need);
    CKR(cudaGetLastError());
    std::vector<unsigned char> need(ncb);
    CKR(cudaMemcpyAsync(need.data(), d_need, ncb, cudaMemcpyDeviceToHost, st));
    CKR(cudaStreamSynchronize(st));
    cudaFree(d_need);
    const int n = S.n, h = n / 2;
    for (int lev = 1; lev < S.maxlev; lev++)
        for (int p : S.parents_at[lev])
            for (int cidx = 0; cidx < S.vstride; cidx++) {
                if (!need[(size_t)p * S.vstride + cidx]) continue;
                const int pi = cidx % n, pj = (cidx / n) % n, pk = cidx / (n * n);
                const int q = (pi >= h) | ((pj >= h) << 1) | ((pk >= h) << 2);
                const int ch = S.blk[p].child[q];
                if (S.blk[ch].leaf >= 0) continue;
                const int i0 = 2 * (pi - (q & 1) * h), j0 = 2 * (pj - ((q >> 1) & 1) * h),
                          k0 = 2 * (pk - ((q >> 2) & 1) * h);
                for (int kk = 0; kk < 2; kk++) for (int jj = 0; jj < 2; jj++) for (int ii = 0; ii < 2; ii++)
                    need[(size_t)ch * S.vstride + ((k0 + kk) * n + (j0 + jj)) * n + (i0 + ii)] = 1;
            }
    std::vector<int2> rl;
    S.rlist_off.assign(S.maxlev + 1, 0);
    for (int lev = 1; lev <= S.maxlev; lev++) {
        S.rlist_off[lev] = (long)rl.size();
        if (lev == S.maxlev) break;
        for (int p : S.parents_at[lev])
            for (int cidx = 0; cidx < S.vstride; cidx++)
                if (need[(size_t)p * S.vstride + cidx]) rl.push_back(make_int2(p, cidx));
    }
    dfree(S.d_rlist);
    return upload(S.d_rlist, rl);
#undef CKR
}

// the step's entry lists and queue over the active leaves (all leaves, or a
// rank's roles): [one batch][first pass of several batches][corrected leaves],
// the flags of d_entries, and role 2 never updated
int set_step_entries()
{
    const bool split = !S.roles.empty();
    auto role = [&](int l) { return split ? (int)S.roles[l] : 1; };
    std::vector<AmrEntry3> ent, per(S.nleaf);
    std::vector<int> act;
    for (int l = 0; l < S.nleaf; l++)
        if (role(l)) act.push_back(l);
    for (int pass = 0; pass < 2; pass++)
        for (int l : act) {
            const bool fin = S.finer_h[l] != 0;
            const bool skip = role(l) == 2 || (pass == 1 && fin);
            ent.push_back(AmrEntry3{S.leaf_blk[l], S.blk[S.leaf_blk[l]].level, l, skip ? (int)AMR_SKIP_UPDATE : 0});
        }
    int nfin = 0;
    for (int l : act)
        if (role(l) == 1 && S.finer_h[l]) { ent.push_back(AmrEntry3{S.leaf_blk[l], S.blk[S.leaf_blk[l]].level, l, 0}); nfin++; }
    for (int l = 0; l < S.nleaf; l++)
        per[l] = AmrEntry3{S.leaf_blk[l], S.blk[S.leaf_blk[l]].level, l, role(l) == 2 ? (int)AMR_SKIP_UPDATE : 0};
    dfree(S.d_step_entries);
    dfree(S.d_leaf_entry);
    CKA(upload(S.d_step_entries, ent));
    CKA(upload(S.d_leaf_entry, per));
    S.nstep = (int)act.size();
    S.nstep_finer = nfin;
    if (S.persist_ok) {
        // the persistent queue: the active leaves, finest level first
        std::vector<int> order(act);
        std::stable_sort(order.begin(), order.end(), [](int x, int y) {
            return S.blk[S.leaf_blk[x]].level > S.blk[S.leaf_blk[y]].level;
        });
        dfree(S.d_order);
        CKA(upload(S.d_order, order));
        return persist_upload();
    }
    return FXB_OK;
}

// The persistent step: on by default when the mesh has a guard-fill plan and
// no option that needs the extended-option kernels (FXB_AMR_PERSISTENT=0
// keeps the batched launches).  Queue order, restriction items (chunks of
// the needed parent cells, deepest level first) and one scratch slot per
// resident CTA of the kernel.
// clusters of K CTAs of the persistent kernel to launch: those that fit at
// once, at most one per scratch slot of the batch arrays
int persist_clusters(int K)
{
    const int n = S.C.prm.precision == FXB_MIXED ? persist_grid_mixed(K) : persist_grid_fp64(K);
    return std::min(n, S.batch);
}


int persist_setup()
{
    const char *ev = getenv("FXB_AMR_PERSISTENT");
    S.persist_ok = !(ev && ev[0] == '0') && S.d_plan && !extended_options(S.C.dprm);
    // the batched launches until the tuner times both forms (FXB_AMR_PERSISTENT=1 forces this one)
    S.persist = S.persist_ok && ev && ev[0] == '1';
    if (!S.persist_ok) return FXB_OK;
    const char *tw = getenv("FXB_TEST_WAIT_TIMEOUT");
    if (tw && tw[0] == '1') { S.test_stall = 1; S.wait_budget = 1000000; }
    const char *ek = getenv("FXB_AMR_CLUSTER");
    if (ek) S.pK = atoi(ek);
    if (S.pK != 1 && S.pK != 2 && S.pK != 4 && S.pK != 8) S.pK = 4;
    const int most = persist_clusters(1);
    if (most <= 0) return record_error(FXB_ECUDA, "fxb_register_blocks: persistent AMR kernel does not fit on an SM");
    S.pslots = most;
    S.pclusters = persist_clusters(S.pK);
    std::vector<int> order(S.nleaf);
    for (int l = 0; l < S.nleaf; l++) order[l] = l;
    std::stable_sort(order.begin(), order.end(), [](int x, int y) {
        return S.blk[S.leaf_blk[x]].level > S.blk[S.leaf_blk[y]].level;
    });
    CKA(upload(S.d_order, order));
    std::vector<int4> items;
    const long rch = 2048;
    for (int i = 0; i < 32; i++) S.rlev_items[i] = 0;
    if (S.d_rlist)
        for (int lev = S.maxlev - 1; lev >= 1; lev--) {
            const long off = S.rlist_off[lev], cnt = S.rlist_off[lev + 1] - off;
            for (long b = 0; b < cnt; b += rch) {
                items.push_back(make_int4(lev, (int)(off + b), (int)(off + std::min(b + rch, cnt)), 0));
                S.rlev_items[lev]++;
            }
        }
    S.nritem = (int)items.size();
    if (S.nritem) CKA(upload(S.d_ritems, items));
    CKA(cudaMalloc(&S.d_ctl, sizeof(int) * PQ_WORDS));
    CKA(cudaMalloc(&S.d_emitted, sizeof(int) * (size_t)S.nleaf));
    CKA(cudaMalloc(&S.d_slots, sizeof(AmrEntry3) * (size_t)S.pslots));
    return FXB_OK;    // the argument sets are uploaded with the step's entry lists
}

// the kernel's argument sets for current store 0 and 1 (dt read from the
// library's device dt, AmrCommon::dtv)
int persist_upload()
{
    PersistArgs p[2];
    for (int w = 0; w < 2; w++) {
        memset((void *)&p[w], 0, sizeof(PersistArgs));
        const int keep = S.cur;
        S.cur = w;
        p[w].a = batch_args(S.C.dtv, 0.0);
        p[w].m = mesh_args(w);
        S.cur = keep;
        p[w].a.batch = S.d_slots;
        p[w].slots = S.d_slots;
        p[w].leaf_entry = S.d_leaf_entry;
        p[w].order = S.d_order;
        p[w].leaf_blk = S.leaf_blk_dev;
        p[w].plan = (const GuardPlan *)S.d_plan;
        p[w].glist = S.d_glist;
        p[w].nglist = S.nglist;
        p[w].prol = (const ProlRec *)S.d_prol;
        p[w].poff = S.d_poff;
        p[w].has_prol = S.nprol > 0;
        p[w].ritems = S.d_ritems;
        p[w].rlist = S.d_rlist;
        p[w].child = S.d_child;
        p[w].nritem = S.nritem;
        p[w].nleaf = S.nstep;
        for (int i = 0; i < 32; i++) p[w].rlev_items[i] = S.rlev_items[i];
        p[w].bflux = S.bflux;
        p[w].nfc = S.nfc;
        p[w].fine = S.d_fine;
        p[w].finer_mask = S.d_finer;
        p[w].ctl = S.d_ctl;
        p[w].emitted = S.d_emitted;
        p[w].budget = S.wait_budget;
        p[w].test_stall = S.test_stall;
    }
    CKA(S.C.prm.precision == FXB_MIXED ? persist_upload_mixed(p) : persist_upload_fp64(p));
    return FXB_OK;
}

// one step as the persistent kernel; dt from dtv (a device pointer, the
// library's dt in graph-captured loops) or from the argument
int persist_step(const double *dtv, double dt)
{
    const bool mixed = S.C.prm.precision == FXB_MIXED;
    if (!dtv) CKA(cudaMemcpyAsync(S.C.dtv, &dt, sizeof(double), cudaMemcpyHostToDevice, S.C.stream));
    else if (dtv != S.C.dtv) return record_error(FXB_EARG, "persistent AMR step: dt must be the library's device dt");
    CKA(cudaMemsetAsync(S.d_ctl, 0, sizeof(int) * PQ_WORDS, S.C.stream));
    CKA(cudaMemsetAsync(S.d_emitted, 0, sizeof(int) * (size_t)S.nleaf, S.C.stream));
    if (S.pclusters <= 0) return record_error(FXB_ECUDA, "persistent AMR kernel: no cluster fits");
    CKA(mixed ? launch_amr_persist_mixed(S.cur, S.pclusters, S.pK, S.C.stream)
              : launch_amr_persist_fp64(S.cur, S.pclusters, S.pK, S.C.stream));
    CKA(cudaGetLastError());
    return FXB_OK;
}

} // namespace

// ----------------------------------------------------------------- interface
bool amr_active() { return S.active; }
int amr_cur() { return S.cur; }
long amr_leaf_cells() { return (long)S.nleaf * S.n * S.n * S.n; }

namespace {
void free_device(State &s)
{
    dfree(s.store[0]); dfree(s.store[1]);
    dfree(s.d_blk); dfree(s.d_ntab); dfree(s.d_child); dfree(s.d_plist); dfree(s.d_eosmask);
    dfree(s.d_finer); dfree(s.d_fine); dfree(s.d_dxl); dfree(s.d_entries); dfree(s.leaf_blk_dev);
    dfree(s.gcb); dfree(s.sig); dfree(s.slp); dfree(s.flat); dfree(s.hyb);
    for (int d = 0; d < 3; d++) { dfree(s.w[d]); dfree(s.f[d]); }
    dfree(s.bflux); dfree(s.stage); dfree(s.d_dmap); dfree(s.d_pmap); dfree(s.d_glist);
    dfree(s.d_plan); dfree(s.d_prol); dfree(s.d_poff); dfree(s.d_rlist);
    dfree(s.d_order); dfree(s.d_ctl); dfree(s.d_emitted); dfree(s.d_ritems); dfree(s.d_slots);
    dfree(s.d_roles); dfree(s.d_step_entries); dfree(s.d_leaf_entry); dfree(s.d_xlist);
    dfree(s.d_own_blk); dfree(s.d_own_entries);
    dfree(s.d_active); dfree(s.d_act_eos); dfree(s.d_act_bnd); dfree(s.d_ext); dfree(s.d_err);
}
} // namespace

void amr_destroy()
{
    free_device(S);
    S = State();
}

int amr_create(const AmrCommon &c, const fxb_block_desc *leaves, int nleaf)
{
    amr_destroy();
    S.C = c;
    const fxb_domain &D = c.dom;
    if (D.ndim != 3) return record_error(FXB_EUNSUPPORTED, "fxb_register_blocks: AMR meshes are implemented for 3-D");
    if (D.nxb != D.nyb || D.nxb != D.nzb || D.nxb % 2 || D.nxb < D.nguard)
        return record_error(FXB_EUNSUPPORTED, "fxb_register_blocks: AMR blocks must be cubes of an even size >= NGUARD");
    if (c.dprm.shock_detect)
        return record_error(FXB_EUNSUPPORTED, "fxb_register_blocks: the shock detector is implemented for uniform grids");
    S.n = D.nxb;
    S.ng = D.nguard;
    S.nleaf = nleaf;
    // artificial viscosity reads the total energy of the guard-filled blocks
    // (the variable after EINT in the device order)
    S.ngcb = c.prm.use_avisc ? DV_ENER + 1 : NV_GCB;
    std::vector<int> finer, fine;
    int rc = build_tree(leaves, nleaf, finer, fine);
    if (rc) { S = State(); return rc; }
    S.parents_at.assign(S.maxlev + 1, {});
    for (int b = 0; b < S.nblk; b++)
        if (S.blk[b].leaf < 0) S.parents_at[S.blk[b].level].push_back(b);
    std::vector<int> plist;
    S.plist_off.assign(S.maxlev + 1, 0);
    for (int lev = 1; lev <= S.maxlev; lev++) {
        S.plist_off[lev] = (long)plist.size();
        plist.insert(plist.end(), S.parents_at[lev].begin(), S.parents_at[lev].end());
    }
    std::vector<DevBlk> hb(S.nblk);
    std::vector<int> ntab((size_t)S.nblk * 27), child((size_t)S.nblk * 8);
    for (int b = 0; b < S.nblk; b++) {
        const HBlock &B = S.blk[b];
        hb[b] = DevBlk{B.level, B.c[0], B.c[1], B.c[2], B.parent};
        for (int k = -1; k <= 1; k++) for (int j = -1; j <= 1; j++) for (int i = -1; i <= 1; i++)
            ntab[(size_t)b * 27 + (k + 1) * 9 + (j + 1) * 3 + (i + 1)] = (i | j | k) ? neigh(b, i, j, k) : b;
        for (int q = 0; q < 8; q++) child[(size_t)b * 8 + q] = B.child[q];
    }
    std::vector<unsigned> eos(nleaf);
    for (int l = 0; l < nleaf; l++) eos[l] = eos_regions(S.leaf_blk[l]);
    std::vector<double> dxl(3 * (size_t)S.maxlev);
    double d0[3];
    for (int a = 0; a < 3; a++) {
        int nb = a == 0 ? D.nblockx : a == 1 ? D.nblocky : D.nblockz;
        int nn = a == 0 ? D.nxb : a == 1 ? D.nyb : D.nzb;
        d0[a] = (D.bbox[a][1] - D.bbox[a][0]) / (1.0 * nn * nb);   // gr_initSpecific.F90:172-178
    }
    for (int lev = 1; lev <= S.maxlev; lev++)
        for (int a = 0; a < 3; a++) {
            dxl[3 * (lev - 1) + a] = d0[a];
            d0[a] = d0[a] / 2.0;
        }
    std::vector<AmrEntry3> ent;
    ent.reserve(2 * (size_t)nleaf + 64);
    for (int pass = 0; pass < 2; pass++)
        for (int l = 0; l < nleaf; l++)
            ent.push_back(AmrEntry3{S.leaf_blk[l], S.blk[S.leaf_blk[l]].level, l,
                                    (pass == 1 && finer[l]) ? (int)AMR_SKIP_UPDATE : 0});
    for (int l = 0; l < nleaf; l++)
        if (finer[l]) ent.push_back(AmrEntry3{S.leaf_blk[l], S.blk[S.leaf_blk[l]].level, l, 0});
    S.nfiner = (int)ent.size() - 2 * nleaf;

    cudaStream_t st = c.stream;
    S.vstride = (long)S.n * S.n * S.n;
    S.bstride = S.vstride * NV_DEV;
    auto up = [&](auto *&dst, const auto &v) -> cudaError_t {
        using T = typename std::remove_const<typename std::remove_reference<decltype(v[0])>::type>::type;
        cudaError_t e = cudaMalloc((void **)&dst, sizeof(T) * std::max<size_t>(1, v.size()));
        if (e != cudaSuccess) return e;
        if (v.empty()) return cudaSuccess;
        return cudaMemcpyAsync((void *)dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
    };
    for (int i = 0; i < 2; i++) {
        CKA(cudaMalloc(&S.store[i], sizeof(double) * S.bstride * S.nblk));
        CKA(cudaMemsetAsync(S.store[i], 0, sizeof(double) * S.bstride * S.nblk, st));
    }
    CKA(up(S.d_blk, hb));
    CKA(up(S.d_ntab, ntab));
    CKA(up(S.d_child, child));
    CKA(up(S.d_plist, plist));
    CKA(up(S.d_eosmask, eos));
    CKA(up(S.d_finer, finer));
    S.finer_h = finer;
    CKA(up(S.d_fine, fine));
    CKA(up(S.d_dxl, dxl));
    CKA(up(S.d_entries, ent));
    CKA(up(S.leaf_blk_dev, S.leaf_blk));
    std::vector<int> dm(c.dmap, c.dmap + NV_DEV);
    CKA(up(S.d_dmap, dm));
    // guard cells the 3-D pipeline reads: the padded box [-1, n]^3, and
    // outside it cells with one coordinate out: layers -2 and n+1 with the
    // others in [-1, n] (sigma), layers -3 and n+2 with the others interior
    // (PPM slopes, WENO stencils); with flattening (pressures three cells
    // either side of the padded box) every layer with the others in [-1, n]
    {
        std::vector<int> gl;
        const int n = S.n, g = S.ng, ne = n + 2 * g;
        auto in_box = [&](int x) { return x >= -1 && x <= n; };
        auto in_int = [&](int x) { return x >= 0 && x < n; };
        for (int k = -g; k < n + g; k++) for (int j = -g; j < n + g; j++) for (int i = -g; i < n + g; i++) {
            if (in_int(i) && in_int(j) && in_int(k)) continue;           // interior: copied separately
            int x[3] = {i, j, k}, outside = 0, ax = -1;
            for (int a = 0; a < 3; a++) if (!in_box(x[a])) { outside++; ax = a; }
            bool need = false;
            if (outside == 0) need = true;
            else if (outside == 1) {
                int o1 = x[(ax + 1) % 3], o2 = x[(ax + 2) % 3];
                bool depth1 = x[ax] == -2 || x[ax] == n + 1;
                bool depth2 = x[ax] == -3 || x[ax] == n + 2;
                if (c.prm.flattening || depth1) need = in_box(o1) && in_box(o2);
                else if (depth2) need = in_int(o1) && in_int(o2);
            }
            if (c.prm.hybrid_order) need = true;     // DivU reads four cells out, edges and corners too
            if (need) gl.push_back(((k + g) * ne + (j + g)) * ne + (i + g));
        }
        S.nglist = (int)gl.size();
        CKA(up(S.d_glist, gl));
    }
    // guard-fill plan, when every store offset fits 32 bits
    if ((unsigned long long)S.bstride * S.nblk < (1ull << 32) && S.nglist > 0) {
        int *d_cnt = nullptr;
        CKA(cudaMalloc(&S.d_plan, sizeof(GuardPlan) * (size_t)nleaf * S.nglist));
        CKA(cudaMalloc(&d_cnt, sizeof(int) * (size_t)nleaf));
        amr_plan_kernel<<<nleaf, 256, 0, st>>>(mesh_args(0), S.leaf_blk_dev, S.d_eosmask, S.d_glist, S.nglist,
                                               (GuardPlan *)S.d_plan, d_cnt, nullptr, nullptr, 0);
        CKA(cudaGetLastError());
        std::vector<int> cnt(nleaf), poff(nleaf + 1, 0);
        CKA(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * (size_t)nleaf, cudaMemcpyDeviceToHost, st));
        CKA(cudaStreamSynchronize(st));
        cudaFree(d_cnt);
        for (int l = 0; l < nleaf; l++) poff[l + 1] = poff[l] + cnt[l];
        S.nprol = poff[nleaf];
        CKA(up(S.d_poff, poff));
        CKA(cudaMalloc(&S.d_prol, sizeof(ProlRec) * std::max<size_t>(1, (size_t)S.nprol)));
        if (S.nprol)
            amr_plan_kernel<<<nleaf, 256, 0, st>>>(mesh_args(0), S.leaf_blk_dev, S.d_eosmask, S.d_glist, S.nglist,
                                                   nullptr, nullptr, (ProlRec *)S.d_prol, S.d_poff, 1);
        CKA(cudaGetLastError());
        CKA(build_rlist());
    }
    // active blocks for refinement marking: Eos masks and non-periodic domain faces
    {
        std::vector<unsigned> aeos, abnd;
        for (int b = 0; b < S.nblk; b++) {
            const HBlock &B = S.blk[b];
            if (B.nodetype != 1 && B.nodetype != 2) continue;
            S.act_blk.push_back(b);
            aeos.push_back(eos_regions(b));
            unsigned bits = 0;
            for (int a = 0; a < 3; a++) {
                if (B.c[a] == 0 && D.bc[2 * a] != FXB_BC_PERIODIC) bits |= 1u << a;
                if (B.c[a] == nb_at(B.level, a) - 1 && D.bc[2 * a + 1] != FXB_BC_PERIODIC) bits |= 1u << (3 + a);
            }
            abnd.push_back(bits);
        }
        CKA(up(S.d_active, S.act_blk));
        CKA(up(S.d_act_eos, aeos));
        CKA(up(S.d_act_bnd, abnd));
    }
    const size_t r = rsize();
    S.nfc = (long)S.n * S.n;
    CKA(cudaMalloc(&S.bflux, r * 6 * NF * S.nfc * (size_t)nleaf));
    // UNK staging for attach/sync: chunks of up to 1 GiB
    const size_t per_unk = sizeof(double) * ne3() * c.nunk;
    S.stage_leaves = (int)std::max<size_t>(1, std::min<size_t>(nleaf, (1ull << 30) / per_unk));
    CKA(cudaMalloc(&S.stage, per_unk * S.stage_leaves));
    // batch of guard-filled blocks + pipeline intermediates: up to 60 % of what is free
    const size_t per_entry = r * S.ngcb * ne3() + sig3d_bytes(S.n, S.n, S.n, r) +
                             w3d_bytes(0, S.n, S.n, S.n, r) + w3d_bytes(1, S.n, S.n, S.n, r) + w3d_bytes(2, S.n, S.n, S.n, r) +
                             f3d_bytes(0, S.n, S.n, S.n, r) + f3d_bytes(1, S.n, S.n, S.n, r) + f3d_bytes(2, S.n, S.n, S.n, r) +
                             (c.prm.order == 3 && r == 8 ? slp3d_bytes(S.n, S.n, S.n, r) : 0) +
                             (c.prm.flattening ? r * 3 * (size_t)(S.n + 2) * (S.n + 2) * (S.n + 2) : 0) +
                             (c.prm.hybrid_order ? r * (size_t)(S.n + 6) * (S.n + 6) * (S.n + 6) +
                                                       (size_t)(S.n + 2) * (S.n + 2) * (S.n + 2) : 0);
    size_t fr = 0, tot = 0;
    CKA(cudaMemGetInfo(&fr, &tot));
    long cap = (long)((fr * 6 / 10) / per_entry);
    if (cap < 1) return record_error(FXB_ECUDA, "fxb_register_blocks: not enough device memory for one AMR block");
    S.batch = (int)std::min<long>(std::min<long>(cap, nleaf), 65535);
    // FXB_AMR_MAX_BATCH caps the leaves processed per batch (device memory for
    // guard-filled blocks and pipeline intermediates grows with it)
    if (const char *ev = getenv("FXB_AMR_MAX_BATCH")) {
        long mb = atol(ev);
        if (mb >= 1) S.batch = (int)std::min<long>(S.batch, mb);
    }
    CKA(cudaMalloc(&S.gcb, r * S.ngcb * ne3() * S.batch));
    CKA(cudaMalloc(&S.sig, sig3d_bytes(S.n, S.n, S.n, r) * S.batch));
    // PPM slopes in memory: FP64 only (the FP32 face-state kernel computes them itself)
    if (c.prm.order == 3 && r == 8) CKA(cudaMalloc(&S.slp, slp3d_bytes(S.n, S.n, S.n, r) * S.batch));
    if (c.prm.flattening) CKA(cudaMalloc(&S.flat, r * 3 * (size_t)(S.n + 2) * (S.n + 2) * (S.n + 2) * S.batch));
    if (c.prm.hybrid_order)
        CKA(cudaMalloc(&S.hyb, (r * (size_t)(S.n + 6) * (S.n + 6) * (S.n + 6) + (size_t)(S.n + 2) * (S.n + 2) * (S.n + 2)) *
                                   S.batch));
    for (int d = 0; d < 3; d++) {
        CKA(cudaMalloc(&S.w[d], w3d_bytes(d, S.n, S.n, S.n, r) * S.batch));
        CKA(cudaMalloc(&S.f[d], f3d_bytes(d, S.n, S.n, S.n, r) * S.batch));
    }
    CKA(cudaStreamSynchronize(st));
    S.cur = 0;
    S.active = true;
    int prc = persist_setup();
    if (prc) return prc;
    return set_step_entries();
}

// one step as batched launches of the stage kernels (the current state is
// not switched); nl: the launches
int batched_step(const double *dtv, double dt, int &nl)
{
    const bool mixed = S.C.prm.precision == FXB_MIXED;
    nl = 0;
    nl += restrict_needed(S.cur);
    Args3D a = batch_args(dtv, dt);
    auto fluxes = [&](int cnt) {
        const int all = AMR_SIG | AMR_STATES;
        if (mixed) launch_amr3d_fluxes_mixed(a, cnt, all, S.C.stream);
        else launch_amr3d_fluxes_fp64(a, cnt, all, S.C.stream);
    };
    auto emit = [&](int cnt) {
        if (mixed) launch_amr3d_emit_mixed(a, cnt, S.bflux, S.nfc, S.C.stream);
        else launch_amr3d_emit_fp64(a, cnt, S.bflux, S.nfc, S.C.stream);
    };
    auto correct = [&](int cnt) {
        if (mixed) launch_amr3d_correct_mixed(a, cnt, S.bflux, S.nfc, S.d_fine, S.d_finer, S.C.stream);
        else launch_amr3d_correct_fp64(a, cnt, S.bflux, S.nfc, S.d_fine, S.d_finer, S.C.stream);
    };
    auto update = [&](int cnt) {
        if (mixed) launch_amr3d_update_mixed(a, cnt, S.C.stream); else launch_amr3d_update_fp64(a, cnt, S.C.stream);
    };
    // sigma (+ flattening), then per direction the slopes, face states and
    // fluxes (one fused kernel in FP32; slopes (PPM), face states and fluxes
    // as separate kernels in FP64)
    const int pipe = 1 + (S.C.prm.flattening ? 1 : 0) + 3 * (mixed ? 1 : (S.C.prm.order == 3 ? 3 : 2));
    if (S.nstep <= S.batch) {
        a.batch = S.d_step_entries;
        nl += fill_batch(a.batch, S.nstep, S.cur);
        fluxes(S.nstep); emit(S.nstep); correct(S.nstep); update(S.nstep);
        nl += pipe + 3;
    } else {
        for (int l0 = 0; l0 < S.nstep; l0 += S.batch) {
            int cnt = std::min(S.batch, S.nstep - l0);
            a.batch = S.d_step_entries + S.nstep + l0;
            nl += fill_batch(a.batch, cnt, S.cur);
            fluxes(cnt); emit(cnt); update(cnt);
            nl += pipe + 2;
        }
        for (int l0 = 0; l0 < S.nstep_finer; l0 += S.batch) {
            int cnt = std::min(S.batch, S.nstep_finer - l0);
            a.batch = S.d_step_entries + 2 * S.nstep + l0;
            nl += fill_batch(a.batch, cnt, S.cur);
            fluxes(cnt); correct(cnt); update(cnt);
            nl += pipe + 2;
        }
    }
    CKA(cudaGetLastError());
    return FXB_OK;
}

// Launch-shape search on the attached state: the guard fill, sigma, the PPM
// slopes and the update are timed with 1, 2, 4, 8 and 16 CTAs per block (one
// warm-up pass, one timed pass each) and the fastest count per stage is kept
// (the face-state and flux kernel has fixed tiles and is timed with the
// slopes).  The stages compute cells independently, so the choice changes
// timings, never results.  The update writes the other interior store, which
// the next step overwrites.
int amr_tune()
{
    const char *ev = getenv("FXB_AMR_TUNE");
    if (ev && atoi(ev) == 0) {
        snprintf(S.tune_log, sizeof(S.tune_log), "AMR launch shape (CTAs per block): fill=%d sig=%d slopes=%d "
                 "update=%d, defaults (tuning off); step form: %s", S.fill_cta, S.cta[0], S.cta[1], S.cta[3],
                 S.persist ? "persistent" : "batched launches");
        return FXB_OK;
    }
    const bool mixed = S.C.prm.precision == FXB_MIXED;
    const int cand[5] = {1, 2, 4, 8, 16};
    const int cnt = std::min(S.nleaf, S.batch);
    cudaEvent_t e[5];
    for (int i = 0; i < 5; i++) CKA(cudaEventCreate(&e[i]));
    float best[4] = {1e30f, 1e30f, 1e30f, 1e30f};
    int pick[4] = {S.fill_cta, S.cta[0], S.cta[1], S.cta[3]};
    restrict_all(S.cur);
    for (int c : cand) {
        S.fill_cta = c;
        for (int q = 0; q < 4; q++) S.cta[q] = c;
        Args3D a = batch_args(nullptr, 0.0);
        a.batch = S.d_entries;
        float t[4] = {0, 0, 0, 0};
        for (int rep = 0; rep < 2; rep++) {
            CKA(cudaEventRecord(e[0], S.C.stream));
            fill_batch(a.batch, cnt, S.cur);
            CKA(cudaEventRecord(e[1], S.C.stream));
            for (int st = 0; st < 2; st++) {
                if (mixed) launch_amr3d_fluxes_mixed(a, cnt, 1 << st, S.C.stream);
                else launch_amr3d_fluxes_fp64(a, cnt, 1 << st, S.C.stream);
                CKA(cudaEventRecord(e[2 + st], S.C.stream));
            }
            if (mixed) launch_amr3d_update_mixed(a, cnt, S.C.stream); else launch_amr3d_update_fp64(a, cnt, S.C.stream);
            CKA(cudaEventRecord(e[4], S.C.stream));
            CKA(cudaGetLastError());
            CKA(cudaEventSynchronize(e[4]));
            for (int k = 0; k < 4; k++) CKA(cudaEventElapsedTime(&t[k], e[k], e[k + 1]));
        }
        for (int k = 0; k < 4; k++)
            if (t[k] < best[k]) { best[k] = t[k]; pick[k] = c; }
    }
    S.fill_cta = pick[0];
    S.cta[0] = pick[1];
    S.cta[1] = pick[2];
    S.cta[2] = pick[2];
    S.cta[3] = pick[3];
    // the step's form: one persistent kernel with clusters of K CTAs per
    // leaf, or the batched launches; each timed over a whole step (one
    // warm-up run, one timed run), the fastest kept.  FXB_AMR_PERSISTENT=1
    // keeps the persistent kernel, FXB_AMR_CLUSTER=K its cluster size.
    char form[160] = "";
    if (S.persist_ok && !S.test_stall) {
        auto time_step = [&](bool pers, float &ms) -> int {
            for (int rep = 0; rep < 2; rep++) {
                CKA(cudaEventRecord(e[0], S.C.stream));
                int nl = 0;
                int rc = pers ? persist_step(nullptr, 0.0) : batched_step(nullptr, 0.0, nl);
                if (rc) return rc;
                CKA(cudaEventRecord(e[1], S.C.stream));
                CKA(cudaEventSynchronize(e[1]));
                CKA(cudaEventElapsedTime(&ms, e[0], e[1]));
            }
            return FXB_OK;
        };
        float tb = 0.f;
        int rc = time_step(false, tb);
        if (rc) return rc;
        const char *ek = getenv("FXB_AMR_CLUSTER"), *ep = getenv("FXB_AMR_PERSISTENT");
        const int kc[4] = {1, 2, 4, 8};
        float tk[4] = {-1.f, -1.f, -1.f, -1.f}, tbest = 1e30f;
        int kbest = S.pK;
        for (int q = 0; q < 4; q++) {
            if (ek && kc[q] != S.pK) continue;
            const int nc = persist_clusters(kc[q]);
            if (nc < 1) continue;
            S.pK = kc[q];
            S.pclusters = nc;
            rc = time_step(true, tk[q]);
            if (rc) return rc;
            if (tk[q] < tbest) { tbest = tk[q]; kbest = kc[q]; }
        }
        S.pK = kbest;
        S.pclusters = persist_clusters(kbest);
        S.persist = (ep && ep[0] == '1') || tbest < tb;
        snprintf(form, sizeof(form), "; step form: %s (ms per step: batched %.2f, persistent K=1 %.2f K=2 %.2f K=4 %.2f "
                 "K=8 %.2f)", S.persist ? (kbest == 1 ? "persistent, 1 CTA per leaf" : "persistent, cluster per leaf")
                 : "batched launches", tb, tk[0], tk[1], tk[2], tk[3]);
    } else {
        snprintf(form, sizeof(form), "; step form: %s (not timed)", S.persist ? "persistent" : "batched launches");
    }
    for (int i = 0; i < 5; i++) cudaEventDestroy(e[i]);
    CKA(cudaMemsetAsync(S.C.rate_max, 0, sizeof(unsigned long long), S.C.stream));
    CKA(cudaStreamSynchronize(S.C.stream));
    snprintf(S.tune_log, sizeof(S.tune_log),
             "AMR launch shape (CTAs of 256 per block, %d blocks of %d^3): fill=%d sig=%d slopes=%d update=%d "
             "(ms fill %.3f, sigma %.3f, slopes + face states + fluxes %.3f, update %.3f)%s", cnt, S.n, pick[0],
             pick[1], pick[2], pick[3], best[0], best[1], best[2], best[3], form);
    return FXB_OK;
}

const char *amr_tuning_log() { return S.tune_log; }

static int copy_leaves(const int *leaves, int n, double *buf, long mstride, bool pack);

// the leaves a host UNK holds: every leaf, or a split mesh's own leaves
static bool split_unk() { return !S.roles.empty(); }
static int host_nleaf() { return split_unk() ? S.nown : S.nleaf; }
static const int *host_leaf_blk() { return split_unk() ? S.d_own_blk : S.leaf_blk_dev; }
static const AmrEntry3 *host_entries() { return split_unk() ? S.d_own_entries : S.d_entries; }

int amr_host_leaves() { return host_nleaf(); }

int amr_attach(const double *unk_host)
{
    const size_t per_unk = (size_t)ne3() * S.C.nunk;
    const int nh = host_nleaf();
    for (int l0 = 0; l0 < nh; l0 += S.stage_leaves) {
        int nl = std::min(S.stage_leaves, nh - l0);
        CKA(cudaMemcpyAsync(S.stage, unk_host + per_unk * l0, sizeof(double) * per_unk * nl, cudaMemcpyHostToDevice,
                            S.C.stream));
        long work = (long)nl * S.vstride;
        int grid = (int)std::min<long>((work + 255) / 256, 148L * 16);
        amr_unk_to_store_kernel<<<grid, 256, 0, S.C.stream>>>(S.stage, l0, nl, host_leaf_blk(), S.store[S.cur],
                                                             S.vstride, S.bstride, S.n, S.ng, S.C.nunk, S.d_dmap);
        CKA(cudaGetLastError());
    }
    if (split_unk() && nh > 0 && nh < S.nleaf) {
        // the other ranks' leaves start as copies of the first own leaf (a
        // valid state for the launch-shape timing; the exchange before each
        // step replaces the ones the step reads)
        std::vector<int> rest;
        rest.reserve(S.nleaf - nh);
        for (int l = 0; l < S.nleaf; l++)
            if (S.roles[l] != 1) rest.push_back(l);
        int first = 0;
        while (S.roles[first] != 1) first++;
        const double *src = S.store[S.cur] + (long)S.leaf_blk[first] * S.bstride;
        for (size_t q0 = 0; q0 < rest.size(); q0 += 65535) {
            const int cnt = (int)std::min<size_t>(65535, rest.size() - q0);
            int rc = copy_leaves(rest.data() + q0, cnt, const_cast<double *>(src), 0, false);
            if (rc) return rc;
        }
    }
    CKA(cudaStreamSynchronize(S.C.stream));
    if (S.tuned) return FXB_OK;      // new data on the same mesh keeps the launch shapes
    S.tuned = true;
    return amr_tune();
}

int amr_sync_to_host(double *unk_host)
{
    const size_t per_unk = (size_t)ne3() * S.C.nunk;
    restrict_all(S.cur);
    const int chunk = S.stage_leaves, nh = host_nleaf();
    for (int l0 = 0; l0 < nh; l0 += chunk) {
        int nl = std::min(chunk, nh - l0);
        // variables the device does not hold keep their host values
        CKA(cudaMemcpyAsync(S.stage, unk_host + per_unk * l0, sizeof(double) * per_unk * nl, cudaMemcpyHostToDevice,
                            S.C.stream));
        // guard fill straight into the FP64 staging copy
        amr_fill_kernel<double, true><<<dim3(S.fill_cta, nl), 256, 0, S.C.stream>>>(
            mesh_args(S.cur), host_entries() + l0, S.leaf_blk_dev, S.d_eosmask, S.stage, 0, (long)per_unk, S.C.nunk,
            S.d_dmap, nullptr, 0, S.C.dprm, S.C.gam1inv, S.C.ggprodinv);
        CKA(cudaGetLastError());
        CKA(cudaMemcpyAsync(unk_host + per_unk * l0, S.stage, sizeof(double) * per_unk * nl, cudaMemcpyDeviceToHost,
                            S.C.stream));
    }
    CKA(cudaStreamSynchronize(S.C.stream));
    return FXB_OK;
}

int amr_fill_to_host(double *unk_host, const int pos[NV_DEV], int n, const int slot[NV_DEV], bool do_eos)
{
    const long per = ne3();
    restrict_all(S.cur);
    if (!S.d_pmap) CKA(cudaMalloc(&S.d_pmap, sizeof(int) * NV_DEV));
    CKA(cudaMemcpyAsync(S.d_pmap, pos, sizeof(int) * NV_DEV, cudaMemcpyHostToDevice, S.C.stream));
    // the staging buffer holds stage_leaves whole UNK blocks, so at least as
    // many packed ones
    const int chunk = S.stage_leaves, nh = host_nleaf();
    for (int l0 = 0; l0 < nh; l0 += chunk) {
        const int nl = std::min(chunk, nh - l0);
        amr_fill_kernel<double, true><<<dim3(S.fill_cta, nl), 256, 0, S.C.stream>>>(
            mesh_args(S.cur), host_entries() + l0, S.leaf_blk_dev, do_eos ? S.d_eosmask : nullptr, S.stage, 0,
            per * n, n, S.d_pmap, nullptr, 0, S.C.dprm, S.C.gam1inv, S.C.ggprodinv);
        CKA(cudaGetLastError());
        int rc = pack_to_host(S.stage, per * nl, n, slot, unk_host + per * S.C.nunk * l0);
        if (rc) return rc;
    }
    return FXB_OK;
}

int amr_step(const double *dtv, double dt, int *launches)
{
    int nl = 1;
    int rc = S.persist ? persist_step(dtv, dt) : batched_step(dtv, dt, nl);
    if (rc) return rc;
    S.cur = 1 - S.cur;
    if (launches) *launches = nl;
    return FXB_OK;
}

// Grid_updateRefinement's data movement on the device after the caller's tree
// update (Paramesh4/Grid_updateRefinement.F90:109, gr_updateRefinement.F90:
// 130-265): the old tree's parents are restricted from their children; the
// new mesh is built from `leaves`; each of its blocks that existed before
// keeps its data (a derefined parent its children's average); new children,
// level by level from coarse to fine, are prolonged from their parent in
// conserved form (mpi_amr_prolong.F90); Eos on every leaf.  Only the old
// interior store stays allocated while the new mesh is built, and the launch
// shapes tuned on the old mesh are kept.  A rejected list, or a new block
// whose parent was not an old leaf, restores the old mesh and its data.
int amr_regrid(const fxb_block_desc *leaves, int nleaf)
{
    if (!S.active) return record_error(FXB_EARG, "fxb_regrid: needs a registered AMR mesh");
    restrict_all(S.cur);
    CKA(cudaStreamSynchronize(S.C.stream));
    State old = std::move(S);
    S = State();
    double *ostore = old.store[old.cur];
    old.store[old.cur] = nullptr;
    free_device(old);
    const long obstride = old.bstride;
    std::vector<fxb_block_desc> olist(old.nleaf);
    for (int l = 0; l < old.nleaf; l++) {
        const HBlock &B = old.blk[old.leaf_blk[l]];
        olist[l].level = B.level;
        for (int a = 0; a < 3; a++) olist[l].bcoord[a] = B.c[a];
    }
    // the old mesh back, with its data, after a failure
    auto restore = [&](int code) -> int {
        amr_destroy();
        int rc = amr_create(old.C, olist.data(), old.nleaf);
        if (rc == FXB_OK && S.bstride == obstride)
            cudaMemcpyAsync(S.store[0], ostore, sizeof(double) * obstride * S.nblk, cudaMemcpyDeviceToDevice,
                            S.C.stream);
        cudaStreamSynchronize(S.C.stream);
        cudaFree(ostore);
        S.fill_cta = old.fill_cta;
        for (int q = 0; q < 4; q++) S.cta[q] = old.cta[q];
        snprintf(S.tune_log, sizeof(S.tune_log), "%s", old.tune_log);
        S.tuned = old.tuned;
        return code;
    };
    int rc = amr_create(old.C, leaves, nleaf);
    if (rc) return restore(rc);
    std::vector<int2> pairs;
    std::vector<std::vector<int>> fresh(S.maxlev + 1);
    for (int b = 0; b < S.nblk; b++) {
        const HBlock &B = S.blk[b];
        auto it = old.map.find(key(B.level, B.c));
        if (it != old.map.end()) { pairs.push_back(make_int2(b, it->second)); continue; }
        bool ok = B.parent >= 0;
        if (ok) {
            const HBlock &P = S.blk[B.parent];
            auto ip = old.map.find(key(P.level, P.c));
            ok = ip != old.map.end() && old.blk[ip->second].leaf >= 0;
        }
        if (!ok) {
            record_error(FXB_EARG, "fxb_regrid: a new block's parent was not a leaf (one level of change per update)");
            return restore(FXB_EARG);
        }
        fresh[B.level].push_back(b);
    }
    int2 *d_pairs = nullptr;
    int *d_fresh = nullptr;
    CKA(cudaMalloc(&d_pairs, sizeof(int2) * std::max<size_t>(1, pairs.size())));
    CKA(cudaMalloc(&d_fresh, sizeof(int) * std::max(1, S.nblk)));
    if (!pairs.empty()) {
        CKA(cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(int2) * pairs.size(), cudaMemcpyHostToDevice, S.C.stream));
        const long work = (long)pairs.size() * S.bstride;
        const int grid = (int)std::min<long>((work + 255) / 256, 148L * 16);
        amr_copy_blocks_kernel<<<grid, 256, 0, S.C.stream>>>(ostore, S.store[0], d_pairs, (int)pairs.size(), S.bstride);
        CKA(cudaGetLastError());
    }
    long off = 0;
    for (int lev = 2; lev <= S.maxlev; lev++) {
        const int nb = (int)fresh[lev].size();
        if (!nb) continue;
        CKA(cudaMemcpyAsync(d_fresh + off, fresh[lev].data(), sizeof(int) * nb, cudaMemcpyHostToDevice, S.C.stream));
        const long work = (long)nb * S.vstride;
        const int grid = (int)std::min<long>((work + 255) / 256, 148L * 16);
        amr_newchild_kernel<<<grid, 256, 0, S.C.stream>>>(mesh_args(0), d_fresh + off, nb);
        CKA(cudaGetLastError());
        off += nb;
    }
    S.cur = 0;
    rc = amr_eos();
    CKA(cudaStreamSynchronize(S.C.stream));
    cudaFree(d_pairs);
    cudaFree(d_fresh);
    cudaFree(ostore);
    // the launch shapes tuned on the old mesh carry over (blocks of the same
    // size; the shapes change timings, never results)
    S.fill_cta = old.fill_cta;
    for (int q = 0; q < 4; q++) S.cta[q] = old.cta[q];
    snprintf(S.tune_log, sizeof(S.tune_log), "%s", old.tune_log);
    S.tuned = old.tuned;
    return rc;
}

int amr_rate()
{
    long work = amr_leaf_cells();
    int grid = (int)std::min<long>((work + 255) / 256, 148L * 16);
    amr_rate_kernel<<<grid, 256, 0, S.C.stream>>>(S.store[S.cur], S.vstride, S.bstride, S.n, S.leaf_blk_dev, S.d_blk,
                                                  S.d_dxl, S.nleaf, S.C.rate_max, S.d_roles);
    CKA(cudaGetLastError());
    return FXB_OK;
}

int amr_eos()
{
    long work = amr_leaf_cells();
    int grid = (int)std::min<long>((work + 255) / 256, 148L * 16);
    amr_eos_kernel<<<grid, 256, 0, S.C.stream>>>(S.store[S.cur], S.vstride, S.bstride, S.n, S.leaf_blk_dev, S.nleaf,
                                                 S.C.dprm, S.C.gam1inv, S.C.ggprodinv);
    CKA(cudaGetLastError());
    return FXB_OK;
}

int amr_locate(unsigned long long *key)
{
    long work = amr_leaf_cells();
    int grid = (int)std::min<long>((work + 255) / 256, 148L * 16);
    amr_locate_kernel<<<grid, 256, 0, S.C.stream>>>(S.store[S.cur], S.vstride, S.bstride, S.n, S.leaf_blk_dev, S.d_blk,
                                                    S.d_dxl, S.nleaf, S.C.rate_max, key, S.d_roles);
    CKA(cudaGetLastError());
    return FXB_OK;
}

int amr_mark_refine(int nvars, const int *dvar, const int *need_eos, const double *refine_cutoff,
                    const double *derefine_cutoff, const double *refine_filter, int max_refine, int *flags,
                    double *error_out)
{
    const int nact = (int)S.act_blk.size();
    const long next = ne3();
    if (!S.d_ext) {
        CKA(cudaMalloc(&S.d_ext, sizeof(double) * next * std::max(1, nact)));
        CKA(cudaMalloc(&S.d_err, sizeof(double) * std::max(1, nact)));
    }
    restrict_all(S.cur);
    std::vector<double> err(S.nblk, 0.), e(nact);
    std::vector<unsigned char> refine(S.nblk, 0), derefine(S.nblk, 0), stay(S.nblk, 0);
    int any_eos = 0;
    for (int l = 0; l < nvars; l++) any_eos |= need_eos[l];
    for (int l = 0; l < nvars; l++) {
        amr_ext_fill_kernel<<<dim3(8, nact), 256, 0, S.C.stream>>>(mesh_args(S.cur), S.d_active, S.d_act_eos, dvar[l],
                                                                  any_eos, S.d_ext, S.C.dprm, S.C.gam1inv,
                                                                  S.C.ggprodinv);
        amr_error_kernel<<<nact, 256, 0, S.C.stream>>>(S.d_ext, S.d_act_bnd, S.d_active, S.d_blk, S.d_dxl, S.n, S.ng,
                                                       refine_filter[l], S.d_err);
        CKA(cudaGetLastError());
        CKA(cudaMemcpyAsync(e.data(), S.d_err, sizeof(double) * nact, cudaMemcpyDeviceToHost, S.C.stream));
        CKA(cudaStreamSynchronize(S.C.stream));
        // Paramesh4/gr_markRefineDerefine.F90:110-160
        std::fill(err.begin(), err.end(), 0.);
        for (int s = 0; s < nact; s++) err[S.act_blk[s]] = e[s];
        for (int b : S.act_blk) {
            const HBlock &B = S.blk[b];
            const double ep = B.parent >= 0 ? err[B.parent] : 0.;
            if (B.nodetype == 1 && !refine[b] && !stay[b] && err[b] <= derefine_cutoff[l] && ep <= derefine_cutoff[l])
                derefine[b] = 1;
            else
                derefine[b] = 0;
            if (err[b] > refine_cutoff[l]) { derefine[b] = 0; refine[b] = 1; }
            if ((B.nodetype == 1 && err[b] > derefine_cutoff[l]) || ep > derefine_cutoff[l]) stay[b] = 1;
            if (B.level >= max_refine) refine[b] = 0;
        }
    }
    for (int l = 0; l < S.nleaf; l++) {
        const int b = S.leaf_blk[l];
        flags[l] = refine[b] ? 1 : derefine[b] ? -1 : 0;
        if (error_out) error_out[l] = err[b];
    }
    return FXB_OK;
}

int amr_leaf_level(int leaf) { return (leaf >= 0 && leaf < S.nleaf) ? S.blk[S.leaf_blk[leaf]].level : 0; }

int amr_set_roles(const unsigned char *roles, int nleaf)
{
    if (nleaf != S.nleaf) return record_error(FXB_EARG, "fxb_amr_set_roles: one role per leaf");
    dfree(S.d_own_blk);
    dfree(S.d_own_entries);
    S.nown = 0;
    if (!roles) {
        S.roles.clear();
        dfree(S.d_roles);
    } else {
        for (int l = 0; l < nleaf; l++)
            if (roles[l] > 2) return record_error(FXB_EARG, "fxb_amr_set_roles: roles are 0, 1 or 2");
        std::vector<int> own_blk;
        std::vector<AmrEntry3> own_ent;
        for (int l = 0; l < nleaf; l++)
            if (roles[l] == 1) {
                own_blk.push_back(S.leaf_blk[l]);
                own_ent.push_back(AmrEntry3{S.leaf_blk[l], S.blk[S.leaf_blk[l]].level, l, 0});
            }
        if (own_blk.empty()) return record_error(FXB_EARG, "fxb_amr_set_roles: a rank owns at least one leaf");
        S.roles.assign(roles, roles + nleaf);
        if (!S.d_roles) CKA(cudaMalloc(&S.d_roles, (size_t)nleaf));
        CKA(cudaMemcpyAsync(S.d_roles, roles, (size_t)nleaf, cudaMemcpyHostToDevice, S.C.stream));
        CKA(upload(S.d_own_blk, own_blk));
        CKA(upload(S.d_own_entries, own_ent));
        S.nown = (int)own_blk.size();
    }
    if (S.d_plan) CKA(build_rlist());     // restriction of the parent cells the active leaves read
    int rc = set_step_entries();
    if (rc) return rc;
    CKA(cudaStreamSynchronize(S.C.stream));
    return FXB_OK;
}

long amr_leaf_doubles() { return S.bstride; }

// leaf interiors of the current state <-> a device message [q][var][cell]:
// one CTA row per listed leaf, 16-byte copies (a block's interior is
// NV_DEV * n^3 doubles, an even count at every supported n)
static int copy_leaves(const int *leaves, int n, double *buf, long mstride, bool pack)
{
    if (n > S.xcap) {
        dfree(S.d_xlist);
        CKA(cudaMalloc(&S.d_xlist, sizeof(int) * (size_t)n));
        S.xcap = n;
    }
    CKA(cudaMemcpyAsync(S.d_xlist, leaves, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, S.C.stream));
    const int chunks = (int)std::min<long>(8, (S.bstride / 2 + 255) / 256);
    amr_leaf_copy_kernel<<<dim3(chunks, n), 256, 0, S.C.stream>>>(S.store[S.cur], S.bstride, S.leaf_blk_dev,
                                                                   S.d_xlist, buf, mstride, pack ? 1 : 0);
    CKA(cudaGetLastError());
    return FXB_OK;
}

int amr_copy_leaves(const int *leaves, int n, double *buf, bool pack)
{
    if (n == 0) return FXB_OK;
    if (n > 65535) return record_error(FXB_EARG, "fxb_amr_pack_leaves: at most 65535 leaves per message");
    if (((uintptr_t)buf & 15) != 0) return record_error(FXB_EARG, "fxb_amr_pack_leaves: buffer not 16-byte aligned");
    for (int q = 0; q < n; q++)
        if (leaves[q] < 0 || leaves[q] >= S.nleaf) return record_error(FXB_EARG, "fxb_amr_pack_leaves: leaf out of range");
    return copy_leaves(leaves, n, buf, S.bstride, pack);
}

int amr_integrals(double *out7, double *partials, int npartials)
{
    amr_integrals_kernel<<<npartials, 256, 0, S.C.stream>>>(S.store[S.cur], S.vstride, S.bstride, S.n, S.leaf_blk_dev,
                                                            S.d_blk, S.d_dxl, S.nleaf, partials, S.d_roles);
    amr_integrals_final_kernel<<<1, 32, 0, S.C.stream>>>(partials, npartials, partials + (long)npartials * 7);
    CKA(cudaGetLastError());
    CKA(cudaMemcpyAsync(out7, partials + (long)npartials * 7, 7 * sizeof(double), cudaMemcpyDeviceToHost, S.C.stream));
    CKA(cudaStreamSynchronize(S.C.stream));
    return FXB_OK;
}

} // namespace fxb
