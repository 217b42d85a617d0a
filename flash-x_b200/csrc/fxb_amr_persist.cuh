// fxb_amr_persist.cuh -- one persistent kernel per AMR step over the
// device-resident leaf list.
//
// Replaces, on a block-structured mesh, the leaf loop of
// levelFlux/Hydro.F90:161-270 (Grid_fillGuardCells, hy_computeFluxes per
// leaf, Grid_putFluxData, Grid_conserveFluxes, hy_updateSolution) with a
// device work queue.  Every CTA pulls items from one counter:
//
//   1. restriction items, deepest level first: chunks of the parent cells
//      the guard-fill plan reads (amr_restrict_unk); an item of level L
//      starts once every item of level L+1 is done;
//   2. leaf items, finest level first: once every restriction item is done,
//      the CTA copies the leaf's entry into its scratch slot and runs the
//      whole pipeline on it -- guard fill (same-level copies, multilinear
//      prolongation, Eos on guard regions), flattening, sigma, per direction
//      the slopes, face states and Riemann fluxes, the boundary fluxes
//      (Grid_putFluxData), then, for a leaf next to finer leaves, waits until
//      those leaves have emitted their boundary fluxes and replaces its own
//      fluxes on the shared faces (Grid_conserveFluxes), and finally the
//      conserved update, energyFix, Eos and CFL rate.
//
// Every wait is on items that sit earlier in the queue (finer leaves, deeper
// restriction levels), which were taken by CTAs that are running, so the
// queue always progresses without a cooperative launch.  Each wait is
// nevertheless bounded by a clock budget: on expiry the CTA sets ERR_TIMEOUT
// in the device error word and the abort flag, every CTA leaves at its next
// wait or dequeue, and the host reports FXB_ETIMEOUT.
//
// A leaf runs on one thread-block cluster of K CTAs (K = 1, 2, 4 or 8, chosen
// by the library's tuner): every stage's cells are split over the K CTAs and
// the stages are separated by cluster barriers, so a leaf's dependency chain
// is cut K-fold while all leaves stay independent.  The queue item and the
// outcome of every wait are decided by CTA 0 of the cluster and read by the
// others from its shared memory.
//
// The intermediates of a leaf live in the scratch slot of the cluster that
// runs it (the batch arrays, indexed by the slot), so the scratch grows with
// the number of resident clusters, not with the number of leaves.
#pragma once
#include <cooperative_groups.h>
#include "fxb_amr_dev.cuh"
#include "fxb_hydro3d.cuh"
#include "fxb_tma.cuh"

namespace fxb {

enum { PQ_HEAD = 0, PQ_RDONE = 1, PQ_ABORT = 2, PQ_LEVEL = 3, PQ_WORDS = PQ_LEVEL + 32 };

struct PersistArgs {
    Args3D a;                     // batch arguments; a.batch is the slot table
    MeshArgs m;                   // the mesh, store = the step's input state
    AmrEntry3 *slots;             // one entry per CTA (the leaf it runs)
    const AmrEntry3 *leaf_entry;  // entry of every leaf (flags 0)
    const int *order;             // leaves in queue order, finest level first
    const int *leaf_blk;
    const GuardPlan *plan;
    const int *glist;
    int nglist;
    const ProlRec *prol;
    const int *poff;
    int has_prol;
    const int4 *ritems;           // restriction items: level, first and last+1 entry of rlist
    const int2 *rlist;
    const int *child;
    int nritem, nleaf;
    int rlev_items[32];           // restriction items per level
    void *bflux;
    long nfc;
    const int *fine;
    const int *finer_mask;
    int *ctl;                     // PQ_* words, zeroed before the launch
    int *emitted;                 // per leaf: 1 once its boundary fluxes are stored, zeroed before the launch
    long long budget;             // clock cycles of one bounded wait
    int test_stall;               // test hook: leaves next to finer ones wait on a flag nothing sets
};

// The kernel's arguments, one set per current interior store (the step reads
// store `which` and writes the other), uploaded once per mesh: in constant
// memory the stage functions read every field through the constant bank, as
// the stand-alone stage kernels read their parameters, instead of holding
// them in registers.  The step's dt is read from the device (a.dtv).
// (raw storage: the argument structs have default member initialisers,
// which a __constant__ variable cannot run)
static __constant__ __align__(16) unsigned char c_persist_raw[2 * sizeof(PersistArgs)];
#define c_persist (reinterpret_cast<const PersistArgs *>(c_persist_raw))

__device__ __forceinline__ int ld_acquire_gpu(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// thread 0: wait until *ctr >= target; false on abort or on an expired budget
// (which raises the abort flag for everyone)
__device__ __forceinline__ bool persist_wait(const PersistArgs &p, const int *ctr, int target)
{
    const long long t0 = clock64();
    while (ld_acquire_gpu(ctr) < target) {
        if (ld_acquire_gpu(p.ctl + PQ_ABORT)) return false;
        if (clock64() - t0 > p.budget) {
            atomicOr(p.a.err, ERR_TIMEOUT);
            atomicExch(p.ctl + PQ_ABORT, 1);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// a barrier over every thread of the leaf's cluster (release / acquire at
// cluster scope, so the stages' global stores are seen by all its CTAs)
__device__ __forceinline__ void leaf_sync() { cooperative_groups::this_cluster().sync(); }

// every thread's stores of the cluster done, then one release increment
__device__ __forceinline__ void persist_signal(int *ctr)
{
    leaf_sync();
    if (cooperative_groups::this_cluster().block_rank() == 0 && threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1);
    }
}

// the cluster-wide outcome of a wait by thread 0 of the cluster's CTA 0
__device__ __forceinline__ bool persist_block_wait(const PersistArgs &p, const int *ctr, int target)
{
    __shared__ int ok;
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    if (cl.block_rank() == 0 && threadIdx.x == 0) ok = persist_wait(p, ctr, target) ? 1 : 0;
    cl.sync();
    const bool r = *cl.map_shared_rank(&ok, 0) != 0;
    cl.sync();
    return r;
}

// one direction's slopes (FP64 PPM), face states and fluxes for the slot's
// leaf, reconstruction ORDER 3 (PPM) or 5 (WENO5)
template <class R, int ORDER, int DIR>
__device__ __forceinline__ void persist_direction(const Args3D &a, const VB vb, unsigned char *smem)
{
    if constexpr (FusedFaces<R>::value) {
        const int N = DIR == 0 ? a.nx : DIR == 1 ? a.ny : a.nz;
        const int N1 = DIR == 0 ? a.ny : a.nx, N2 = DIR == 2 ? a.ny : a.nz;
        const int Ls = a.sf_len[DIR], T1 = a.sf_lines[DIR];
        const int nseg = (N + Ls - 1) / (Ls - 1), nt1 = (N1 + T1 - 1) / T1;
        const int ntile = nseg * nt1 * N2;
        const int nt = ORDER == 5 ? Ls * T1 : (Ls + 2) * T1;
        for (int tile = vb.x; tile < ntile; tile += vb.nx) {
            sflux3d_kernel_body<R, ORDER, true, DIR, false>(a, VB{tile, vb.y, ntile}, smem, nt);
            __syncthreads();   // the tile's shared face states are reused by the CTA's next tile
        }
    } else {
        if constexpr (ORDER == 3) {
            slope3d_kernel_body<R, true>(a, vb, DIR);
            leaf_sync();
        }
        states3d_kernel_body<R, ORDER, true, DIR, false>(a, vb);
        leaf_sync();
        flux3d_kernel_body<R, true, DIR, false>(a, vb);
    }
    leaf_sync();
}

// Each stage is a function of its own (not inlined), so that the registers
// of one stage do not stay live through, or crowd, the next: the kernel's
// budget is that of the batched stage kernels (two 256-thread CTAs per SM in
// FP64, three 288-thread CTAs in FP32).
template <class R>
__device__ __noinline__ void persist_fill(const int which, const VB vb)
{
    const PersistArgs &p = c_persist[which];
    const Args3D &a = p.a;
    amr_copy_kernel_body<R>(vb, p.m, p.slots, p.leaf_blk, p.plan, p.glist, p.nglist, (R *)a.gcb, a.gcb_vstride,
                            a.gcb_bstride, a.prm, a.gam1inv, a.ggprodinv);
    if (p.has_prol)
        amr_prolong_kernel_body<R>(vb, p.m, p.slots, p.prol, p.poff, (R *)a.gcb, a.gcb_vstride, a.gcb_bstride, a.prm,
                                   a.gam1inv, a.ggprodinv);
}
template <class R> __device__ __noinline__ void persist_flat(const int which, const VB vb)
{ flat3d_kernel_body<R, true>(c_persist[which].a, vb); }
template <class R> __device__ __noinline__ void persist_sig(const int which, const VB vb)
{ sig3d_kernel_body<R, true>(c_persist[which].a, vb); }
template <class R, int ORDER, int DIR>
__device__ __noinline__ void persist_dir(const int which, const VB vb, unsigned char *smem)
{ persist_direction<R, ORDER, DIR>(c_persist[which].a, vb, smem); }
template <class R>
__device__ __noinline__ void persist_emit(const int which, const VB vb)
{
    const PersistArgs &p = c_persist[which];
    amr_emit_flux_kernel_body<R>(p.a, vb, (R *)p.bflux, p.nfc);
}
template <class R>
__device__ __noinline__ void persist_correct(const int which, const VB vb)
{
    const PersistArgs &p = c_persist[which];
    amr_correct_flux_kernel_body<R>(p.a, vb, (const R *)p.bflux, p.nfc, p.fine, p.finer_mask);
}
template <class R> __device__ __noinline__ void persist_update(const int which, const VB vb)
{ update3d_kernel_body<R, true>(c_persist[which].a, vb); }

template <class R> struct PersistThreads { static constexpr int value = FusedFaces<R>::value ? FXB_SF_MAXT : 256; };
template <class R> struct PersistMinB { static constexpr int value = FusedFaces<R>::value ? 3 : 2; };
template <class R> constexpr int persist_smem_bytes() { return FusedFaces<R>::value ? 14 * (int)sizeof(R) * FXB_SF_MAXT : 0; }

template <class R>
__global__ void __launch_bounds__(PersistThreads<R>::value, PersistMinB<R>::value)
amr_persist_kernel(const int which)
{
    const PersistArgs &p = c_persist[which];
    extern __shared__ __align__(16) unsigned char psmem[];
    __shared__ int s_item;
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    const int K = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int slot = blockIdx.x / K;     // the grid is 1-D: consecutive CTAs form a cluster
    const VB vb{rank, slot, K};
    const Args3D &a = p.a;
    for (;;) {
        if (rank == 0 && threadIdx.x == 0)
            s_item = ld_acquire_gpu(p.ctl + PQ_ABORT) ? 0x7fffffff : atomicAdd(p.ctl + PQ_HEAD, 1);
        cl.sync();
        const int item = *cl.map_shared_rank(&s_item, 0);
        cl.sync();
        if (item >= p.nritem + p.nleaf) return;
        if (item < p.nritem) {
            // ---- restriction of one chunk of parent cells
            const int4 it = p.ritems[item];
            const int lev = it.x;
            if (lev + 1 < 32 && p.rlev_items[lev + 1] > 0 &&
                !persist_block_wait(p, p.ctl + PQ_LEVEL + lev + 1, p.rlev_items[lev + 1]))
                return;
            for (int t = it.y + rank * (int)blockDim.x + threadIdx.x; t < it.z; t += K * (int)blockDim.x) {
                const int2 pc = p.rlist[t];
                restrict_cell(const_cast<double *>(p.m.store), p.m.vstride, p.m.bstride, p.m.n, pc.x, pc.y, p.child);
            }
            cl.sync();
            if (rank == 0 && threadIdx.x == 0) {
                __threadfence();
                atomicAdd(p.ctl + PQ_LEVEL + lev, 1);
                atomicAdd(p.ctl + PQ_RDONE, 1);
            }
            continue;
        }
        // ---- one leaf
        const int leaf = p.order[item - p.nritem];
        if (p.nritem > 0 && !persist_block_wait(p, p.ctl + PQ_RDONE, p.nritem)) return;
        if (rank == 0 && threadIdx.x == 0) p.slots[slot] = p.leaf_entry[leaf];
        cl.sync();
        persist_fill<R>(which, vb);
        cl.sync();
        if (a.prm.flattening) {
            persist_flat<R>(which, vb);
            cl.sync();
        }
        persist_sig<R>(which, vb);
        cl.sync();
        if (a.prm.order == 5) {
            persist_dir<R, 5, 0>(which, vb, psmem);
            persist_dir<R, 5, 1>(which, vb, psmem);
            persist_dir<R, 5, 2>(which, vb, psmem);
        } else {
            persist_dir<R, 3, 0>(which, vb, psmem);
            persist_dir<R, 3, 1>(which, vb, psmem);
            persist_dir<R, 3, 2>(which, vb, psmem);
        }
        persist_emit<R>(which, vb);
        persist_signal(p.emitted + leaf);
        // flux ghosts of a split mesh (never updated) skip the correction
        const int mask = (p.leaf_entry[leaf].flags & AMR_SKIP_UPDATE) ? 0 : p.finer_mask[leaf];
        if (mask) {
            // Grid_conserveFluxes: the finer leaves across each refined face
            // must have stored their boundary fluxes
            for (int f = 0; f < 6; f++) {
                if (!((mask >> f) & 1)) continue;
                for (int q = 0; q < 4; q++) {
                    const int fl = p.fine[(long)leaf * 24 + f * 4 + q];
                    const int *flag = p.test_stall ? p.ctl + PQ_WORDS - 1 : p.emitted + fl;
                    if (!persist_block_wait(p, flag, 1)) return;
                }
            }
            persist_correct<R>(which, vb);
            cl.sync();
        }
        persist_update<R>(which, vb);
        cl.sync();   // the slot's entry and scratch are rewritten by the next item
    }
}

template <class R> cudaLaunchConfig_t persist_config(int clusters, int K, cudaStream_t s, cudaLaunchAttribute *attr)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(clusters * K));
    cfg.blockDim = dim3(PersistThreads<R>::value);
    cfg.dynamicSmemBytes = persist_smem_bytes<R>();
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// clusters of K CTAs of the persistent kernel that fit on this device at once
template <class R> int persist_grid(int K)
{
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = persist_config<R>(1, K, 0, attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, amr_persist_kernel<R>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// the two argument sets (current store 0 and 1), once per mesh (synchronous)
template <class R> cudaError_t persist_upload_t(const PersistArgs p0[2])
{
    PersistArgs p[2] = {p0[0], p0[1]};
    for (int w = 0; w < 2; w++) p[w].a = with_divisors(p0[w].a, sflux_halo<R>(p0[w].a));
    return cudaMemcpyToSymbol(c_persist_raw, p, sizeof(p));
}

// `clusters` clusters of K CTAs, one scratch slot each, on argument set `which`
template <class R> cudaError_t launch_amr_persist_t(int which, int clusters, int K, cudaStream_t s)
{
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = persist_config<R>(clusters, K, s, attr);
    return cudaLaunchKernelEx(&cfg, amr_persist_kernel<R>, which);
}

} // namespace fxb
