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
// The intermediates of a leaf live in the scratch slot of the CTA that runs
// it (the batch arrays, indexed by the slot), so the scratch grows with the
// number of resident CTAs, not with the number of leaves.
#pragma once
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

// every thread's stores of this CTA done, then one release increment by thread 0
__device__ __forceinline__ void persist_signal(int *ctr)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1);
    }
}

// the CTA-wide outcome of a thread-0 wait
__device__ __forceinline__ bool persist_block_wait(const PersistArgs &p, const int *ctr, int target)
{
    __shared__ int ok;
    if (threadIdx.x == 0) ok = persist_wait(p, ctr, target) ? 1 : 0;
    __syncthreads();
    const bool r = ok != 0;
    __syncthreads();
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
        for (int tile = 0; tile < ntile; tile++) {
            sflux3d_kernel_body<R, ORDER, true, DIR, false>(a, VB{tile, vb.y, ntile}, smem, nt);
            __syncthreads();   // the tile's shared face states are reused by the next tile
        }
    } else {
        if constexpr (ORDER == 3) {
            slope3d_kernel_body<R, true>(a, vb, DIR);
            __syncthreads();
        }
        states3d_kernel_body<R, ORDER, true, DIR, false>(a, vb);
        __syncthreads();
        flux3d_kernel_body<R, true, DIR, false>(a, vb);
    }
    __syncthreads();
}

// Each stage is a function of its own (not inlined), so that the registers
// of one stage do not stay live through, or crowd, the next: the kernel's
// budget is that of the batched stage kernels (two 256-thread CTAs per SM in
// FP64, three 288-thread CTAs in FP32).
template <class R>
__device__ __noinline__ void persist_fill(const PersistArgs &p, const VB vb)
{
    const Args3D &a = p.a;
    amr_copy_kernel_body<R>(vb, p.m, p.slots, p.leaf_blk, p.plan, p.glist, p.nglist, (R *)a.gcb, a.gcb_vstride,
                            a.gcb_bstride, a.prm, a.gam1inv, a.ggprodinv);
    if (p.has_prol)
        amr_prolong_kernel_body<R>(vb, p.m, p.slots, p.prol, p.poff, (R *)a.gcb, a.gcb_vstride, a.gcb_bstride, a.prm,
                                   a.gam1inv, a.ggprodinv);
}
template <class R> __device__ __noinline__ void persist_flat(const Args3D &a, const VB vb) { flat3d_kernel_body<R, true>(a, vb); }
template <class R> __device__ __noinline__ void persist_sig(const Args3D &a, const VB vb) { sig3d_kernel_body<R, true>(a, vb); }
template <class R, int ORDER, int DIR>
__device__ __noinline__ void persist_dir(const Args3D &a, const VB vb, unsigned char *smem)
{ persist_direction<R, ORDER, DIR>(a, vb, smem); }
template <class R>
__device__ __noinline__ void persist_emit(const PersistArgs &p, const VB vb)
{ amr_emit_flux_kernel_body<R>(p.a, vb, (R *)p.bflux, p.nfc); }
template <class R>
__device__ __noinline__ void persist_correct(const PersistArgs &p, const VB vb)
{ amr_correct_flux_kernel_body<R>(p.a, vb, (const R *)p.bflux, p.nfc, p.fine, p.finer_mask); }
template <class R> __device__ __noinline__ void persist_update(const Args3D &a, const VB vb) { update3d_kernel_body<R, true>(a, vb); }

template <class R> struct PersistThreads { static constexpr int value = FusedFaces<R>::value ? FXB_SF_MAXT : 256; };
template <class R> struct PersistMinB { static constexpr int value = FusedFaces<R>::value ? 3 : 2; };
template <class R> constexpr int persist_smem_bytes() { return FusedFaces<R>::value ? 14 * (int)sizeof(R) * FXB_SF_MAXT : 0; }

template <class R>
__global__ void __launch_bounds__(PersistThreads<R>::value, PersistMinB<R>::value)
amr_persist_kernel(const __grid_constant__ PersistArgs p)
{
    extern __shared__ __align__(16) unsigned char psmem[];
    __shared__ int s_item;
    const int slot = blockIdx.x;
    const VB vb{0, slot, 1};
    const Args3D &a = p.a;
    for (;;) {
        if (threadIdx.x == 0) s_item = ld_acquire_gpu(p.ctl + PQ_ABORT) ? 0x7fffffff : atomicAdd(p.ctl + PQ_HEAD, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= p.nritem + p.nleaf) return;
        if (item < p.nritem) {
            // ---- restriction of one chunk of parent cells
            const int4 it = p.ritems[item];
            const int lev = it.x;
            if (lev + 1 < 32 && p.rlev_items[lev + 1] > 0 &&
                !persist_block_wait(p, p.ctl + PQ_LEVEL + lev + 1, p.rlev_items[lev + 1]))
                return;
            for (int t = it.y + threadIdx.x; t < it.z; t += blockDim.x) {
                const int2 pc = p.rlist[t];
                restrict_cell(const_cast<double *>(p.m.store), p.m.vstride, p.m.bstride, p.m.n, pc.x, pc.y, p.child);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(p.ctl + PQ_LEVEL + lev, 1);
                atomicAdd(p.ctl + PQ_RDONE, 1);
            }
            continue;
        }
        // ---- one leaf
        const int leaf = p.order[item - p.nritem];
        if (p.nritem > 0 && !persist_block_wait(p, p.ctl + PQ_RDONE, p.nritem)) return;
        if (threadIdx.x == 0) p.slots[slot] = p.leaf_entry[leaf];
        __syncthreads();
        persist_fill<R>(p, vb);
        __syncthreads();
        if (a.prm.flattening) {
            persist_flat<R>(a, vb);
            __syncthreads();
        }
        persist_sig<R>(a, vb);
        __syncthreads();
        if (a.prm.order == 5) {
            persist_dir<R, 5, 0>(a, vb, psmem);
            persist_dir<R, 5, 1>(a, vb, psmem);
            persist_dir<R, 5, 2>(a, vb, psmem);
        } else {
            persist_dir<R, 3, 0>(a, vb, psmem);
            persist_dir<R, 3, 1>(a, vb, psmem);
            persist_dir<R, 3, 2>(a, vb, psmem);
        }
        persist_emit<R>(p, vb);
        persist_signal(p.emitted + leaf);
        const int mask = p.finer_mask[leaf];
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
            persist_correct<R>(p, vb);
            __syncthreads();
        }
        persist_update<R>(a, vb);
        __syncthreads();
    }
}

// resident CTAs of the persistent kernel on this device (its grid size)
template <class R> int persist_grid()
{
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, amr_persist_kernel<R>, PersistThreads<R>::value,
                                                      persist_smem_bytes<R>()) != cudaSuccess)
        return 0;
    return nsm * per;
}

template <class R> void launch_amr_persist_t(const PersistArgs &p0, int grid, cudaStream_t s)
{
    PersistArgs p = p0;
    p.a = with_divisors(p0.a, sflux_halo<R>(p0.a));
    amr_persist_kernel<R><<<grid, PersistThreads<R>::value, persist_smem_bytes<R>(), s>>>(p);
}

} // namespace fxb
