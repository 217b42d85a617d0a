// fxb_integrals_noalloc.cu -- volume integrals of caller-owned device arrays
// without any device allocation.
//
// Some callers cannot call cudaMalloc: a Fortran application whose device
// memory is owned by another runtime (an OpenACC/OpenMP-offload data region,
// or a pool allocator that reserved the whole GPU up front) gets an error or
// a fragmented pool from a stray allocation, and a service that accounts
// for every byte it places on the GPU must not have a library allocate
// behind its back.  For them this entry point keeps its only scratch -- the
// per-CTA partial sums of the deterministic two-pass reduction -- in a
// fixed-size array in the library's own device image.
//
// The scratch array is a file-scope __device__ variable.  In host code its
// name is only a host-side handle, not a device address, so the host never
// passes it to a kernel: the first call on each device looks up the device
// address with cudaGetSymbolAddress (with that device current) and caches
// it; every later call on that device reuses the cached address.  Because
// the first call on a device does this set-up, make that first call before
// any stream capture.
//
// The cached address belongs to the device's current CUDA context: after a
// cudaDeviceReset the module is loaded again, possibly elsewhere, and the
// cached address is stale, so a caller that resets a device must not call
// this entry point on it again in the same process.  The set-up is guarded
// by a mutex, so host threads may make their first calls concurrently.
//
// Every call on a device shares the one array and leaves its partial sums
// there; each call writes every slot it later reads, so nothing needs to be
// cleared first.  Calls that overlap on the GPU (different streams, or
// different host threads, on the same device) race on the array and must be
// serialised by the caller.
//
// Results are deterministic for a given ncell (fixed chunks per CTA, fixed
// reduction trees) but are summed in a different order from fxb_integrals,
// so the two differ by roundoff.
#include "../../include/flashx_b200.h"

#include <cuda_runtime.h>
#include <stdio.h>

#include <atomic>
#include <mutex>

namespace fxb {
int record_error(int code, const char *msg);   // fxb_api.cu: feeds fxb_last_error
}

namespace {

constexpr int kThreads = 256;
constexpr long kChunkCells = 4096;        // cells summed by one CTA
constexpr int kMaxPartials = 8192;        // CTAs the static scratch can hold
constexpr int kMaxDevices = 64;

// 8192 x 7 doubles = 448 KiB, held by every GPU that loads the library until exit
static __device__ __align__(256) double g_partials[kMaxPartials * 7];

double *g_partials_dev[kMaxDevices];      // device address of g_partials, per device
std::atomic<bool> g_ready[kMaxDevices];   // g_partials_dev[d] is set
std::mutex g_setup;

__global__ void noalloc_partial_kernel(const double *__restrict__ dens, const double *__restrict__ velx,
                                       const double *__restrict__ vely, const double *__restrict__ velz,
                                       const double *__restrict__ ener, const double *__restrict__ eint,
                                       long ncell, double dv, double *__restrict__ partials)
{
    double s[7] = {0., 0., 0., 0., 0., 0., 0.};
    long lo = blockIdx.x * kChunkCells;
    long hi = lo + kChunkCells < ncell ? lo + kChunkCells : ncell;
    for (long c = lo + threadIdx.x; c < hi; c += kThreads) {
        double rho = dens[c], vx = velx[c], vy = vely[c], vz = velz[c];
        s[0] += rho * dv; s[1] += rho * vx * dv; s[2] += rho * vy * dv; s[3] += rho * vz * dv;
        s[4] += rho * ener[c] * dv; s[5] += rho * eint[c] * dv;
        s[6] += 0.5 * rho * (vx * vx + vy * vy + vz * vz) * dv;
    }
    __shared__ double sh[7][kThreads];
    for (int q = 0; q < 7; q++) sh[q][threadIdx.x] = s[q];
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 7; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 7; q++) partials[blockIdx.x * 7 + q] = sh[q][0];
}

// one CTA: each thread sums a fixed stride of the partials, then a tree
__global__ void __launch_bounds__(kThreads) noalloc_final_kernel(const double *partials, int n, double *out)
{
    double t[7] = {0., 0., 0., 0., 0., 0., 0.};
    for (int b = threadIdx.x; b < n; b += kThreads)
        for (int q = 0; q < 7; q++) t[q] += partials[b * 7 + q];
    __shared__ double sh[7][kThreads];
    for (int q = 0; q < 7; q++) sh[q][threadIdx.x] = t[q];
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 7; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 7) out[threadIdx.x] = sh[threadIdx.x][0];
}

} // namespace

extern "C" int fxb_integrals_noalloc(const double *dens, const double *velx, const double *vely,
                                     const double *velz, const double *ener, const double *eint,
                                     long ncell, double cell_volume, double *out_dev, void *stream)
{
    if (!dens || !velx || !vely || !velz || !ener || !eint || !out_dev)
        return fxb::record_error(FXB_EARG, "fxb_integrals_noalloc: null device pointer");
    if (ncell <= 0) return fxb::record_error(FXB_EARG, "fxb_integrals_noalloc: ncell must be positive");
    long nparts = (ncell + kChunkCells - 1) / kChunkCells;
    if (nparts > kMaxPartials) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "fxb_integrals_noalloc: %ld cells exceed the static scratch capacity of %ld cells "
                 "(%d partial sums of %ld cells)", ncell, (long)kMaxPartials * kChunkCells, kMaxPartials,
                 kChunkCells);
        return fxb::record_error(FXB_EARG, msg);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fxb::record_error(FXB_ECUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fxb::record_error(FXB_EARG, "fxb_integrals_noalloc: device index too large");
    if (!g_ready[dev].load(std::memory_order_acquire)) {
        // set-up, once per device, with that device current
        std::lock_guard<std::mutex> lock(g_setup);
        if (!g_ready[dev].load(std::memory_order_relaxed)) {
            e = cudaGetSymbolAddress((void **)&g_partials_dev[dev], g_partials);
            if (e != cudaSuccess) return fxb::record_error(FXB_ECUDA, cudaGetErrorString(e));
            g_ready[dev].store(true, std::memory_order_release);
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    noalloc_partial_kernel<<<(unsigned)nparts, kThreads, 0, s>>>(dens, velx, vely, velz, ener, eint, ncell,
                                                                 cell_volume, g_partials_dev[dev]);
    noalloc_final_kernel<<<1, kThreads, 0, s>>>(g_partials_dev[dev], (int)nparts, out_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fxb::record_error(FXB_ECUDA, cudaGetErrorString(e));
    return FXB_OK;
}
