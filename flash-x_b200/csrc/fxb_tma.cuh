// fxb_tma.cuh -- tensor-memory-accelerator (TMA) staging of grid windows
// into shared memory, with an mbarrier whose wait is bounded.
//
// A window of several state variables is one 3-D box [var][y][x] of a
// tensor map over the device mirror (x fastest, rows of nx doubles,
// variables vstride doubles apart).  One thread arms the CTA's mbarrier
// with the box's byte count and issues cp.async.bulk.tensor; every thread
// then waits on the barrier's phase.  The wait gives up after a clock
// budget (the copy of a few tens of kB completes in microseconds), sets
// ERR_TIMEOUT in the device error word and, before the CTA may exit, waits
// once more, again bounded, for the copy still in flight.
//
// Alignment (checked by the callers): the shared-memory destination is 128-B
// aligned, the box's inner extent times 8 B and its x origin times 8 B are
// multiples of 16 B.  No multicast: every CTA loads its own box from this
// GPU's memory.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fxb {

enum { ERR_TIMEOUT = 32 };

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// 3-D tiled load of the box at (x, y, z) of `map` into shared memory `dst`,
// completing on `bar` (no cluster multicast)
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];"
                 ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
                 : "memory");
}

// Wait for phase `parity` of `bar` for at most `budget` clock cycles.  On
// expiry: ERR_TIMEOUT into *err, then one more bounded wait so that no copy
// is left writing into shared memory of a CTA that returns; false is
// returned and the caller's CTA returns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, long long budget, int *err)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > budget) {
            atomicOr(err, ERR_TIMEOUT);
            const long long t1 = clock64();
            while (!mbar_try_wait(bar, parity) && clock64() - t1 < budget) {
            }
            return false;
        }
    }
    return true;
}

// about 1 s at the B200's 1.965 GHz: far above any window copy
constexpr long long kTmaWaitBudget = 2000000000LL;

} // namespace fxb
