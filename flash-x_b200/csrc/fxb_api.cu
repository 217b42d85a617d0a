// fxb_api.cu -- extern "C" entry points of libflashx_b200.so (see
// include/flashx_b200.h for the contract and the reference interfaces each
// one replaces).  Host code only orchestrates: device memory, the library
// stream, kernel launches, CUDA graphs and error reporting.
#include "../../include/flashx_b200.h"
#include "fxb_launch.h"
#include "fxb_amr.h"
#include "fxb_species.cuh"

#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include <algorithm>
#include <array>
#include <unordered_map>
#include <thread>
#include <unordered_set>
#include <vector>

using namespace fxb;

namespace {

struct Lib {
    bool inited = false;
    fxb_params prm{};
    fxb_domain dom{};
    DevParams dprm{};
    int dmap[NV_DEV];              // device variable -> UNK slot
    int nunk = 0;
    int nx = 0, ny = 1, nz = 1;    // extents of the stored grid (a slab: its interior and halos)
    long ncell = 0, vstride = 0;
    int gext[3] = {1, 1, 1};       // cells per axis of the whole grid (cell widths)
    int kbc[6];                    // boundary handling of the stored grid (outflow beside a halo)
    unsigned char *shok = nullptr; // shock detector on: the SHOK flag of every stored cell
    int shock_slot = -1;           // UNK slot of SHOK_VAR (< 0: not written to the host)
    bool shok_valid = false;       // the flags belong to a step taken since the last attach
    fxb_slab slab{};               // this rank's layers of the slowest axis and its halos
    long plane = 1;                // cells in one plane of the slowest axis
    int nint = 1;                  // interior planes of the slowest axis
    long unk_doubles = 0;
    double *buf[2] = {nullptr, nullptr};
    int cur = 0;
    double *unk_dev = nullptr;     // UNK staging mirror (blocks with guard cells)
    int *bcoord = nullptr;         // 3 ints per block
    int *dmap_dev = nullptr;
    int nblk = 0;
    double *dtv = nullptr;         // [dt, dtOld]
    unsigned long long *rate_max = nullptr;
    int *err = nullptr;
    double *partials = nullptr;
    int npartials = 0;
    bool rate_valid = false;
    // Hydro_computeDt result of the current state: computed by the first
    // fxb_compute_dt after the state changed, returned by the later ones
    bool dt_valid = false, loc_valid = false;
    double dt_cached = 0.;
    int32_t loc_cached[5] = {0, 0, 0, 0, 0};
    long long counts[FXB_NCOUNTERS] = {};
    double *pack_host = nullptr;   // pinned staging of masked guard fills
    size_t pack_host_doubles = 0;
    double *pack_dev = nullptr;    // packed selected variables (uniform grid)
    size_t pack_dev_doubles = 0;
    const void *mapped_host = nullptr;   // caller's UNK page-locked for the interior transfers
    size_t mapped_bytes = 0;
    bool mapped_registered = false;      // locked by the library (released at finalize)
    int *pmap_dev = nullptr;       // device variable -> place in a packed cell vector
    const double *unk_attached = nullptr;
    bool attached = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int last_launches = 0;
    bool timing_valid = false;
    cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};   // two steps starting from buffer 0 / 1
    double gam1inv = 0., ggprodinv = 0.;
    void *sig3 = nullptr, *w3[3] = {nullptr, nullptr, nullptr}, *f3[3] = {nullptr, nullptr, nullptr};
    void *slp3 = nullptr;          // PPM slopes of one direction (3-D)
    void *flat = nullptr;          // flattening coefficients (2-D and 3-D)
    void *hyb = nullptr;           // hybrid order (3-D): DivU and the per-cell flags
    // species and mass scalars (fxb_init_species): mass fractions [ns][vstride]
    // per state buffer, their scratch, the hydro's exports
    int ns = 0, nsp = 0;
    int sslot[FXB_MAX_SPECIES];
    int *sslot_dev = nullptr;
    double *spb[2] = {nullptr, nullptr};
    void *ssg = nullptr, *ssl = nullptr, *ssr = nullptr;
    void *sfd[2] = {nullptr, nullptr};             // 2-D mass fluxes
    unsigned char *ctufb[3] = {nullptr, nullptr, nullptr};   // 3-D CTU fallback flags
    long snpad = 0, snw = 0;
    CUtensorMap tmap2d[2];         // 2-D: the window variables of buf[0] / buf[1] for TMA
    int use_tma = 1;
    // launch shapes of the uniform grid, chosen by ug_tune at the first attach
    bool ug_tuned = false;
    int ug_cta[4] = {8, 8, 8, 8};  // 3-D: CTAs per SM of sigma, face states, fluxes, update
    int sf_t1[3] = {0, 0, 0};      // 3-D FP32: lines per fused face-state tile (0: by lane count)
    char ug_log[512] = "";
    unsigned tma_extra_tx = 0;     // test hook (FXB_TEST_WAIT_TIMEOUT): a window barrier that never completes
    long long wait_budget = kTmaWaitBudget;
    fxb_error lasterr{};
};
Lib L;

int fail(int code, const char *msg)
{
    L.lasterr.code = code;
    snprintf(L.lasterr.message, sizeof(L.lasterr.message), "%s", msg);
    return code;
}

int cuda_fail(cudaError_t e, const char *where)
{
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    return fail(FXB_ECUDA, buf);
}

// the device state changed: a cached Hydro_computeDt result is stale; the
// CFL rate is valid only when the change was a fused hydro step
void state_changed(bool fused_rate)
{
    L.rate_valid = fused_rate;
    L.dt_valid = L.loc_valid = false;
}

#define CK(call)                                                    \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return cuda_fail(_e, #call);         \
    } while (0)

// device variable order -> fxb_var
const int kDevToVar[NV_DEV] = {FXB_DENS, FXB_VELX, FXB_VELY, FXB_VELZ, FXB_PRES,
                               FXB_GAMC, FXB_GAME, FXB_EINT, FXB_ENER, FXB_TEMP};

// ------------------------------------------------------------------ kernels
struct UnkGeom {
    int ndim, nxb, nyb, nzb, ng, nig, njg, nkg, nunk;
    int nx, ny, nz;
    int bc[6];
    long vstride;
    int soff;      // stored plane of a global index of the slowest axis: global + soff
};

// hy_shockDetectBlk.F90 on the stored grid: 1 where the summed |central
// pressure differences| / 2 reach 0.5 min p over the cell's 3^d box and the
// velocity divergence is at most -0.1 min c_s over the box, cells outside the
// domain mapped as the guard fill maps them (the oracle's arithmetic)
__global__ void __launch_bounds__(256) shock_kernel(const double *__restrict__ st, long vs, int ndim, int nx, int ny,
                                                    int nz, UnkGeom g, unsigned char *__restrict__ shok)
{
    const long n = (long)nx * ny * nz;
    auto var = [&](int q, int i, int j, int k) {
        double sx = 1.0, sy = 1.0, sz = 1.0;
        const int mi = map_axis(i, nx, g.bc[0], g.bc[1], &sx);
        const int mj = ndim > 1 ? map_axis(j, ny, g.bc[2], g.bc[3], &sy) : 0;
        const int mk = ndim > 2 ? map_axis(k, nz, g.bc[4], g.bc[5], &sz) : 0;
        double x = st[q * vs + ((long)mk * ny + mj) * nx + mi];
        if (q == VX) x = x * sx;
        if (q == VY) x = x * sy;
        if (q == VZ) x = x * sz;
        return x;
    };
    const int k2 = ndim > 1, k3 = ndim > 2;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx), j = (int)((idx / nx) % ny), k = (int)(idx / ((long)nx * ny));
        double minP = 0., minC = 0.;
        bool first = true;
        for (int kk = k - k3; kk <= k + k3; kk++)
            for (int jj = j - k2; jj <= j + k2; jj++)
                for (int ii = i - 1; ii <= i + 1; ii++) {
                    const double pr = var(P, ii, jj, kk);
                    const double cs = sqrt(var(GC, ii, jj, kk) * var(P, ii, jj, kk) / var(D, ii, jj, kk));
                    if (first || pr < minP) minP = pr;
                    if (first || cs < minC) minC = cs;
                    first = false;
                }
        double divv = var(VX, i + 1, j, k) - var(VX, i - 1, j, k);
        if (ndim > 1) divv = divv + var(VY, i, j + 1, k) - var(VY, i, j - 1, k);
        if (ndim > 2) divv = divv + var(VZ, i, j, k + 1) - var(VZ, i, j, k - 1);
        divv = 0.5 * divv;
        const double gx = 0.5 * (var(P, i + 1, j, k) - var(P, i - 1, j, k));
        double gy = 0., gz = 0.;
        if (ndim > 1) gy = 0.5 * (var(P, i, j + 1, k) - var(P, i, j - 1, k));
        if (ndim > 2) gz = 0.5 * (var(P, i, j, k + 1) - var(P, i, j, k - 1));
        const bool sw1 = fabs(gx) + fabs(gy) + fabs(gz) >= 0.5 * minP;
        const bool sw2 = -0.1 * minC >= divv;
        shok[idx] = (sw1 && sw2) ? 1 : 0;
    }
}

// the flags into UNK slot `slot` of every block cell, guard cells mapped
__global__ void shok_to_unk_kernel(const unsigned char *__restrict__ shok, double *__restrict__ unk, UnkGeom g,
                                   const int *__restrict__ bcoord, int nblk, int slot)
{
    long per = (long)g.nig * g.njg * g.nkg;
    long n = (long)nblk * per;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        int blk = (int)(idx / per);
        long r = idx - blk * per;
        int k = (int)(r / ((long)g.nig * g.njg)); r -= (long)k * g.nig * g.njg;
        int j = (int)(r / g.nig), i = (int)(r - (long)j * g.nig);
        int gj = g.ndim >= 2 ? g.ng : 0, gk = g.ndim == 3 ? g.ng : 0;
        double s_;
        int mx = map_axis(bcoord[3 * blk] * g.nxb + i - g.ng, g.nx, g.bc[0], g.bc[1], &s_);
        int my = g.ndim >= 2 ? map_axis(bcoord[3 * blk + 1] * g.nyb + j - gj + (g.ndim == 2 ? g.soff : 0), g.ny,
                                        g.bc[2], g.bc[3], &s_) : 0;
        int mz = g.ndim == 3 ? map_axis(bcoord[3 * blk + 2] * g.nzb + k - gk + g.soff, g.nz, g.bc[4], g.bc[5], &s_) : 0;
        unk[idx * g.nunk + slot] = (double)shok[((long)mz * g.ny + my) * g.nx + mx];
    }
}

__global__ void unk_to_state_kernel(const double *__restrict__ unk, double *__restrict__ st, UnkGeom g,
                                    const int *__restrict__ bcoord, const int *__restrict__ dmap, int nblk)
{
    long n = (long)nblk * g.nxb * g.nyb * g.nzb;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        long per = (long)g.nxb * g.nyb * g.nzb;
        int blk = (int)(idx / per);
        long r = idx - blk * per;
        int k = (int)(r / ((long)g.nxb * g.nyb)); r -= (long)k * g.nxb * g.nyb;
        int j = (int)(r / g.nxb), i = (int)(r - (long)j * g.nxb);
        int gj = g.ndim >= 2 ? g.ng : 0, gk = g.ndim == 3 ? g.ng : 0;
        long u = ((((long)blk * g.nkg + k + gk) * g.njg + j + gj) * g.nig + i + g.ng) * g.nunk;
        long gx = (long)bcoord[3 * blk] * g.nxb + i;
        long gy = (long)bcoord[3 * blk + 1] * g.nyb + j + (g.ndim == 2 ? g.soff : 0);
        long gz = (long)bcoord[3 * blk + 2] * g.nzb + k + (g.ndim == 3 ? g.soff : 0);
        long c = (gz * g.ny + gy) * g.nx + gx;
        for (int v = 0; v < NV_DEV; v++) st[v * g.vstride + c] = unk[u + dmap[v]];
    }
}

__global__ void state_to_unk_kernel(const double *__restrict__ st, double *__restrict__ unk, UnkGeom g,
                                    const int *__restrict__ bcoord, const int *__restrict__ dmap, int nblk)
{
    long per = (long)g.nig * g.njg * g.nkg;
    long n = (long)nblk * per;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        int blk = (int)(idx / per);
        long r = idx - blk * per;
        int k = (int)(r / ((long)g.nig * g.njg)); r -= (long)k * g.nig * g.njg;
        int j = (int)(r / g.nig), i = (int)(r - (long)j * g.nig);
        int gj = g.ndim >= 2 ? g.ng : 0, gk = g.ndim == 3 ? g.ng : 0;
        double sx = 1.0, sy = 1.0, sz = 1.0;
        int mx = map_axis(bcoord[3 * blk] * g.nxb + i - g.ng, g.nx, g.bc[0], g.bc[1], &sx);
        int my = g.ndim >= 2 ? map_axis(bcoord[3 * blk + 1] * g.nyb + j - gj + (g.ndim == 2 ? g.soff : 0), g.ny,
                                        g.bc[2], g.bc[3], &sy) : 0;
        int mz = g.ndim == 3 ? map_axis(bcoord[3 * blk + 2] * g.nzb + k - gk + g.soff, g.nz, g.bc[4], g.bc[5], &sz) : 0;
        long c = ((long)mz * g.ny + my) * g.nx + mx;
        long u = idx * g.nunk;
        for (int v = 0; v < NV_DEV; v++) {
            if (dmap[v] < 0) continue;          // not selected by a guard-fill mask
            double val = st[v * g.vstride + c];
            if (v == VX) val = val * sx;
            if (v == VY) val = val * sy;
            if (v == VZ) val = val * sz;
            unk[u + dmap[v]] = val;
        }
    }
}

// UNK species slots <-> device mass fractions (interior on the way in; with
// the guard cells, filled by the boundary conditions without sign flips, on
// the way out)
__global__ void unk_to_spec_kernel(const double *__restrict__ unk, double *__restrict__ sp, UnkGeom g,
                                   const int *__restrict__ bcoord, const int *__restrict__ slot, int ns, int nblk)
{
    long n = (long)nblk * g.nxb * g.nyb * g.nzb;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        long per = (long)g.nxb * g.nyb * g.nzb;
        int blk = (int)(idx / per);
        long r = idx - blk * per;
        int k = (int)(r / ((long)g.nxb * g.nyb)); r -= (long)k * g.nxb * g.nyb;
        int j = (int)(r / g.nxb), i = (int)(r - (long)j * g.nxb);
        int gj = g.ndim >= 2 ? g.ng : 0, gk = g.ndim == 3 ? g.ng : 0;
        long u = ((((long)blk * g.nkg + k + gk) * g.njg + j + gj) * g.nig + i + g.ng) * g.nunk;
        long gx = (long)bcoord[3 * blk] * g.nxb + i;
        long gy = (long)bcoord[3 * blk + 1] * g.nyb + j;
        long gz = (long)bcoord[3 * blk + 2] * g.nzb + k;
        long c = (gz * g.ny + gy) * g.nx + gx;
        for (int q = 0; q < ns; q++) sp[q * g.vstride + c] = unk[u + slot[q]];
    }
}

__global__ void spec_to_unk_kernel(const double *__restrict__ sp, double *__restrict__ unk, UnkGeom g,
                                   const int *__restrict__ bcoord, const int *__restrict__ slot, int ns, int nblk)
{
    long per = (long)g.nig * g.njg * g.nkg;
    long n = (long)nblk * per;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        int blk = (int)(idx / per);
        long r = idx - blk * per;
        int k = (int)(r / ((long)g.nig * g.njg)); r -= (long)k * g.nig * g.njg;
        int j = (int)(r / g.nig), i = (int)(r - (long)j * g.nig);
        int gj = g.ndim >= 2 ? g.ng : 0, gk = g.ndim == 3 ? g.ng : 0;
        double s_ = 1.0;
        int mx = map_axis(bcoord[3 * blk] * g.nxb + i - g.ng, g.nx, g.bc[0], g.bc[1], &s_);
        int my = g.ndim >= 2 ? map_axis(bcoord[3 * blk + 1] * g.nyb + j - gj, g.ny, g.bc[2], g.bc[3], &s_) : 0;
        int mz = g.ndim == 3 ? map_axis(bcoord[3 * blk + 2] * g.nzb + k - gk, g.nz, g.bc[4], g.bc[5], &s_) : 0;
        long c = ((long)mz * g.ny + my) * g.nx + mx;
        for (int q = 0; q < ns; q++) unk[idx * g.nunk + slot[q]] = sp[q * g.vstride + c];
    }
}

// Eos_wrapped(MODE_DENS_EI) on every interior cell of the device mirror
__global__ void eos_kernel(double *st, long vstride, long ncell, DevParams prm, double gam1inv, double ggprodinv)
{
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < ncell; c += (long)gridDim.x * blockDim.x) {
        double dens = st[D * vstride + c];
        double vx = st[VX * vstride + c], vy = st[VY * vstride + c], vz = st[VZ * vstride + c];
        double ener = st[DV_ENER * vstride + c], eint = st[EI * vstride + c];
        double ekin = 0.5 * (vx * vx + vy * vy + vz * vz);
        if (ener - ekin > fmax2(prm.small_e, prm.eint_switch * ekin)) eint = ener - ekin;
        double pres = dens * eint * gam1inv;
        st[P * vstride + c] = pres;
        st[DV_TEMP * vstride + c] = eint * ggprodinv * prm.abar;
        st[GC * vstride + c] = prm.gamma;
        st[EI * vstride + c] = eint;
        st[DV_ENER * vstride + c] = eint + ekin;
        st[GE * vstride + c] = pres / (eint * dens) + 1;
    }
}

// Hydro_computeDt.F90:215-225 rate of one cell; the hydro kernels' epilogues
// compute the same expression from the values they store
__device__ __forceinline__ double cell_rate(const double *st, long vstride, long c, int ndim,
                                            double dx, double dy, double dz)
{
    double dens = st[D * vstride + c], pres = st[P * vstride + c], gamc = st[GC * vstride + c];
    double cs = sqrt(gamc * pres / dens);
    double t = (fabs(st[VX * vstride + c] - 0.) + cs) * (1.0 / dx);
    if (ndim > 1) t = fmax2(t, (fabs(st[VY * vstride + c] - 0.) + cs) * (1.0 / dy));
    if (ndim > 2) t = fmax2(t, (fabs(st[VZ * vstride + c] - 0.) + cs) * (1.0 / dz));
    return t;
}

// Hydro_computeDt rate over a state (used when no fused step produced it)
__global__ void rate_kernel(const double *st, long vstride, int nx, int ny, int nz, int ndim,
                            double dx, double dy, double dz, unsigned long long *rate_max)
{
    long ncell = (long)nx * ny * nz;
    double r = 0.;
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < ncell; c += (long)gridDim.x * blockDim.x)
        r = fmax2(r, cell_rate(st, vstride, c, ndim, dx, dy, dz));
    for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, off));
    if ((threadIdx.x & 31) == 0) atomicMax(rate_max, (unsigned long long)__double_as_longlong(r));
}

// the limiting cell: the first (block in list order, then k, j, i) whose rate
// equals the reduced maximum, as Hydro_computeDt's strict '>' scan keeps it
__global__ void locate_kernel(const double *st, long vstride, int nx, int ny, int nz, int ndim, double dx,
                              double dy, double dz, const unsigned long long *rate_max, int nxb, int nyb, int nzb,
                              unsigned long long *key)
{
    const unsigned long long rm = *rate_max;
    const long ncell = (long)nx * ny * nz;
    const int nbx = nx / nxb, nby = ny / nyb;
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < ncell; c += (long)gridDim.x * blockDim.x) {
        double r = cell_rate(st, vstride, c, ndim, dx, dy, dz);
        if ((unsigned long long)__double_as_longlong(r) != rm) continue;
        long gx = c % nx, gy = (c / nx) % ny, gz = c / ((long)nx * ny);
        long b = ((gz / nzb) * nby + gy / nyb) * nbx + gx / nxb;
        unsigned long long k = (unsigned long long)((((b * nzb) + gz % nzb) * nyb + gy % nyb) * nxb + gx % nxb);
        atomicMin(key, k);
    }
}

// Driver_computeDt on the device: dtNew = min(cfl/rate, f*dtOld), clamp.
__global__ void dt_finalize_kernel(double *dtv, unsigned long long *rate_max, double cfl, double f,
                                   double dtmin, double dtmax, int *err)
{
    double r = __longlong_as_double((long long)*rate_max);
    double dtcfl = (r != 0.) ? cfl / r : 1.79769313486231570e308;
    if (!(dtcfl > 0.)) atomicOr(err, 8);
    double dtold = dtv[0];
    double dtnew = fmin2(dtcfl, dtold * f);
    dtnew = fmin2(fmax2(dtnew, dtmin), dtmax);
    dtv[1] = dtold;
    dtv[0] = dtnew;
    *rate_max = 0ull;
}

// volume integrals: per-CTA partial sums in a fixed order (deterministic)
__global__ void integrals_kernel(const double *st, long vstride, long ncell, double dv, double *partials)
{
    double s[7] = {0., 0., 0., 0., 0., 0., 0.};
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < ncell; c += (long)gridDim.x * blockDim.x) {
        double rho = st[D * vstride + c];
        double vx = st[VX * vstride + c], vy = st[VY * vstride + c], vz = st[VZ * vstride + c];
        s[0] += rho * dv; s[1] += rho * vx * dv; s[2] += rho * vy * dv; s[3] += rho * vz * dv;
        s[4] += rho * st[DV_ENER * vstride + c] * dv; s[5] += rho * st[EI * vstride + c] * dv;
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

__global__ void integrals_final_kernel(const double *partials, int n, double *out)
{
    if (threadIdx.x < 7) {
        double t = 0.;
        for (int b = 0; b < n; b++) t += partials[b * 7 + threadIdx.x];
        out[threadIdx.x] = t;
    }
}

UnkGeom unk_geom()
{
    UnkGeom g;
    g.ndim = L.dom.ndim; g.nxb = L.dom.nxb; g.nyb = L.dom.nyb; g.nzb = L.dom.nzb; g.ng = L.dom.nguard;
    g.nig = g.nxb + 2 * g.ng;
    g.njg = g.ndim >= 2 ? g.nyb + 2 * g.ng : 1;
    g.nkg = g.ndim == 3 ? g.nzb + 2 * g.ng : 1;
    g.nunk = L.nunk;
    g.nx = L.nx; g.ny = L.ny; g.nz = L.nz;
    for (int i = 0; i < 6; i++) g.bc[i] = L.kbc[i];
    g.vstride = L.vstride;
    const int nb = L.dom.ndim == 3 ? L.dom.nzb : L.dom.nyb;
    g.soff = L.slab.halo_lo - L.slab.layer_lo * nb;
    return g;
}

double cell_dx(int a)
{
    if (a >= L.dom.ndim) return 1.0;
    return (L.dom.bbox[a][1] - L.dom.bbox[a][0]) / (double)L.gext[a];
}

// the slab's own cells: first stored cell and extents (the slowest axis
// without its halos)
const double *interior(int buf) { return L.buf[buf] + (long)L.slab.halo_lo * L.plane; }
int int_ny() { return L.dom.ndim == 2 ? L.nint : L.ny; }
int int_nz() { return L.dom.ndim == 3 ? L.nint : 1; }
bool has_halo() { return L.slab.halo_lo > 0 || L.slab.halo_hi > 0; }


// tensor map of the 2-D kernel's window: the first 8 device variables of a
// state buffer as a [var][y][x] FP64 tensor (rows of nx, variables vstride
// apart), boxes of 8 x 22 x 24 (cuTensorMapEncodeTiled, reached through the
// runtime's driver entry point so the library needs no link to libcuda)
int encode_window_map(CUtensorMap *m, const double *base)
{
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return fail(FXB_ECUDA, "fxb_init: cuTensorMapEncodeTiled not available from the driver");
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)L.nx, (cuuint64_t)L.ny, 8};
    const cuuint64_t strides[2] = {(cuuint64_t)L.nx * sizeof(double), (cuuint64_t)L.vstride * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)WP, (cuuint32_t)WIN, 8};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(FXB_ECUDA, "fxb_init: cuTensorMapEncodeTiled rejected the window map");
    return FXB_OK;
}

int launch_species(int src, const double *dtv, double dt);

// launch one fused hydro step reading buffer `src`, writing 1-src
int launch_hydro(int src, const double *dtv, double dt)
{
    if (L.shok) {   // levelFlux/Hydro.F90:133-149: the flags of the step's initial state
        UnkGeom g = unk_geom();
        shock_kernel<<<148 * 8, 256, 0, L.stream>>>(L.buf[src], L.vstride, L.dom.ndim, L.nx, L.ny, L.nz, g, L.shok);
        L.shok_valid = true;
    }
    if (L.dom.ndim == 2) {
        Args2D a;
        a.in = L.buf[src]; a.out = L.buf[1 - src]; a.vstride = L.vstride;
        a.nx = L.nx; a.ny = L.ny;
        for (int i = 0; i < 4; i++) a.bc[i] = L.kbc[i];
        a.rate_c0 = (long)L.slab.halo_lo * L.plane;
        a.rate_c1 = a.rate_c0 + (long)L.nint * L.plane;
        a.dx = cell_dx(0); a.dy = cell_dx(1);
        a.dt_arg = dt; a.dtv = dtv;
        a.gam1inv = L.gam1inv; a.ggprodinv = L.ggprodinv;
        a.prm = L.dprm; a.rate_max = L.rate_max; a.err = L.err;
        a.flat = L.flat;
        a.tmap = L.tmap2d[src];
        a.fd[0] = L.sfd[0]; a.fd[1] = L.sfd[1];
        a.shok = L.shok;
        a.use_tma = L.use_tma;
        a.tma_extra_tx = L.tma_extra_tx;
        a.wait_budget = L.wait_budget;
        dim3 grid(L.nx / T2, L.ny / T2);
        if (L.prm.precision == FXB_MIXED) launch_hydro2d_mixed(a, grid, L.stream);
        else launch_hydro2d_fp64(a, grid, L.stream);
    } else {
        Args3D a;
        a.in = L.buf[src]; a.out = L.buf[1 - src]; a.vstride = L.vstride;
        a.nx = L.nx; a.ny = L.ny; a.nz = L.nz;
        for (int i = 0; i < 6; i++) a.bc[i] = L.kbc[i];
        a.rate_c0 = (long)L.slab.halo_lo * L.plane;
        a.rate_c1 = a.rate_c0 + (long)L.nint * L.plane;
        a.dx = cell_dx(0); a.dy = cell_dx(1); a.dz = cell_dx(2);
        a.dt_arg = dt; a.dtv = dtv;
        a.gam1inv = L.gam1inv; a.ggprodinv = L.ggprodinv;
        a.prm = L.dprm; a.rate_max = L.rate_max; a.err = L.err;
        a.sig = L.sig3;
        a.slp = L.slp3;
        a.slp_bstride = 0;
        a.flat = L.flat;
        a.flat_bstride = 0;
        a.hyb = (const unsigned char *)L.hyb;
        for (int d = 0; d < 3; d++) { a.wst[d] = L.w3[d]; a.flx[d] = L.f3[d]; a.ctufb[d] = L.ctufb[d]; }
        for (int q = 0; q < 4; q++) a.cta[q] = 148 * L.ug_cta[q];
        a.shok = L.shok;
        for (int d = 0; d < 3; d++) a.sf_t1[d] = L.sf_t1[d];
        for (int d = 0; d < 3 && L.ns; d++)
            if (cudaMemsetAsync(L.ctufb[d], 0, L.snw, L.stream) != cudaSuccess) return cuda_fail(cudaGetLastError(), "memset");
        if (L.prm.precision == FXB_MIXED) launch_hydro3d_mixed(a, L.stream);
        else launch_hydro3d_fp64(a, L.stream);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "hydro kernel launch");
    if (L.ns) return launch_species(src, dtv, dt);
    return FXB_OK;
}

// species after the hydro step that read buffer `src` and wrote 1-src
int launch_species(int src, const double *dtv, double dt)
{
    SpecArgs s;
    memset((void *)&s, 0, sizeof(s));
    s.st_old = L.buf[src]; s.st_new = L.buf[1 - src]; s.vstride = L.vstride;
    s.sp_in = L.spb[src]; s.sp_out = L.spb[1 - src];
    s.ns = L.ns; s.nsp = L.nsp;
    s.ndim = L.dom.ndim; s.nx = L.nx; s.ny = L.ny; s.nz = L.nz;
    for (int i = 0; i < 6; i++) s.bc[i] = L.kbc[i];
    s.dx = cell_dx(0); s.dy = cell_dx(1); s.dz = cell_dx(2);
    s.dt_arg = dt; s.dtv = dtv;
    s.prm = L.dprm;
    if (L.dom.ndim == 2) {
        s.fd[0] = L.sfd[0]; s.fd[1] = L.sfd[1];
    } else {
        for (int d = 0; d < 3; d++) { s.fd[d] = L.f3[d]; s.ctufb[d] = L.ctufb[d]; }
    }
    s.flat = L.flat;
    s.sg = L.ssg; s.sl = L.ssl; s.sr = L.ssr;
    s.npad = L.snpad; s.nwmax = L.snw;
    if (L.prm.precision == FXB_MIXED) launch_species_mixed(s, L.stream);
    else launch_species_fp64(s, L.stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "species kernel launch");
    return FXB_OK;
}

// kernels of one 3-D step: sigma, per direction the slopes, face states and
// fluxes (one fused kernel in FP32; slopes (PPM), face states and fluxes as
// separate kernels in FP64), the update
int hydro3d_launches(const fxb_params &p)
{
    const int per_dir = p.precision == FXB_MIXED ? 1 : (p.order == 3 ? 3 : 2);
    return 1 + 3 * per_dir + 1;
}
// launches of one uniform-grid step (flattening and species add kernels)
int ug_step_launches()
{
    return (L.dom.ndim == 2 ? 1 : hydro3d_launches(L.prm)) + (L.prm.flattening ? 1 : 0) + (L.ns ? 3 : 0);
}

int check_err_word()
{
    int h = 0;
    CK(cudaMemcpyAsync(&h, L.err, sizeof(int), cudaMemcpyDeviceToHost, L.stream));
    CK(cudaStreamSynchronize(L.stream));
    if (h) {
        CK(cudaMemsetAsync(L.err, 0, sizeof(int), L.stream));
        if (h & ERR_SOUND)
            return fail(FXB_ESOUND, "[hy_eigenParameters]: Zero or imaginary sound speed has obtained!");
        if (h & ERR_RIEMANN) return fail(FXB_ERIEMANN, "[hy_getFaceFlux]: Riemann solver returned ierr /= 0");
        if (h & 8) return fail(FXB_EDT, "[Hydro]: Computed dt is not positive! Aborting!");
        if (h & 16) return fail(FXB_EARG, "[Grid_fillGuardCells]: AMR guard cell without a covering block");
        if (h & ERR_TIMEOUT) return fail(FXB_ETIMEOUT, "[Hydro]: a bounded device wait ran out (data never arrived)");
        return fail(FXB_ECUDA, "device error word set");
    }
    return FXB_OK;
}

void free_all()
{
    amr_destroy();
    for (int i = 0; i < 2; i++) {
        if (L.graph_exec[i]) cudaGraphExecDestroy(L.graph_exec[i]);
        L.graph_exec[i] = nullptr;
        if (L.buf[i]) cudaFree(L.buf[i]);
        L.buf[i] = nullptr;
    }
    if (L.unk_dev) cudaFree(L.unk_dev);
    if (L.bcoord) cudaFree(L.bcoord);
    if (L.dmap_dev) cudaFree(L.dmap_dev);
    if (L.sslot_dev) cudaFree(L.sslot_dev);
    for (int i = 0; i < 2; i++) {
        if (L.spb[i]) cudaFree(L.spb[i]);
        if (L.sfd[i]) cudaFree(L.sfd[i]);
    }
    if (L.ssg) cudaFree(L.ssg);
    if (L.ssl) cudaFree(L.ssl);
    if (L.ssr) cudaFree(L.ssr);
    for (int d = 0; d < 3; d++)
        if (L.ctufb[d]) cudaFree(L.ctufb[d]);
    if (L.pmap_dev) cudaFree(L.pmap_dev);
    if (L.pack_dev) cudaFree(L.pack_dev);
    if (L.pack_host) cudaFreeHost(L.pack_host);
    if (L.dtv) cudaFree(L.dtv);
    if (L.shok) cudaFree(L.shok);
    if (L.rate_max) cudaFree(L.rate_max);
    if (L.err) cudaFree(L.err);
    if (L.partials) cudaFree(L.partials);
    if (L.sig3) cudaFree(L.sig3);
    if (L.slp3) cudaFree(L.slp3);
    if (L.flat) cudaFree(L.flat);
    if (L.hyb) cudaFree(L.hyb);
    for (int d = 0; d < 3; d++) {
        if (L.w3[d]) cudaFree(L.w3[d]);
        if (L.f3[d]) cudaFree(L.f3[d]);
    }
    if (L.mapped_registered) cudaHostUnregister(const_cast<void *>(L.mapped_host));
    if (L.ev0) cudaEventDestroy(L.ev0);
    if (L.ev1) cudaEventDestroy(L.ev1);
    if (L.stream) cudaStreamDestroy(L.stream);
    fxb_error keep = L.lasterr;
    L = Lib();
    L.lasterr = keep;
}

} // namespace

namespace fxb {
// lets other translation units of the library report through fxb_last_error
int record_error(int code, const char *msg) { return fail(code, msg); }
} // namespace fxb

// ====================================================================== ABI
extern "C" int fxb_init(const fxb_params *params, const fxb_domain *domain, const int32_t *var_map, int nunk)
{
    return fxb_init_slab(params, domain, var_map, nunk, nullptr);
}

extern "C" int fxb_init_slab(const fxb_params *params, const fxb_domain *domain, const int32_t *var_map, int nunk,
                             const fxb_slab *slab)
{
    if (!params || !domain || !var_map) return fail(FXB_EARG, "fxb_init: null argument");
    if (L.inited) free_all();
    const fxb_domain &d = *domain;
    const fxb_params &p = *params;
    if (d.ndim != 2 && d.ndim != 3) return fail(FXB_EUNSUPPORTED, "fxb_init: ndim must be 2 or 3");
    if (d.nguard < 4) return fail(FXB_EARG, "fxb_init: NGUARD must be at least 4");
    if (p.order != 2 && p.order != 3 && p.order != 5)
        return fail(FXB_EUNSUPPORTED, "fxb_init: order must be 2 (MUSCL-Hancock), 3 (PPM) or 5 (WENO)");
    if (p.riemann < 1 || p.riemann > 8 || p.riemann == 6)
        return fail(FXB_EUNSUPPORTED,
                    "fxb_init: RiemannSolver must be Roe, LLF, HLL, HLLC, Marquina, MarquinaModified or hybrid");
    if (p.shock_slot >= nunk) return fail(FXB_EARG, "fxb_init: shock_slot outside UNK");
    if (p.limiter < 1 || p.limiter > 5) return fail(FXB_EARG, "fxb_init: unknown slope limiter");
    if (p.precision != FXB_FP64 && p.precision != FXB_MIXED) return fail(FXB_EARG, "fxb_init: unknown precision");
    if (p.flattening && p.use_gravity) return fail(FXB_EUNSUPPORTED, "fxb_init: use_flattening with gravity is not implemented");
    if (p.entropy_fix < 0 || p.entropy_fix > 2) return fail(FXB_EARG, "fxb_init: unknown entropyFixMethod");
    // unsplit/Hydro_init.F90:137: use_upwindTVD only acts with more than four guard cells
    if (p.upwind_tvd && d.nguard > 4)
        return fail(FXB_EUNSUPPORTED, "fxb_init: use_upwindTVD with NGUARD > 4 is not implemented");
    for (int i = 0; i < 2 * d.ndim; i++)
        if (d.bc[i] < 0 || d.bc[i] > 2) return fail(FXB_EARG, "fxb_init: unknown boundary condition");
    for (int a = 0; a < d.ndim; a++) {
        bool per_lo = d.bc[2 * a] == FXB_BC_PERIODIC, per_hi = d.bc[2 * a + 1] == FXB_BC_PERIODIC;
        if (per_lo != per_hi) return fail(FXB_EARG, "fxb_init: periodic boundaries must be paired");
    }
    if (nunk < FXB_NVAR) return fail(FXB_EARG, "fxb_init: nunk too small");
    for (int v = 0; v < FXB_NVAR; v++)
        if (var_map[v] < 0 || var_map[v] >= nunk) return fail(FXB_EARG, "fxb_init: var_map out of range");
    // the slab: layers of the slowest axis and halo planes (UG/Grid_fillGuardCells.F90:261-306)
    const int sa = d.ndim - 1;                                   // split axis
    const int nlay = sa == 1 ? d.nblocky : d.nblockz;            // block layers of the whole grid
    const int nbs = sa == 1 ? d.nyb : d.nzb;                     // cells per block along it
    fxb_slab sl = slab ? *slab : fxb_slab{0, nlay, 0, 0};
    if (sl.layer_lo < 0 || sl.layer_hi > nlay || sl.layer_lo >= sl.layer_hi)
        return fail(FXB_EARG, "fxb_init_slab: layer range outside the grid");
    const int nint = (sl.layer_hi - sl.layer_lo) * nbs;
    const bool periodic_s = d.bc[2 * sa] == FXB_BC_PERIODIC;
    for (int side = 0; side < 2; side++) {
        const int h = side ? sl.halo_hi : sl.halo_lo;
        const bool edge = side ? sl.layer_hi == nlay : sl.layer_lo == 0;
        if (h < 0 || h > nint || (h > 0 && h < d.nguard))
            return fail(FXB_EARG, "fxb_init_slab: a halo must be 0 or between NGUARD and the slab's own planes");
        if (!edge && h == 0) return fail(FXB_EARG, "fxb_init_slab: a side facing another slab needs a halo");
        if (edge && h > 0 && !periodic_s)
            return fail(FXB_EARG, "fxb_init_slab: a halo on a non-periodic domain boundary");
    }
    L.prm = p;
    L.dom = d;
    L.nunk = nunk;
    L.slab = sl;
    L.nint = nint;
    for (int v = 0; v < NV_DEV; v++) L.dmap[v] = var_map[kDevToVar[v]];
    for (int i = 0; i < 6; i++) L.kbc[i] = d.bc[i];
    if (sl.halo_lo > 0) L.kbc[2 * sa] = FXB_BC_OUTFLOW;       // cells beyond a halo only feed halo cells
    if (sl.halo_hi > 0) L.kbc[2 * sa + 1] = FXB_BC_OUTFLOW;
    L.gext[0] = d.nxb * d.nblockx;
    L.gext[1] = d.ndim >= 2 ? d.nyb * d.nblocky : 1;
    L.gext[2] = d.ndim == 3 ? d.nzb * d.nblockz : 1;
    L.nx = L.gext[0];
    L.ny = sa == 1 ? nint + sl.halo_lo + sl.halo_hi : L.gext[1];
    L.nz = sa == 2 ? nint + sl.halo_lo + sl.halo_hi : 1;
    L.plane = sa == 1 ? (long)L.nx : (long)L.nx * L.ny;
    if (d.ndim == 2 && (L.nx % T2 || L.ny % T2))
        return fail(FXB_EUNSUPPORTED, "fxb_init: 2-D grid extents (a slab's with its halos) must be multiples of 16");
    if (d.ndim == 3 && (L.nx % T3X || L.ny % T3Y || L.nz % T3Z))
        return fail(FXB_EUNSUPPORTED, "fxb_init: 3-D grid extents must be multiples of the 3-D tile");
    // the 3-D kernels walk padded boxes with 32-bit indices
    if (d.ndim == 3 && (long)(L.nx + 4) * (L.ny + 4) * (L.nz + 4) >= (1L << 30))
        return fail(FXB_EUNSUPPORTED, "fxb_init: 3-D grid larger than 2^30 cells");
    L.ncell = (long)L.nx * L.ny * L.nz;
    L.vstride = (L.ncell + 31) / 32 * 32;
    L.nblk = d.nblockx * (d.ndim == 3 ? d.nblocky : 1) * (sl.layer_hi - sl.layer_lo);
    long per = (long)(d.nxb + 2 * d.nguard) * (d.ndim >= 2 ? d.nyb + 2 * d.nguard : 1) *
               (d.ndim == 3 ? d.nzb + 2 * d.nguard : 1);
    L.unk_doubles = per * L.nblk * nunk;
    DevParams &q = L.dprm;
    q.order = p.order; q.weno_method = p.weno_method; q.riemann = p.riemann; q.limiter = p.limiter;
    q.char_limiting = p.char_limiting; q.use_3d_full_ctu = p.use_3d_full_ctu; q.use_aux_eint = p.use_aux_eint;
    q.use_gravity = p.use_gravity;
    for (int i = 0; i < 3; i++) q.grav[i] = p.grav[i];
    q.cfl = p.cfl; q.gamma = p.gamma; q.eint_switch = p.eint_switch; q.small_dens = p.small_dens;
    q.small_e = p.small_e; q.small_p = p.small_p; q.tiny = p.tiny; q.fpres = p.fpres;
    q.limited_beta = p.limited_beta; q.gas_constant = p.gas_constant; q.abar = p.abar;
    q.flattening = p.flattening ? 1 : 0;
    q.entropy_fix = p.entropy_fix;
    q.steepening = p.steepening ? 1 : 0;
    q.use_avisc = p.use_avisc ? 1 : 0;
    q.cvisc = p.cvisc;
    q.use_hybrid = p.hybrid_order ? 1 : 0;
    q.hybrid_kappa = p.hybrid_kappa;
    // Hydro_init.F90:391-394: the hybrid solver turns the shock detector on
    q.shock_detect = (p.shock_detect || p.riemann == 8) ? 1 : 0;
    L.shock_slot = p.shock_slot;
    // Gamma/Eos_init.F90:86 and Gamma/Eos.F90:177,240-241
    double gammam1 = 1.0 / (p.gamma - 1.0);
    L.gam1inv = 1. / gammam1;
    L.ggprodinv = 1. / (gammam1 * p.gas_constant);

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(FXB_ECUDA, "fxb_init: no CUDA device visible");
    }
    // FXB_TEST_WAIT_TIMEOUT=1 (tests only): window barriers expect 8 bytes
    // more than the box brings, so their bounded waits run out after ~0.5 ms
    const char *tw = getenv("FXB_TEST_WAIT_TIMEOUT");
    if (tw && tw[0] == '1') { L.tma_extra_tx = 8; L.wait_budget = 1000000; }
    CK(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&L.ev0));
    CK(cudaEventCreate(&L.ev1));
    for (int i = 0; i < 2; i++) {
        CK(cudaMalloc(&L.buf[i], sizeof(double) * L.vstride * NV_DEV));
        CK(cudaMemsetAsync(L.buf[i], 0, sizeof(double) * L.vstride * NV_DEV, L.stream));
    }
    CK(cudaMalloc(&L.unk_dev, sizeof(double) * L.unk_doubles));
    CK(cudaMalloc(&L.dmap_dev, sizeof(int) * NV_DEV));
    CK(cudaMalloc(&L.pmap_dev, sizeof(int) * NV_DEV));
    CK(cudaMemcpyAsync(L.dmap_dev, L.dmap, sizeof(int) * NV_DEV, cudaMemcpyHostToDevice, L.stream));
    CK(cudaMalloc(&L.dtv, 2 * sizeof(double)));
    if (L.dprm.shock_detect) {
        CK(cudaMalloc(&L.shok, (size_t)L.vstride));
        CK(cudaMemsetAsync(L.shok, 0, (size_t)L.vstride, L.stream));
    }
    CK(cudaMalloc(&L.rate_max, sizeof(unsigned long long)));
    CK(cudaMalloc(&L.err, sizeof(int)));
    CK(cudaMemsetAsync(L.err, 0, sizeof(int), L.stream));
    CK(cudaMemsetAsync(L.rate_max, 0, sizeof(unsigned long long), L.stream));
    L.npartials = 1024;
    CK(cudaMalloc(&L.partials, sizeof(double) * (L.npartials * 7 + 8)));
    if (q.use_gravity) {   // gravity's face values, once, in each precision's kernels' arithmetic
        launch_gravity_faces_fp64(q, L.partials, L.stream);
        launch_gravity_faces_mixed(q, L.partials + 6, L.stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&q.gface[0][0], L.partials, sizeof(q.gface), cudaMemcpyDeviceToHost, L.stream));
        CK(cudaMemcpyAsync(&q.gfacef[0][0], L.partials + 6, sizeof(q.gfacef), cudaMemcpyDeviceToHost, L.stream));
        CK(cudaStreamSynchronize(L.stream));
    }
    if (p.flattening) {
        size_t rsz0 = p.precision == FXB_MIXED ? sizeof(float) : sizeof(double);
        size_t npad = (size_t)(L.nx + 2) * (L.ny + 2) * (d.ndim == 3 ? L.nz + 2 : 1);
        CK(cudaMalloc(&L.flat, rsz0 * d.ndim * npad));
    }
    if (d.ndim == 2) {
        CK(setup_hydro2d_fp64());
        CK(setup_hydro2d_mixed());
        for (int i = 0; i < 2; i++) {
            int rc = encode_window_map(&L.tmap2d[i], L.buf[i]);
            if (rc) return rc;
        }
        // FXB_TMA=0 stages every window with per-thread loads (for comparisons)
        const char *tv = getenv("FXB_TMA");
        L.use_tma = !(tv && tv[0] == '0');
    } else {
        CK(setup_hydro3d_fp64());
        CK(setup_hydro3d_mixed());
        // intermediates of the unfused 3-D pipeline, in the reconstruction type
        size_t rsz = p.precision == FXB_MIXED ? sizeof(float) : sizeof(double);
        CK(cudaMalloc(&L.sig3, sig3d_bytes(L.nx, L.ny, L.nz, rsz)));
        if (p.hybrid_order) CK(cudaMalloc(&L.hyb, hyb3d_bytes(L.nx, L.ny, L.nz, rsz)));
        // PPM slopes in memory: FP64 only (the FP32 face-state kernel computes them itself)
        if (p.order == 3 && p.precision == FXB_FP64) CK(cudaMalloc(&L.slp3, slp3d_bytes(L.nx, L.ny, L.nz, rsz)));
        for (int dd = 0; dd < 3; dd++) {
            CK(cudaMalloc(&L.w3[dd], w3d_bytes(dd, L.nx, L.ny, L.nz, rsz)));
            CK(cudaMalloc(&L.f3[dd], f3d_bytes(dd, L.nx, L.ny, L.nz, rsz)));
        }
    }
    CK(cudaStreamSynchronize(L.stream));
    L.inited = true;
    return FXB_OK;
}

extern "C" int fxb_init_species(int nspec, int nspecies, const int32_t *unk_slots)
{
    if (!L.inited) return fail(FXB_EARG, "fxb_init_species: call fxb_init first");
    if (nspec < 1 || nspec > FXB_MAX_SPECIES || nspecies < 0 || nspecies > nspec || !unk_slots)
        return fail(FXB_EARG, "fxb_init_species: need 1..FXB_MAX_SPECIES values, at most nspec species, and their slots");
    if (L.ns) return fail(FXB_EARG, "fxb_init_species: species are already set");
    if (amr_active()) return fail(FXB_EUNSUPPORTED, "fxb_init_species: species on AMR meshes are not implemented");
    if (has_halo()) return fail(FXB_EUNSUPPORTED, "fxb_init_species: species on a slab with halos are not implemented");
    for (int q = 0; q < nspec; q++) {
        if (unk_slots[q] < 0 || unk_slots[q] >= L.nunk) return fail(FXB_EARG, "fxb_init_species: slot out of range");
        for (int v = 0; v < NV_DEV; v++)
            if (unk_slots[q] == L.dmap[v]) return fail(FXB_EARG, "fxb_init_species: slot of a hydro variable");
        for (int r = 0; r < q; r++)
            if (unk_slots[r] == unk_slots[q]) return fail(FXB_EARG, "fxb_init_species: duplicate slot");
    }
    const bool mixed = L.prm.precision == FXB_MIXED;
    const size_t rsz = mixed ? sizeof(float) : sizeof(double);
    const int nd = L.dom.ndim;
    L.snpad = (long)(L.nx + 2) * (L.ny + 2) * (nd == 3 ? L.nz + 2 : 1);
    const long nz = nd == 3 ? L.nz : 1;
    L.snw = std::max((long)(L.nx + 2) * L.ny * nz, (long)L.nx * (L.ny + 2) * nz);
    if (nd == 3) L.snw = std::max(L.snw, (long)L.nx * L.ny * (L.nz + 2));
    for (int i = 0; i < 2; i++) {
        CK(cudaMalloc(&L.spb[i], sizeof(double) * L.vstride * nspec));
        CK(cudaMemsetAsync(L.spb[i], 0, sizeof(double) * L.vstride * nspec, L.stream));
    }
    CK(cudaMalloc(&L.ssg, rsz * 3 * nspec * L.snpad));
    CK(cudaMalloc(&L.ssl, rsz * 3 * nspec * L.snw));
    CK(cudaMalloc(&L.ssr, rsz * 3 * nspec * L.snw));
    if (nd == 2) {
        CK(cudaMalloc(&L.sfd[0], rsz * (size_t)(L.nx + 1) * L.ny));
        CK(cudaMalloc(&L.sfd[1], rsz * (size_t)L.nx * (L.ny + 1)));
    } else {
        for (int d = 0; d < 3; d++) CK(cudaMalloc(&L.ctufb[d], (size_t)L.snw));
    }
    CK(cudaMalloc(&L.sslot_dev, sizeof(int) * nspec));
    for (int q = 0; q < nspec; q++) L.sslot[q] = unk_slots[q];
    CK(cudaMemcpyAsync(L.sslot_dev, L.sslot, sizeof(int) * nspec, cudaMemcpyHostToDevice, L.stream));
    CK(cudaStreamSynchronize(L.stream));
    L.ns = nspec;
    L.nsp = nspecies;
    L.dprm.nspec = nspec;          // the step runs the extended-option kernels, which export what species read
    for (int i = 0; i < 2; i++) {
        if (L.graph_exec[i]) cudaGraphExecDestroy(L.graph_exec[i]);
        L.graph_exec[i] = nullptr;
    }
    return FXB_OK;
}

extern "C" int fxb_register_blocks(const fxb_block_desc *blocks, int nblk)
{
    if (!L.inited) return fail(FXB_EARG, "fxb_register_blocks: call fxb_init first");
    if (!blocks || nblk <= 0) return fail(FXB_EARG, "fxb_register_blocks: empty block list");
    bool refined = nblk != L.nblk;
    for (int b = 0; b < nblk && !refined; b++) refined = blocks[b].level != 1;
    L.attached = false;
    state_changed(false);
    for (int i = 0; i < 2; i++) {
        if (L.graph_exec[i]) cudaGraphExecDestroy(L.graph_exec[i]);
        L.graph_exec[i] = nullptr;
    }
    if (refined) {
        if (L.ns) return fail(FXB_EUNSUPPORTED, "fxb_register_blocks: species on AMR meshes are not implemented");
        const int nlay = L.dom.ndim == 3 ? L.dom.nblockz : L.dom.nblocky;
        if (has_halo() || L.slab.layer_lo != 0 || L.slab.layer_hi != nlay)
            return fail(FXB_EUNSUPPORTED, "fxb_register_blocks: a slab of a grid takes its level-1 blocks only");
        // block-structured AMR mesh: parents derived, leaves keep their UNK slots
        AmrCommon c;
        c.stream = L.stream; c.prm = L.prm; c.dom = L.dom; c.dprm = L.dprm; c.nunk = L.nunk;
        for (int v = 0; v < NV_DEV; v++) c.dmap[v] = L.dmap[v];
        c.err = L.err; c.rate_max = L.rate_max; c.dtv = L.dtv;
        c.gam1inv = L.gam1inv; c.ggprodinv = L.ggprodinv;
        return amr_create(c, blocks, nblk);
    }
    amr_destroy();
    // block coordinates stay those of the whole grid; a slab holds layers [lo, hi) of its slowest axis
    const int sa = L.dom.ndim - 1;
    int lo[3] = {0, 0, 0};
    int nb[3] = {L.dom.nblockx, L.dom.ndim >= 2 ? L.dom.nblocky : 1, L.dom.ndim == 3 ? L.dom.nblockz : 1};
    lo[sa] = L.slab.layer_lo;
    nb[sa] = L.slab.layer_hi - L.slab.layer_lo;
    int *h = new int[3 * nblk];
    char *seen = new char[nblk]();
    for (int b = 0; b < nblk; b++) {
        for (int a = 0; a < 3; a++) {
            int c = blocks[b].bcoord[a];
            if (a >= L.dom.ndim) c = 0;
            if (c < lo[a] || c >= lo[a] + nb[a]) { delete[] h; delete[] seen; return fail(FXB_EARG, "fxb_register_blocks: block coordinate out of range"); }
            h[3 * b + a] = c;
        }
        long lin = ((long)(h[3 * b + 2] - lo[2]) * nb[1] + h[3 * b + 1] - lo[1]) * nb[0] + h[3 * b] - lo[0];
        if (seen[lin]) { delete[] h; delete[] seen; return fail(FXB_EARG, "fxb_register_blocks: duplicate block"); }
        seen[lin] = 1;
        if (blocks[b].level != 1) { delete[] h; delete[] seen; return fail(FXB_EUNSUPPORTED, "fxb_register_blocks: only level-1 (uniform) block lists"); }
    }
    delete[] seen;
    if (!L.bcoord) {
        cudaError_t e = cudaMalloc(&L.bcoord, sizeof(int) * 3 * nblk);
        if (e != cudaSuccess) { delete[] h; return cuda_fail(e, "cudaMalloc bcoord"); }
    }
    cudaError_t e = cudaMemcpy(L.bcoord, h, sizeof(int) * 3 * nblk, cudaMemcpyHostToDevice);
    delete[] h;
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy bcoord");
    return FXB_OK;
}

// one step from the current state with dt = 0 (the state is not switched):
// the fastest of `reps` runs, in ms
static int time_ug_step(float &best, int reps)
{
    best = 1e30f;
    for (int r = 0; r < reps; r++) {
        CK(cudaEventRecord(L.ev0, L.stream));
        int rc = launch_hydro(L.cur, nullptr, 0.0);
        if (rc) return rc;
        CK(cudaEventRecord(L.ev1, L.stream));
        CK(cudaEventSynchronize(L.ev1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, L.ev0, L.ev1));
        best = ms < best ? ms : best;
    }
    return FXB_OK;
}

// The uniform grid's launch shapes, timed over whole steps on the attached
// state at the first attach: 2-D window staging by TMA or by per-thread
// loads; 3-D CTAs per SM of each stage (2, 4, 8, 16), one stage at a time,
// and in FP32 the lines per fused face-state tile of each direction.  A
// candidate replaces the current choice when it is more than 1 % faster.
// FXB_UG_TUNE=0 keeps the defaults; FXB_TMA=0/1 fixes the 2-D staging.  The
// timed steps leave no trace: the CFL rate and the error word are cleared.
static int ug_tune()
{
    const char *ev = getenv("FXB_UG_TUNE");
    const bool off = ev && ev[0] == '0';
    float base = 0.f;
    int rc = FXB_OK;
    if (!off) {
        // warm-up: about 50 ms of steps (clocks up from idle), then the defaults
        float spent = 0.f;
        for (int w = 0; w < 64 && spent < 50.f && !rc; w++) {
            rc = time_ug_step(base, 1);
            spent += base;
        }
        if (!rc) rc = time_ug_step(base, 3);
        if (rc) return rc;
    }
    if (L.dom.ndim == 2) {
        float t[2] = {-1.f, -1.f};
        if (!off && !getenv("FXB_TMA") && !L.tma_extra_tx) {
            const int keep = L.use_tma;
            t[keep] = base;
            L.use_tma = 1 - keep;
            rc = time_ug_step(t[1 - keep], 3);
            if (rc) return rc;
            L.use_tma = t[1 - keep] < 0.99f * t[keep] ? 1 - keep : keep;
        }
        snprintf(L.ug_log, sizeof(L.ug_log), "uniform grid 2-D: one CTA of 320 threads per 16x16 tile; window "
                 "staging: %s (ms per step: TMA %.3f, per-thread loads %.3f%s)", L.use_tma ? "TMA" : "per-thread loads",
                 t[1], t[0], off ? ", tuning off" : "");
    } else {
        const bool fused = L.prm.precision == FXB_MIXED;
        float cur = base;
        // FXB_UG_CTA="s,f,x,u" and FXB_UG_T1="x,y,z" fix the shapes instead
        const char *ec = getenv("FXB_UG_CTA"), *et = getenv("FXB_UG_T1");
        if (ec) {
            int v[4];
            if (sscanf(ec, "%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3]) != 4)
                return fail(FXB_EARG, "FXB_UG_CTA: four CTA counts per SM expected");
            for (int q = 0; q < 4; q++) L.ug_cta[q] = v[q] < 1 ? 1 : v[q] > 32 ? 32 : v[q];
        }
        if (et) {
            int v[3];
            if (sscanf(et, "%d,%d,%d", &v[0], &v[1], &v[2]) != 3)
                return fail(FXB_EARG, "FXB_UG_T1: three line counts expected");
            for (int d = 0; d < 3; d++) L.sf_t1[d] = v[d] < 0 ? 0 : v[d];
        }
        if (!off && !ec && !et) {
            const int cand[4] = {2, 4, 8, 16};
            for (int q = 0; q < 4; q++) {
                if (fused && (q == 1 || q == 2)) continue;     // the fused kernel's grid follows its tiles
                int keep = L.ug_cta[q];
                for (int c : cand) {
                    if (c == keep) continue;
                    L.ug_cta[q] = c;
                    float t = 0.f;
                    rc = time_ug_step(t, 3);
                    if (rc) return rc;
                    if (t < 0.99f * cur) { cur = t; keep = c; }
                    L.ug_cta[q] = keep;
                }
            }
            if (fused)
                for (int d = 0; d < 3; d++) {
                    int keep = L.sf_t1[d];
                    for (int t1 : {1, 2, 4, 8, 16}) {
                        L.sf_t1[d] = t1;
                        float t = 0.f;
                        rc = time_ug_step(t, 3);
                        if (rc) return rc;
                        if (t < 0.99f * cur) { cur = t; keep = t1; }
                        L.sf_t1[d] = keep;
                    }
                }
        }
        char tiles[96] = "";
        if (fused) snprintf(tiles, sizeof(tiles), "; face-state tile lines x/y/z: %d/%d/%d (0: by lane count)",
                            L.sf_t1[0], L.sf_t1[1], L.sf_t1[2]);
        snprintf(L.ug_log, sizeof(L.ug_log), "uniform grid 3-D: CTAs of 256 threads per SM: sigma %d, face states %d, "
                 "fluxes %d, update %d%s (ms per step: defaults %.3f, tuned %.3f%s)", L.ug_cta[0], L.ug_cta[1],
                 L.ug_cta[2], L.ug_cta[3], tiles, base, cur, off ? ", tuning off" : "");
    }
    CK(cudaMemsetAsync(L.rate_max, 0, sizeof(unsigned long long), L.stream));
    CK(cudaMemsetAsync(L.err, 0, sizeof(int), L.stream));
    CK(cudaStreamSynchronize(L.stream));
    return FXB_OK;
}

extern "C" int fxb_attach_unk(const double *unk_host)
{
    if (!unk_host) return fail(FXB_EARG, "fxb_attach_unk: null UNK");
    if (amr_active()) {
        int rc = amr_attach(unk_host);
        if (rc) return rc;
        L.attached = true;
        L.unk_attached = unk_host;
        state_changed(false);
        return FXB_OK;
    }
    if (!L.inited || !L.bcoord) return fail(FXB_EARG, "fxb_attach_unk: call fxb_init and fxb_register_blocks first");
    CK(cudaMemcpyAsync(L.unk_dev, unk_host, sizeof(double) * L.unk_doubles, cudaMemcpyHostToDevice, L.stream));
    UnkGeom g = unk_geom();
    unk_to_state_kernel<<<1184, 256, 0, L.stream>>>(L.unk_dev, L.buf[L.cur], g, L.bcoord, L.dmap_dev, L.nblk);
    if (L.ns)
        unk_to_spec_kernel<<<1184, 256, 0, L.stream>>>(L.unk_dev, L.spb[L.cur], g, L.bcoord, L.sslot_dev, L.ns, L.nblk);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(L.stream));
    L.attached = true;
    L.unk_attached = unk_host;
    state_changed(false);
    if (!L.ug_tuned) {
        L.ug_tuned = true;        // new data on the same grid keeps the launch shapes
        int rc = ug_tune();
        if (rc) return rc;
        state_changed(false);
    }
    L.shok_valid = false;         // the attached UNK's SHOK stands until the next step
    return FXB_OK;
}

extern "C" int fxb_sync_from_host(const double *unk_host) { return fxb_attach_unk(unk_host); }

extern "C" int fxb_sync_to_host(double *unk_host)
{
    if (!L.attached) return fail(FXB_EARG, "fxb_sync_to_host: no UNK attached");
    if (!unk_host) return fail(FXB_EARG, "fxb_sync_to_host: null UNK");
    if (amr_active()) {
        int rc = amr_sync_to_host(unk_host);
        return rc ? rc : check_err_word();
    }
    UnkGeom g = unk_geom();
    state_to_unk_kernel<<<1184, 256, 0, L.stream>>>(L.buf[L.cur], L.unk_dev, g, L.bcoord, L.dmap_dev, L.nblk);
    if (L.ns)
        spec_to_unk_kernel<<<1184, 256, 0, L.stream>>>(L.spb[L.cur], L.unk_dev, g, L.bcoord, L.sslot_dev, L.ns, L.nblk);
    CK(cudaGetLastError());
    if (L.shok && L.shok_valid && L.shock_slot >= 0)   // SHOK_VAR, guard cells filled like the other variables
        shok_to_unk_kernel<<<1184, 256, 0, L.stream>>>(L.shok, L.unk_dev, g, L.bcoord, L.nblk, L.shock_slot);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(unk_host, L.unk_dev, sizeof(double) * L.unk_doubles, cudaMemcpyDeviceToHost, L.stream));
    CK(cudaStreamSynchronize(L.stream));
    L.counts[FXB_COUNT_GC_FILLS]++;
    L.counts[FXB_COUNT_GC_DOUBLES] += L.unk_doubles;
    return check_err_word();
}

// ---- interior transfers --------------------------------------------------
// The step reads and writes the device variables (and species) of block
// interiors only.  fxb_put_interior / fxb_get_interior move the interior
// rows of every block (nxb cells x nunk slots, contiguous in UNK) between
// the caller's UNK, page-locked at the first call, and the device UNK mirror
// with strided copies on the copy engine; the mirror's rows are then
// unpacked into the state, or packed from it, by the attach and sync kernels.
namespace {
// page-lock unk_host (bytes long) unless it already is; a different UNK
// releases the previous one
int lock_host_unk(const void *unk_host, size_t bytes)
{
    if (L.mapped_host == unk_host && L.mapped_bytes == bytes) return FXB_OK;
    if (L.mapped_registered) cudaHostUnregister(const_cast<void *>(L.mapped_host));
    L.mapped_host = nullptr;
    L.mapped_bytes = 0;
    L.mapped_registered = false;
    cudaPointerAttributes at{};
    const bool locked = cudaPointerGetAttributes(&at, unk_host) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (!locked) {
        CK(cudaHostRegister(const_cast<void *>(unk_host), bytes, cudaHostRegisterDefault));
        L.mapped_registered = true;
    }
    L.mapped_host = unk_host;
    L.mapped_bytes = bytes;
    return FXB_OK;
}

// the interior rows of every block, between the caller's UNK and the device
// mirror: one 3-D copy over all blocks in 2-D (their rows are evenly
// spaced), one per block in 3-D (the k guard planes separate the blocks)
int copy_interior_rows(double *dst, const double *src, cudaMemcpyKind kind)
{
    const UnkGeom g = unk_geom();
    const size_t pitch = sizeof(double) * g.nunk * g.nig;
    cudaMemcpy3DParms p{};
    p.srcPtr = make_cudaPitchedPtr(const_cast<double *>(src), pitch, pitch, g.njg);
    p.dstPtr = make_cudaPitchedPtr(dst, pitch, pitch, g.njg);
    p.kind = kind;
    const size_t x0 = sizeof(double) * g.nunk * g.ng, w = sizeof(double) * g.nunk * g.nxb;
    if (g.ndim == 2) {
        p.srcPos = p.dstPos = make_cudaPos(x0, g.ng, 0);
        p.extent = make_cudaExtent(w, g.nyb, L.nblk);
        CK(cudaMemcpy3DAsync(&p, L.stream));
        return FXB_OK;
    }
    p.extent = make_cudaExtent(w, g.nyb, g.nzb);
    for (int b = 0; b < L.nblk; b++) {
        p.srcPos = p.dstPos = make_cudaPos(x0, g.ng, (size_t)b * g.nkg + g.ng);
        CK(cudaMemcpy3DAsync(&p, L.stream));
    }
    return FXB_OK;
}
} // namespace

extern "C" int fxb_put_interior(const double *unk_host)
{
    if (!unk_host) return fail(FXB_EARG, "fxb_put_interior: null UNK");
    if (!L.attached) return fail(FXB_EARG, "fxb_put_interior: call fxb_attach_unk first");
    if (amr_active()) return fxb_attach_unk(unk_host);
    int rc = lock_host_unk(unk_host, sizeof(double) * L.unk_doubles);
    if (!rc) rc = copy_interior_rows(L.unk_dev, unk_host, cudaMemcpyHostToDevice);
    if (rc) return rc;
    UnkGeom g = unk_geom();
    unk_to_state_kernel<<<1184, 256, 0, L.stream>>>(L.unk_dev, L.buf[L.cur], g, L.bcoord, L.dmap_dev, L.nblk);
    if (L.ns)
        unk_to_spec_kernel<<<1184, 256, 0, L.stream>>>(L.unk_dev, L.spb[L.cur], g, L.bcoord, L.sslot_dev, L.ns, L.nblk);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(L.stream));
    state_changed(false);
    L.shok_valid = false;         // the host's SHOK stands until the next step
    return check_err_word();
}

extern "C" int fxb_get_interior(double *unk_host)
{
    if (!unk_host) return fail(FXB_EARG, "fxb_get_interior: null UNK");
    if (!L.attached) return fail(FXB_EARG, "fxb_get_interior: no UNK attached");
    if (amr_active()) return fxb_sync_to_host(unk_host);
    int rc = lock_host_unk(unk_host, sizeof(double) * L.unk_doubles);
    if (rc) return rc;
    UnkGeom g = unk_geom();
    state_to_unk_kernel<<<1184, 256, 0, L.stream>>>(L.buf[L.cur], L.unk_dev, g, L.bcoord, L.dmap_dev, L.nblk);
    if (L.ns)
        spec_to_unk_kernel<<<1184, 256, 0, L.stream>>>(L.spb[L.cur], L.unk_dev, g, L.bcoord, L.sslot_dev, L.ns, L.nblk);
    if (L.shok && L.shok_valid && L.shock_slot >= 0)
        shok_to_unk_kernel<<<1184, 256, 0, L.stream>>>(L.shok, L.unk_dev, g, L.bcoord, L.nblk, L.shock_slot);
    CK(cudaGetLastError());
    rc = copy_interior_rows(unk_host, L.unk_dev, cudaMemcpyDeviceToHost);
    if (rc) return rc;
    CK(cudaStreamSynchronize(L.stream));
    return check_err_word();
}

namespace {
// the device variables a guard-fill mask selects (bit fxb_var; 0 = all),
// packed per cell in device-variable order: pos[v] is v's place in the
// packed vector (-1: not selected), slot[q] the UNK slot of place q
struct VarPack {
    int pos[NV_DEV];
    int slot[NV_DEV];
    int n = 0;
};

VarPack var_pack(int mask_bits)
{
    VarPack vp;
    for (int v = 0; v < NV_DEV; v++) {
        const bool sel = mask_bits == 0 || ((mask_bits >> kDevToVar[v]) & 1);
        vp.pos[v] = sel ? vp.n : -1;
        if (sel) vp.slot[vp.n++] = L.dmap[v];
    }
    return vp;
}
} // namespace

namespace fxb {
// packed cell vectors (ncell x n doubles, device) into their UNK slots of
// unk_host (ncell x nunk), through a pinned staging copy; variables outside
// the pack keep their host values
int pack_to_host(const double *pack_dev, long ncell, int n, const int *slot, double *unk_host)
{
    const size_t nd = (size_t)ncell * n;
    if (nd > L.pack_host_doubles) {
        if (L.pack_host) cudaFreeHost(L.pack_host);
        L.pack_host = nullptr;
        L.pack_host_doubles = 0;
        CK(cudaMallocHost(&L.pack_host, sizeof(double) * nd));
        L.pack_host_doubles = nd;
    }
    CK(cudaMemcpyAsync(L.pack_host, pack_dev, sizeof(double) * nd, cudaMemcpyDeviceToHost, L.stream));
    CK(cudaStreamSynchronize(L.stream));
    const int nunk = L.nunk;
    const double *src = L.pack_host;
    auto scatter = [&](long c0, long c1) {
        for (long c = c0; c < c1; c++)
            for (int q = 0; q < n; q++) unk_host[c * nunk + slot[q]] = src[c * n + q];
    };
    const int nth = ncell >= (1L << 20) ? 8 : 1;
    std::vector<std::thread> pool;
    for (int t = 1; t < nth; t++) pool.emplace_back(scatter, ncell * t / nth, ncell * (t + 1) / nth);
    scatter(0, ncell / nth);
    for (auto &th : pool) th.join();
    L.counts[FXB_COUNT_GC_DOUBLES] += (long long)nd;
    return FXB_OK;
}
} // namespace fxb

extern "C" int fxb_fill_guardcells(int mask_bits, int do_eos, double *unk_host)
{
    if (!L.attached) return fail(FXB_EARG, "fxb_fill_guardcells: no UNK attached");
    if (mask_bits < 0 || mask_bits >= (1 << FXB_NVAR))
        return fail(FXB_EARG, "fxb_fill_guardcells: mask bits outside the fxb_var range");
    double *dst = unk_host ? unk_host : const_cast<double *>(L.unk_attached);
    if (!dst) return fail(FXB_EARG, "fxb_fill_guardcells: null UNK");
    const VarPack vp = var_pack(mask_bits);
    if (vp.n == 0) return FXB_OK;
    // all variables: the whole UNK in one copy (Eos on the guard regions next
    // to other levels is part of the AMR fill, so doEos = .false. takes the
    // packed path there)
    if (vp.n == NV_DEV && (do_eos || !amr_active())) return fxb_sync_to_host(dst);
    L.counts[FXB_COUNT_GC_FILLS]++;
    if (amr_active()) {
        int rc = amr_fill_to_host(dst, vp.pos, vp.n, vp.slot, do_eos != 0);
        return rc ? rc : check_err_word();
    }
    // UG (UG/Grid_fillGuardCells.F90 does not act on doEos): the selected
    // variables of every block, guard cells included, packed per cell
    const long ncell = L.unk_doubles / L.nunk;
    const size_t need = (size_t)ncell * vp.n;
    if (need > L.pack_dev_doubles) {
        if (L.pack_dev) cudaFree(L.pack_dev);
        L.pack_dev = nullptr;
        L.pack_dev_doubles = 0;
        CK(cudaMalloc(&L.pack_dev, sizeof(double) * need));
        L.pack_dev_doubles = need;
    }
    CK(cudaMemcpyAsync(L.pmap_dev, vp.pos, sizeof(int) * NV_DEV, cudaMemcpyHostToDevice, L.stream));
    UnkGeom g = unk_geom();
    g.nunk = vp.n;
    state_to_unk_kernel<<<1184, 256, 0, L.stream>>>(L.buf[L.cur], L.pack_dev, g, L.bcoord, L.pmap_dev, L.nblk);
    CK(cudaGetLastError());
    int rc = pack_to_host(L.pack_dev, ncell, vp.n, vp.slot, dst);
    return rc ? rc : check_err_word();
}

extern "C" int fxb_eos(void)
{
    if (!L.attached) return fail(FXB_EARG, "fxb_eos: no UNK attached");
    if (amr_active()) {
        state_changed(false);
        return amr_eos();
    }
    eos_kernel<<<1184, 256, 0, L.stream>>>(L.buf[L.cur], L.vstride, L.ncell, L.dprm, L.gam1inv, L.ggprodinv);
    CK(cudaGetLastError());
    state_changed(false);
    return FXB_OK;
}

extern "C" int fxb_hydro_step(double sim_time, double dt, double dt_old)
{
    (void)sim_time; (void)dt_old;
    if (!L.attached) return fail(FXB_EARG, "fxb_hydro_step: no UNK attached");
    if (!(dt > 0.)) return fail(FXB_EARG, "fxb_hydro_step: dt must be positive");
    CK(cudaMemsetAsync(L.rate_max, 0, sizeof(unsigned long long), L.stream));
    CK(cudaEventRecord(L.ev0, L.stream));
    int nl = 1;
    if (amr_active()) {
        int rc = amr_step(nullptr, dt, &nl);
        if (rc) return rc;
    } else {
        int rc = launch_hydro(L.cur, nullptr, dt);
        if (rc) return rc;
        L.cur = 1 - L.cur;
        nl = ug_step_launches();
    }
    CK(cudaEventRecord(L.ev1, L.stream));
    state_changed(true);
    L.counts[FXB_COUNT_STEPS]++;
    L.last_launches = nl;
    L.timing_valid = true;
    return FXB_OK;
}

extern "C" int fxb_compute_dt(double *dt_out, int32_t loc[5])
{
    if (!L.attached) return fail(FXB_EARG, "fxb_compute_dt: no UNK attached");
    if (!dt_out) return fail(FXB_EARG, "fxb_compute_dt: null output");
    // Driver_computeDt.F90:306 calls Hydro_computeDt once per leaf block: the
    // first call after a state change reduces the whole grid on the device,
    // the later ones return the cached global result without a launch or a
    // host synchronisation
    if (L.dt_valid && (!loc || L.loc_valid)) {
        L.counts[FXB_COUNT_DT_CACHED]++;
        if (loc)
            for (int q = 0; q < 5; q++) loc[q] = L.loc_cached[q];
        *dt_out = L.dt_cached;
        if (!(L.dt_cached > 0.)) return fail(FXB_EDT, "[Hydro]: Computed dt is not positive! Aborting!");
        return FXB_OK;
    }
    L.counts[FXB_COUNT_DT_DEVICE]++;
    if (!L.rate_valid && amr_active()) {
        CK(cudaMemsetAsync(L.rate_max, 0, sizeof(unsigned long long), L.stream));
        int rc = amr_rate();
        if (rc) return rc;
        L.rate_valid = true;
    }
    if (!L.rate_valid) {
        CK(cudaMemsetAsync(L.rate_max, 0, sizeof(unsigned long long), L.stream));
        rate_kernel<<<1184, 256, 0, L.stream>>>(interior(L.cur), L.vstride, L.nx, int_ny(), int_nz(), L.dom.ndim,
                                                cell_dx(0), cell_dx(1), cell_dx(2), L.rate_max);
        CK(cudaGetLastError());
        L.rate_valid = true;
    }
    unsigned long long bits = 0, key = ~0ull;
    if (loc) {
        // L.partials doubles as the 8-byte key (fxb_integrals rewrites it before use)
        unsigned long long *dkey = (unsigned long long *)L.partials;
        CK(cudaMemsetAsync(dkey, 0xff, sizeof(unsigned long long), L.stream));
        if (amr_active()) {
            int rc = amr_locate(dkey);
            if (rc) return rc;
        } else {
            locate_kernel<<<1184, 256, 0, L.stream>>>(interior(L.cur), L.vstride, L.nx, int_ny(), int_nz(), L.dom.ndim, cell_dx(0),
                                                      cell_dx(1), cell_dx(2), L.rate_max, L.dom.nxb,
                                                      L.dom.ndim >= 2 ? L.dom.nyb : 1, L.dom.ndim == 3 ? L.dom.nzb : 1,
                                                      dkey);
            CK(cudaGetLastError());
        }
        CK(cudaMemcpyAsync(&key, dkey, sizeof(key), cudaMemcpyDeviceToHost, L.stream));
    }
    CK(cudaMemcpyAsync(&bits, L.rate_max, sizeof(bits), cudaMemcpyDeviceToHost, L.stream));
    CK(cudaStreamSynchronize(L.stream));
    int rc = check_err_word();
    if (rc) return rc;
    double r;
    memcpy(&r, &bits, sizeof(r));
    double dt = (r != 0.) ? L.prm.cfl / r : 1.79769313486231570e308;
    if (loc) {
        // Hydro_computeDt.F90:231-235: i, j, k in the block's guard-inclusive
        // 1-based index space, then the refinement level; the fifth entry is
        // the 1-based UNK block (the reference keeps its MPI rank there)
        for (int q = 0; q < 5; q++) loc[q] = 0;
        if (key != ~0ull) {
            const int ndim = L.dom.ndim, ng = L.dom.nguard;
            const long nxb = L.dom.nxb, nyb = ndim >= 2 ? L.dom.nyb : 1, nzb = ndim == 3 ? L.dom.nzb : 1;
            long i = key % nxb, j = (key / nxb) % nyb, k = (key / (nxb * nyb)) % nzb, b = key / (nxb * nyb * nzb);
            loc[0] = (int32_t)(i + ng + 1);
            loc[1] = (int32_t)(j + (ndim >= 2 ? ng + 1 : 1));
            loc[2] = (int32_t)(k + (ndim == 3 ? ng + 1 : 1));
            loc[3] = amr_active() ? amr_leaf_level((int)b) : 1;
            loc[4] = (int32_t)(b + 1);
        }
        for (int q = 0; q < 5; q++) L.loc_cached[q] = loc[q];
        L.loc_valid = true;
    }
    L.dt_cached = dt;
    L.dt_valid = true;
    *dt_out = dt;
    if (!(dt > 0.)) return fail(FXB_EDT, "[Hydro]: Computed dt is not positive! Aborting!");
    return FXB_OK;
}

extern "C" int fxb_advance(int nsteps, double *dt, double *dt_old, double f, double dtmin, double dtmax)
{
    if (!L.attached) return fail(FXB_EARG, "fxb_advance: no UNK attached");
    if (!dt || !dt_old || nsteps < 0) return fail(FXB_EARG, "fxb_advance: bad argument");
    if (has_halo()) return fail(FXB_EUNSUPPORTED, "fxb_advance: a slab with halos exchanges them between steps");
    double h[2] = {*dt, *dt_old};
    CK(cudaMemcpyAsync(L.dtv, h, sizeof(h), cudaMemcpyHostToDevice, L.stream));
    CK(cudaMemsetAsync(L.rate_max, 0, sizeof(unsigned long long), L.stream));
    // graphs of two steps (buffer c -> 1-c -> c), built once per starting buffer
    const bool amr = amr_active();
    int step_launches = amr ? 0 : ug_step_launches();
    auto one_step = [&](int src) -> int {
        int rc = amr ? amr_step(L.dtv, 0., &step_launches) : launch_hydro(src, L.dtv, 0.);
        if (rc) return rc;
        dt_finalize_kernel<<<1, 1, 0, L.stream>>>(L.dtv, L.rate_max, L.prm.cfl, f, dtmin, dtmax, L.err);
        return cudaGetLastError() == cudaSuccess ? FXB_OK : fail(FXB_ECUDA, "dt kernel launch");
    };
    CK(cudaEventRecord(L.ev0, L.stream));
    int done = 0;
    if (nsteps >= 2) {
        int c = amr ? amr_cur() : L.cur;
        if (!L.graph_exec[c]) {
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(L.stream, cudaStreamCaptureModeThreadLocal));
            int rc = one_step(c);
            if (!rc) rc = one_step(1 - c);
            cudaError_t e = cudaStreamEndCapture(L.stream, &graph);
            if (rc) return rc;
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&L.graph_exec[c], graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
            // f, dtmin, dtmax are baked into the graph; rebuild when they change
        }
        for (; done + 2 <= nsteps; done += 2) CK(cudaGraphLaunch(L.graph_exec[c], L.stream));
    }
    for (; done < nsteps; done++) {
        int rc = one_step(L.cur);
        if (rc) return rc;
        if (!amr) L.cur = 1 - L.cur;
    }
    CK(cudaEventRecord(L.ev1, L.stream));
    CK(cudaMemcpyAsync(h, L.dtv, sizeof(h), cudaMemcpyDeviceToHost, L.stream));
    CK(cudaStreamSynchronize(L.stream));
    *dt = h[0];
    *dt_old = h[1];
    state_changed(false);
    L.counts[FXB_COUNT_STEPS] += nsteps;
    L.last_launches = (step_launches + 1) * nsteps;
    L.timing_valid = true;
    return check_err_word();
}

extern "C" int fxb_integrals(double out[7])
{
    if (!L.attached) return fail(FXB_EARG, "fxb_integrals: no UNK attached");
    if (amr_active()) return amr_integrals(out, L.partials, L.npartials);
    double dv = cell_dx(0) * cell_dx(1) * cell_dx(2);
    integrals_kernel<<<L.npartials, 256, 0, L.stream>>>(interior(L.cur), L.vstride, (long)L.nint * L.plane, dv,
                                                        L.partials);
    integrals_final_kernel<<<1, 32, 0, L.stream>>>(L.partials, L.npartials, L.partials + L.npartials * 7);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, L.partials + L.npartials * 7, 7 * sizeof(double), cudaMemcpyDeviceToHost, L.stream));
    CK(cudaStreamSynchronize(L.stream));
    return FXB_OK;
}

extern "C" long fxb_halo_doubles(int planes)
{
    if (!L.inited || planes < 0) return 0;
    return (long)NV_DEV * planes * L.plane;
}

extern "C" int fxb_halo_pack(double *send_lo, int n_lo, double *send_hi, int n_hi)
{
    if (!L.attached) return fail(FXB_EARG, "fxb_halo_pack: no UNK attached");
    if (n_lo < 0 || n_hi < 0 || n_lo > L.nint || n_hi > L.nint || (n_lo && !send_lo) || (n_hi && !send_hi))
        return fail(FXB_EARG, "fxb_halo_pack: bad plane count or buffer");
    // variable-major messages: one 2-D copy gathers the planes of all variables
    const size_t spitch = sizeof(double) * L.vstride;
    if (n_lo) {
        const size_t w = sizeof(double) * n_lo * L.plane;
        CK(cudaMemcpy2DAsync(send_lo, w, interior(L.cur), spitch, w, NV_DEV, cudaMemcpyDeviceToDevice, L.stream));
    }
    if (n_hi) {
        const size_t w = sizeof(double) * n_hi * L.plane;
        CK(cudaMemcpy2DAsync(send_hi, w, interior(L.cur) + (long)(L.nint - n_hi) * L.plane, spitch, w, NV_DEV,
                             cudaMemcpyDeviceToDevice, L.stream));
    }
    return FXB_OK;
}

extern "C" int fxb_halo_unpack(const double *recv_lo, const double *recv_hi)
{
    if (!L.attached) return fail(FXB_EARG, "fxb_halo_unpack: no UNK attached");
    const fxb_slab &sl = L.slab;
    if ((sl.halo_lo && !recv_lo) || (sl.halo_hi && !recv_hi)) return fail(FXB_EARG, "fxb_halo_unpack: missing buffer");
    const size_t dpitch = sizeof(double) * L.vstride;
    double *st = L.buf[L.cur];
    if (sl.halo_lo) {
        const size_t w = sizeof(double) * sl.halo_lo * L.plane;
        CK(cudaMemcpy2DAsync(st, dpitch, recv_lo, w, w, NV_DEV, cudaMemcpyDeviceToDevice, L.stream));
    }
    if (sl.halo_hi) {
        const size_t w = sizeof(double) * sl.halo_hi * L.plane;
        CK(cudaMemcpy2DAsync(st + (long)(sl.halo_lo + L.nint) * L.plane, dpitch, recv_hi, w, w, NV_DEV,
                             cudaMemcpyDeviceToDevice, L.stream));
    }
    // the fused step's rate covers the slab's own cells only, so a halo
    // update leaves a valid CFL rate valid
    return FXB_OK;
}

extern "C" int fxb_amr_set_roles(const unsigned char *roles, int nleaf)
{
    if (!amr_active()) return fail(FXB_EUNSUPPORTED, "fxb_amr_set_roles: needs a registered AMR mesh");
    int rc = amr_set_roles(roles, nleaf);
    if (rc) return rc;
    state_changed(false);
    for (int i = 0; i < 2; i++) {
        if (L.graph_exec[i]) cudaGraphExecDestroy(L.graph_exec[i]);
        L.graph_exec[i] = nullptr;
    }
    return FXB_OK;
}

extern "C" long fxb_amr_leaf_doubles(void) { return amr_active() ? amr_leaf_doubles() : 0; }

extern "C" int fxb_amr_pack_leaves(const int32_t *leaves, int n, double *buf)
{
    if (!L.attached || !amr_active()) return fail(FXB_EARG, "fxb_amr_pack_leaves: needs an attached AMR mesh");
    if (n < 0 || (n && (!leaves || !buf))) return fail(FXB_EARG, "fxb_amr_pack_leaves: bad list or buffer");
    return amr_copy_leaves(leaves, n, buf, true);
}

extern "C" int fxb_amr_unpack_leaves(const int32_t *leaves, int n, const double *buf)
{
    if (!L.attached || !amr_active()) return fail(FXB_EARG, "fxb_amr_unpack_leaves: needs an attached AMR mesh");
    if (n < 0 || (n && (!leaves || !buf))) return fail(FXB_EARG, "fxb_amr_unpack_leaves: bad list or buffer");
    return amr_copy_leaves(leaves, n, const_cast<double *>(buf), false);
}

extern "C" int fxb_mark_refine_derefine(int nvars, const int *refine_var, const double *refine_cutoff,
                                        const double *derefine_cutoff, const double *refine_filter, int max_refine,
                                        int *flags, double *error)
{
    if (!L.attached) return fail(FXB_EARG, "fxb_mark_refine_derefine: no UNK attached");
    if (!amr_active()) return fail(FXB_EUNSUPPORTED, "fxb_mark_refine_derefine: needs a registered AMR mesh");
    if (nvars <= 0 || nvars > FXB_NVAR || !refine_var || !refine_cutoff || !derefine_cutoff || !refine_filter || !flags)
        return fail(FXB_EARG, "fxb_mark_refine_derefine: bad argument");
    int dvar[FXB_NVAR], need_eos[FXB_NVAR];
    for (int l = 0; l < nvars; l++) {
        dvar[l] = -1;
        for (int v = 0; v < NV_DEV; v++)
            if (kDevToVar[v] == refine_var[l]) dvar[l] = v;
        if (dvar[l] < 0) return fail(FXB_EARG, "fxb_mark_refine_derefine: unknown refinement variable");
        // gr_makeMaskConsistent.F90:376-395 (one temperature, MODE_DENS_EI, constant gamc)
        const int r = refine_var[l];
        need_eos[l] = r == FXB_PRES || r == FXB_TEMP || r == FXB_ENER || r == FXB_EINT || r == FXB_GAME;
    }
    int rc = amr_mark_refine(nvars, dvar, need_eos, refine_cutoff, derefine_cutoff, refine_filter, max_refine, flags,
                             error);
    if (rc) return rc;
    return check_err_word();
}

// ---- PARAMESH's tree update (host only) -----------------------------------------
namespace {
uint64_t tree_key(int lev, const int c[3])
{
    return ((uint64_t)lev << 60) | ((uint64_t)(uint32_t)c[0] << 40) | ((uint64_t)(uint32_t)c[1] << 20) |
           (uint64_t)(uint32_t)c[2];
}
// Morton key of a block scaled to level maxlev: bits of x, y, z interleaved
uint64_t morton(int lev, const int c[3], int maxlev)
{
    const int sh = maxlev - lev;
    uint64_t x = (uint64_t)c[0] << sh, y = (uint64_t)c[1] << sh, z = (uint64_t)c[2] << sh, k = 0;
    for (int b = 0; b < 21; b++)
        k |= ((x >> b) & 1) << (3 * b) | ((y >> b) & 1) << (3 * b + 1) | ((z >> b) & 1) << (3 * b + 2);
    return k;
}
} // namespace

extern "C" int fxb_refine_derefine(const fxb_domain *dom, const fxb_block_desc *leaves, int n, const int *flags,
                                   int lrefine_min, int lrefine_max, fxb_block_desc *out, int cap, int *nout)
{
    if (!dom || !leaves || n <= 0 || !flags || !nout || (cap > 0 && !out))
        return fail(FXB_EARG, "fxb_refine_derefine: bad argument");
    if (dom->ndim != 2 && dom->ndim != 3) return fail(FXB_EARG, "fxb_refine_derefine: ndim must be 2 or 3");
    if (lrefine_min < 1 || lrefine_max < lrefine_min || lrefine_max > 15)
        return fail(FXB_EARG, "fxb_refine_derefine: bad lrefine_min / lrefine_max");
    const int ndim = dom->ndim, nch = ndim == 3 ? 8 : 4;
    const int nb0[3] = {dom->nblockx, ndim >= 2 ? dom->nblocky : 1, ndim == 3 ? dom->nblockz : 1};
    auto nb_at = [&](int lev, int d) { return d < ndim ? nb0[d] << (lev - 1) : 1; };
    std::unordered_map<uint64_t, int> leaf;
    std::unordered_set<uint64_t> parent;
    for (int l = 0; l < n; l++) {
        const fxb_block_desc &B = leaves[l];
        if (B.level < 1 || B.level > 15) return fail(FXB_EARG, "fxb_refine_derefine: level out of range");
        for (int d = 0; d < 3; d++)
            if (B.bcoord[d] < 0 || B.bcoord[d] >= nb_at(B.level, d))
                return fail(FXB_EARG, "fxb_refine_derefine: block coordinate out of range");
        if (!leaf.emplace(tree_key(B.level, B.bcoord), l).second) return fail(FXB_EARG, "fxb_refine_derefine: duplicate leaf");
        int c[3] = {B.bcoord[0], B.bcoord[1], B.bcoord[2]};
        for (int lev = B.level - 1; lev >= 1; lev--) {
            for (int d = 0; d < 3; d++) c[d] /= 2;
            parent.insert(tree_key(lev, c));
        }
    }
    // the leaf covering position p of level lev (itself or a coarser ancestor), or -1
    auto covering = [&](int lev, const int p[3]) {
        int c[3] = {p[0], p[1], p[2]};
        for (int L = lev; L >= 1; L--) {
            auto it = leaf.find(tree_key(L, c));
            if (it != leaf.end()) return it->second;
            for (int d = 0; d < 3; d++) c[d] /= 2;
        }
        return -1;
    };
    // neighbours across faces, edges and corners, wrapped on periodic axes
    auto neighbours = [&](int lev, const int c[3], std::vector<std::array<int, 3>> &v) {
        v.clear();
        const int K3 = ndim == 3 ? 1 : 0;
        for (int k = -K3; k <= K3; k++) for (int j = -1; j <= 1; j++) for (int i = -1; i <= 1; i++) {
            if (!(i | j | k)) continue;
            std::array<int, 3> p = {c[0] + i, c[1] + j, c[2] + k};
            bool ok = true;
            for (int d = 0; d < ndim && ok; d++) {
                const int nb = nb_at(lev, d);
                if (p[d] < 0 || p[d] >= nb) {
                    if (dom->bc[2 * d + (p[d] >= nb)] != FXB_BC_PERIODIC) ok = false;
                    else p[d] = (p[d] + nb) % nb;
                }
            }
            if (ok) v.push_back(p);
        }
    };
    // level limits, mpi_amr_refine_derefine.F90:157-163
    std::vector<char> ref(n), deref(n);
    for (int l = 0; l < n; l++) {
        ref[l] = flags[l] == 1;
        deref[l] = flags[l] == -1;
        if (leaves[l].level >= lrefine_max) ref[l] = 0;
        if (leaves[l].level == lrefine_min) deref[l] = 0;
        if (leaves[l].level < lrefine_min) ref[l] = 1;
    }
    // amr_check_refine: a leaf one level coarser than a refining neighbour refines too
    std::vector<std::array<int, 3>> nbrs;
    for (bool changed = true; changed;) {
        changed = false;
        for (int l = 0; l < n; l++) {
            if (!ref[l]) continue;
            neighbours(leaves[l].level, leaves[l].bcoord, nbrs);
            for (auto &p : nbrs) {
                const int cv = covering(leaves[l].level, p.data());
                if (cv >= 0 && leaves[cv].level < leaves[l].level && !ref[cv]) {
                    ref[cv] = 1;
                    deref[cv] = 0;
                    changed = true;
                }
            }
        }
    }
    // amr_check_derefine: no root blocks, no same-level neighbour that is a
    // parent or refines, all siblings derefining
    std::unordered_map<uint64_t, int> group;
    std::vector<char> grouped(n, 0);
    for (int l = 0; l < n; l++) {
        const int lev = leaves[l].level;
        if (!deref[l] || ref[l] || lev == 1) continue;
        neighbours(lev, leaves[l].bcoord, nbrs);
        bool blocked = false;
        for (auto &p : nbrs) {
            const uint64_t k = tree_key(lev, p.data());
            auto it = leaf.find(k);
            blocked = it != leaf.end() ? (bool)ref[it->second] : parent.count(k) > 0;
            if (blocked) break;
        }
        if (blocked) continue;
        grouped[l] = 1;
        const int pc[3] = {leaves[l].bcoord[0] / 2, leaves[l].bcoord[1] / 2, leaves[l].bcoord[2] / 2};
        group[tree_key(lev - 1, pc)]++;
    }
    std::vector<fxb_block_desc> res;
    std::unordered_set<uint64_t> added;
    for (int l = 0; l < n; l++) {
        const fxb_block_desc &B = leaves[l];
        if (ref[l]) {
            for (int q = 0; q < nch; q++) {
                fxb_block_desc C;
                C.level = B.level + 1;
                C.bcoord[0] = 2 * B.bcoord[0] + (q & 1);
                C.bcoord[1] = 2 * B.bcoord[1] + ((q >> 1) & 1);
                C.bcoord[2] = ndim == 3 ? 2 * B.bcoord[2] + ((q >> 2) & 1) : 0;
                res.push_back(C);
            }
            continue;
        }
        if (grouped[l]) {
            const int pc[3] = {B.bcoord[0] / 2, B.bcoord[1] / 2, B.bcoord[2] / 2};
            const uint64_t pk = tree_key(B.level - 1, pc);
            if (group[pk] == nch) {
                if (added.insert(pk).second) {
                    fxb_block_desc P;
                    P.level = B.level - 1;
                    for (int d = 0; d < 3; d++) P.bcoord[d] = pc[d];
                    res.push_back(P);
                }
                continue;
            }
        }
        res.push_back(B);
    }
    // PARAMESH's Morton order (finest-level scaled key, then level)
    int maxlev = 1;
    for (auto &B : res) maxlev = std::max(maxlev, B.level);
    std::sort(res.begin(), res.end(), [&](const fxb_block_desc &a, const fxb_block_desc &b) {
        const uint64_t ka = morton(a.level, a.bcoord, maxlev), kb = morton(b.level, b.bcoord, maxlev);
        return ka != kb ? ka < kb : a.level < b.level;
    });
    *nout = (int)res.size();
    if ((int)res.size() > cap) return fail(FXB_EARG, "fxb_refine_derefine: output list too small (see *nout)");
    std::copy(res.begin(), res.end(), out);
    return FXB_OK;
}

extern "C" int fxb_regrid(const fxb_block_desc *blocks, int nblk)
{
    if (!L.attached) return fail(FXB_EARG, "fxb_regrid: no UNK attached");
    if (!amr_active()) return fail(FXB_EUNSUPPORTED, "fxb_regrid: needs a registered AMR mesh");
    if (!blocks || nblk <= 0) return fail(FXB_EARG, "fxb_regrid: empty block list");
    for (int i = 0; i < 2; i++) {
        if (L.graph_exec[i]) cudaGraphExecDestroy(L.graph_exec[i]);
        L.graph_exec[i] = nullptr;
    }
    state_changed(false);
    int rc = amr_regrid(blocks, nblk);
    if (rc) return rc;
    return check_err_word();
}

extern "C" int fxb_last_timing(double *ms, int *kernel_launches)
{
    if (!L.timing_valid) return fail(FXB_EARG, "fxb_last_timing: nothing timed yet");
    float f = 0.f;
    CK(cudaEventSynchronize(L.ev1));
    CK(cudaEventElapsedTime(&f, L.ev0, L.ev1));
    if (ms) *ms = f;
    if (kernel_launches) *kernel_launches = L.last_launches;
    return FXB_OK;
}

extern "C" void *fxb_stream(void) { return (void *)L.stream; }

extern "C" int fxb_tuning(char *buf, int len)
{
    if (!buf || len <= 0) return fail(FXB_EARG, "fxb_tuning: null or empty buffer");
    if (amr_active()) snprintf(buf, len, "%s", amr_tuning_log());
    else snprintf(buf, len, "%s", L.ug_tuned ? L.ug_log : "uniform grid: launch shapes are chosen at the first attach");
    return FXB_OK;
}

extern "C" int fxb_counters(long long counts[FXB_NCOUNTERS])
{
    if (!counts) return fail(FXB_EARG, "fxb_counters: null output");
    for (int q = 0; q < FXB_NCOUNTERS; q++) counts[q] = L.counts[q];
    return FXB_OK;
}

extern "C" int fxb_last_error(fxb_error *err)
{
    if (err) *err = L.lasterr;
    return L.lasterr.code;
}

extern "C" void fxb_finalize(void)
{
    if (L.stream) cudaStreamSynchronize(L.stream);
    free_all();
}
