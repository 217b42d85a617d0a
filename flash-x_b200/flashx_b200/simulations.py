"""Initial conditions for the benchmark problems, written into Flash-X UNK
arrays (numpy, C order (blk, k, j, i, var) == Fortran unk(var,i,j,k,blk)).

Sod follows FX/Simulation/SimulationMain/Sod/Simulation_init.F90:120-135 and
Simulation_initBlock.F90 (planar interface at an angle, the cell cut by the
interface gets the average of the two states).  Kelvin-Helmholtz,
Rayleigh-Taylor and the noisy-gas sweep have no setup in the reference; they
are defined here from the benchmark descriptions, with counter-based
Philox4x32-10 noise (seed 20261203, counter = global cell index) so any
implementation can regenerate them bit for bit.
"""
import math

import numpy as np

from .params import (DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ,
                     BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, Geometry, HydroParams, NUNK)

SEED = 20261203

# ---------------------------------------------------------------- Philox4x32-10
_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32(ctr, key):
    """Philox4x32-10 (Salmon et al., SC'11).  ctr: 4 uint32 arrays, key: 2 uint32."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint32) for c in ctr)
    k0, k1 = np.uint32(key[0]), np.uint32(key[1])
    with np.errstate(over="ignore"):
        for r in range(10):
            p0 = _M0 * c0.astype(np.uint64)
            p1 = _M1 * c2.astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & _MASK).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & _MASK).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            if r < 9:
                k0 = np.uint32((int(k0) + int(_W0)) & 0xFFFFFFFF)
                k1 = np.uint32((int(k1) + int(_W1)) & 0xFFFFFFFF)
    return c0, c1, c2, c3


def uniform01(index, stream=0, seed=SEED):
    """Two 53-bit uniforms in [0,1) per index: counter (index_lo, index_hi, stream, 0)."""
    idx = np.asarray(index, dtype=np.uint64)
    lo = (idx & _MASK).astype(np.uint32)
    hi = (idx >> np.uint64(32)).astype(np.uint32)
    z = np.zeros_like(lo)
    x0, x1, x2, x3 = philox4x32((lo, hi, z + np.uint32(stream), z), (seed, 0))
    a = ((x0 >> np.uint32(5)).astype(np.float64) * 67108864.0 + (x1 >> np.uint32(6)).astype(np.float64)) / 9007199254740992.0
    b = ((x2 >> np.uint32(5)).astype(np.float64) * 67108864.0 + (x3 >> np.uint32(6)).astype(np.float64)) / 9007199254740992.0
    return a, b


# ---------------------------------------------------------------- grid helpers
def cell_coords(geom: Geometry):
    """Global cell-centre and edge coordinates along each axis."""
    dx, dy, dz = geom.deltas()
    (x0, _), (y0, _), (z0, _) = geom.bbox
    nx = geom.nxb * geom.nblockx
    ny = geom.nyb * geom.nblocky if geom.ndim >= 2 else 1
    nz = geom.nzb * geom.nblockz if geom.ndim == 3 else 1
    gx, gy, gz = np.arange(nx), np.arange(ny), np.arange(nz)
    xc = x0 + (gx + 0.5) * dx
    yc = y0 + (gy + 0.5) * dy if geom.ndim >= 2 else np.zeros(1)
    zc = z0 + (gz + 0.5) * dz if geom.ndim == 3 else np.zeros(1)
    xl, xr = x0 + gx * dx, x0 + (gx + 1) * dx
    return xc, yc, zc, xl, xr


def scatter_global(geom: Geometry, field_zyx):
    """Global (nz, ny, nx, nvar) interior -> UNK with zeroed guard cells
    (nvar values per cell: UNK's, or the mass fractions of a species array)."""
    nv = field_zyx.shape[-1]
    unk = np.zeros(geom.unk_shape[:-1] + (nv,))
    g = geom.nguard
    nk, nj, ni = (geom.nzb if geom.ndim == 3 else 1), (geom.nyb if geom.ndim >= 2 else 1), geom.nxb
    gk, gj = (g if geom.ndim == 3 else 0), (g if geom.ndim >= 2 else 0)
    f = field_zyx.reshape(geom.nblockz if geom.ndim == 3 else 1, nk,
                          geom.nblocky if geom.ndim >= 2 else 1, nj, geom.nblockx, ni, nv)
    blocks = f.transpose(0, 2, 4, 1, 3, 5, 6).reshape(-1, nk, nj, ni, nv)
    unk[:, gk:gk + nk, gj:gj + nj, g:g + ni, :] = blocks
    return unk


def gather_global(geom: Geometry, unk):
    """UNK interiors -> global (nz, ny, nx, nvar) array."""
    g = geom.nguard
    nk, nj, ni = (geom.nzb if geom.ndim == 3 else 1), (geom.nyb if geom.ndim >= 2 else 1), geom.nxb
    gk, gj = (g if geom.ndim == 3 else 0), (g if geom.ndim >= 2 else 0)
    bz = geom.nblockz if geom.ndim == 3 else 1
    by = geom.nblocky if geom.ndim >= 2 else 1
    nv = unk.shape[-1]
    inner = unk[:, gk:gk + nk, gj:gj + nj, g:g + ni, :].reshape(bz, by, geom.nblockx, nk, nj, ni, nv)
    return inner.transpose(0, 3, 1, 4, 2, 5, 6).reshape(bz * nk, by * nj, geom.nblockx * ni, nv)


def eos_dens_ei(hp: HydroParams, u):
    """Eos_wrapped(MODE_DENS_EI) on a (..., NUNK) array (Eos_getData.F90:116-150,
    Gamma/Eos.F90:238-250, Eos_putData.F90:208-222)."""
    vx, vy, vz = u[..., VELX], u[..., VELY], u[..., VELZ]
    ekin = 0.5 * (vx * vx + vy * vy + vz * vz)
    eint = u[..., EINT].copy()
    cand = u[..., ENER] - ekin
    use = cand > np.maximum(hp.smalle, hp.eintSwitch * ekin)
    eint[use] = cand[use]
    dens = u[..., DENS]
    gammam1 = 1.0 / (hp.gamma - 1.0)
    ggprodinv = 1.0 / (gammam1 * hp.gasConstant)
    gam1inv = 1.0 / gammam1
    pres = dens * eint * gam1inv
    u[..., PRES] = pres
    u[..., TEMP] = eint * ggprodinv * hp.eos_singleSpeciesA
    u[..., GAMC] = hp.gamma
    u[..., EINT] = eint
    u[..., ENER] = eint + ekin
    u[..., GAME] = pres / (eint * dens) + 1.0
    return u


def _finish(hp, rho, vx, vy, vz, p, smallp_floor=True):
    f = np.zeros(rho.shape + (NUNK,))
    f[..., DENS], f[..., VELX], f[..., VELY], f[..., VELZ], f[..., PRES] = rho, vx, vy, vz, p
    ekin = 0.5 * (vx * vx + vy * vy + vz * vz)
    eint = p / (hp.gamma - 1.0)
    eint = eint / rho
    ener = eint + ekin
    if smallp_floor:
        ener = np.maximum(ener, hp.smallp)
    f[..., ENER], f[..., EINT] = ener, eint
    f[..., GAMC], f[..., GAME], f[..., TEMP] = hp.gamma, hp.gamma, 1.0e-10
    return eos_dens_ei(hp, f)


# ---------------------------------------------------------------- problems
def sod(geom: Geometry, hp: HydroParams, rho_l=1.0, rho_r=0.125, p_l=1.0, p_r=0.1,
        xangle=45.0, yangle=45.0, posn=1.0):
    """Sod shock tube at an angle (Sod/Simulation_initBlock.F90)."""
    xa = xangle * 0.0174532925
    ya = yangle * 0.0174532925
    xcos = math.cos(xa)
    if geom.ndim == 1:
        xcos, ycos, zcos = 1.0, 0.0, 0.0
    elif geom.ndim == 2:
        ycos, zcos = math.sqrt(1.0 - xcos * xcos), 0.0
    else:
        ycos = math.cos(ya)
        zcos = math.sqrt(max(0.0, 1.0 - xcos * xcos - ycos * ycos))
    xc, yc, zc, xl, xr = cell_coords(geom)
    Z, Y, XL = np.meshgrid(zc, yc, xl, indexing="ij")
    XR = np.broadcast_to(xr, XL.shape)
    lposn = (posn - Z * zcos / xcos) - Y * ycos / xcos
    left = XR <= lposn
    mid = (XL < lposn) & (XR > lposn)
    rho = np.where(left, rho_l, np.where(mid, 0.5 * (rho_l + rho_r), rho_r))
    p = np.where(left, p_l, np.where(mid, 0.5 * (p_l + p_r), p_r))
    zero = np.zeros_like(rho)
    return scatter_global(geom, _finish(hp, rho, zero, zero, zero, p))


def kelvin_helmholtz(geom: Geometry, hp: HydroParams, amp=0.01):
    """Periodic shear layer: rho=2, vx=+0.5 for |y-0.5|<0.25, else rho=1,
    vx=-0.5; p=2.5; vy = amp * U(-1,1) * sin(4 pi x)."""
    xc, yc, zc, _, _ = cell_coords(geom)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    inner = np.abs(Y - 0.5) < 0.25
    rho = np.where(inner, 2.0, 1.0)
    vx = np.where(inner, 0.5, -0.5)
    idx = np.arange(X.size, dtype=np.uint64).reshape(X.shape)
    u, _ = uniform01(idx)
    vy = amp * (2.0 * u - 1.0) * np.sin(4.0 * math.pi * X)
    p = np.full_like(rho, 2.5)
    return scatter_global(geom, _finish(hp, rho, vx, vy, np.zeros_like(rho), p))


def rayleigh_taylor(geom: Geometry, hp: HydroParams, g=-0.1, p0=2.5, amp=0.01, nmodes=16):
    """Heavy (rho=2) over light (rho=1) fluid at z=0.5 in hydrostatic balance
    under constant gravity g in z; vz = amp * sum of nmodes random-phase
    Fourier modes times a Gaussian envelope around the interface.  In 2-D the
    vertical axis is y (interface at y=0.5, vy perturbed by modes in x)."""
    xc, yc, zc, _, _ = cell_coords(geom)
    if geom.ndim == 2:
        Zc, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
        heavy = Y > 0.5
        rho = np.where(heavy, 2.0, 1.0)
        p = np.where(heavy, p0 + 2.0 * g * (Y - 0.5), p0 + 1.0 * g * (Y - 0.5))
        a, _ = uniform01(np.arange(nmodes, dtype=np.uint64), stream=1)
        c, _ = uniform01(np.arange(nmodes, dtype=np.uint64), stream=2)
        kx = 1.0 + np.floor(4.0 * a)
        s = np.zeros_like(X)
        for m in range(nmodes):
            s += np.sin(2.0 * math.pi * kx[m] * X + 2.0 * math.pi * c[m])
        vy = amp * s * np.exp(-((Y - 0.5) / 0.1) ** 2)
        zero = np.zeros_like(rho)
        return scatter_global(geom, _finish(hp, rho, zero, vy, zero, p))
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    heavy = Z > 0.5
    rho = np.where(heavy, 2.0, 1.0)
    p = np.where(heavy, p0 + 2.0 * g * (Z - 0.5), p0 + 1.0 * g * (Z - 0.5))
    a, b = uniform01(np.arange(nmodes, dtype=np.uint64), stream=1)
    c, _ = uniform01(np.arange(nmodes, dtype=np.uint64), stream=2)
    kx = 1.0 + np.floor(4.0 * a)
    ky = 1.0 + np.floor(4.0 * b)
    phi = 2.0 * math.pi * c
    s = np.zeros_like(X)
    for m in range(nmodes):
        s += np.sin(2.0 * math.pi * (kx[m] * X + ky[m] * Y) + phi[m])
    vz = amp * s * np.exp(-((Z - 0.5) / 0.1) ** 2)
    zero = np.zeros_like(rho)
    return scatter_global(geom, _finish(hp, rho, zero, zero, vz, p))


def noisy_gas(geom: Geometry, hp: HydroParams, vmag=0.1, noise=0.05):
    """Uniform rho=1, p=1, |v|=vmag in a random direction, each field times
    (1 + noise*N(0,1)) from Philox + Box-Muller."""
    xc, yc, zc, _, _ = cell_coords(geom)
    shape = (len(zc), len(yc), len(xc))
    idx = np.arange(int(np.prod(shape)), dtype=np.uint64).reshape(shape)
    def normal(stream):
        u1, u2 = uniform01(idx, stream=stream)
        return np.sqrt(-2.0 * np.log(1.0 - u1)) * np.cos(2.0 * math.pi * u2)
    u1, u2 = uniform01(idx, stream=10)
    cost = 2.0 * u1 - 1.0
    sint = np.sqrt(np.maximum(0.0, 1.0 - cost * cost))
    ph = 2.0 * math.pi * u2
    dirx, diry, dirz = sint * np.cos(ph), sint * np.sin(ph), cost
    if geom.ndim == 2:
        dirx, diry, dirz = np.cos(ph), np.sin(ph), np.zeros_like(ph)
    rho = 1.0 * (1.0 + noise * normal(11))
    p = 1.0 * (1.0 + noise * normal(12))
    vm = vmag * (1.0 + noise * normal(13))
    return scatter_global(geom, _finish(hp, rho, vm * dirx, vm * diry, vm * dirz, p))


def noisy_gas_blocks(geom: Geometry, hp: HydroParams, bcoords, out, vmag=0.1, noise=0.05, chunk=2048, threads=1):
    """noisy_gas's values for the listed blocks of a 3-D `geom`, written
    block chunk by block chunk into the UNK `out` (len(bcoords), k, j, i, var)
    (guard cells untouched): the same global cell indices, so the same values,
    without a copy of the whole grid.  threads > 1 fills disjoint chunks
    concurrently."""
    nbx, nby, nbz = geom.nxb, geom.nyb, geom.nzb
    nx, ny = nbx * geom.nblockx, nby * geom.nblocky
    dx, dy, dz = geom.deltas()
    g = geom.nguard
    kk, jj, ii = np.meshgrid(np.arange(nbz), np.arange(nby), np.arange(nbx), indexing="ij")
    bc = np.asarray(bcoords, dtype=np.int64)

    def fill(c0):
        b = bc[c0:c0 + chunk]
        gi = b[:, 0, None, None, None] * nbx + ii
        gj = b[:, 1, None, None, None] * nby + jj
        gk = b[:, 2, None, None, None] * nbz + kk
        idx = ((gk * ny + gj) * nx + gi).astype(np.uint64)

        def normal(stream):
            u1, u2 = uniform01(idx, stream=stream)
            return np.sqrt(-2.0 * np.log(1.0 - u1)) * np.cos(2.0 * math.pi * u2)
        u1, u2 = uniform01(idx, stream=10)
        cost = 2.0 * u1 - 1.0
        sint = np.sqrt(np.maximum(0.0, 1.0 - cost * cost))
        ph = 2.0 * math.pi * u2
        dirx, diry, dirz = sint * np.cos(ph), sint * np.sin(ph), cost
        rho = 1.0 * (1.0 + noise * normal(11))
        p = 1.0 * (1.0 + noise * normal(12))
        vm = vmag * (1.0 + noise * normal(13))
        out[c0:c0 + len(b), g:g + nbz, g:g + nby, g:g + nbx, :] = _finish(hp, rho, vm * dirx, vm * diry, vm * dirz, p)
    starts = range(0, len(bc), chunk)
    if threads > 1:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(fill, starts))
    else:
        for c0 in starts:
            fill(c0)
    return out


# ---------------------------------------------------------------- configurations
def species_blob(geom: Geometry, ns=3, nspecies=2, center=(0.5, 0.5, 0.5), radius=0.2, width=0.03):
    """Advected mass fractions, (blk, k, j, i, ns) like UNK: species 0 is a
    smoothed disc (sphere in 3-D) of `radius` around `center`, species 1 its
    complement (the species add up to one), further values mass scalars
    0.3 + 0.2 sin(2 pi x) sin(2 pi y) (not renormalised)."""
    xc, yc, zc, _, _ = cell_coords(geom)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    r2 = (X - center[0]) ** 2 + (Y - center[1]) ** 2
    if geom.ndim == 3:
        r2 = r2 + (Z - center[2]) ** 2
    blob = 0.5 * (1.0 - np.tanh((np.sqrt(r2) - radius) / width))
    f = np.zeros(X.shape + (ns,))
    f[..., 0] = blob
    if nspecies > 1:
        f[..., 1] = 1.0 - blob
    for q in range(nspecies, ns):
        f[..., q] = 0.3 + 0.2 * np.sin(2 * math.pi * X) * np.sin(2 * math.pi * Y) + 0.01 * q
    return scatter_global(geom, f)


def config(name, scale=1):
    """(Geometry, HydroParams, init function) for a named benchmark problem.
    scale < 1 shrinks the block count per axis for quick parity cases."""
    if name == "sod2d":
        nb = max(1, int(16 * scale))
        geom = Geometry(2, 16, 16, 1, nb, nb, 1, bc=(BC_OUTFLOW,) * 6)
        return geom, HydroParams(), sod
    if name == "kh2d":
        nb = max(1, int(128 * scale))
        geom = Geometry(2, 16, 16, 1, nb, nb, 1, bc=(BC_PERIODIC,) * 6)
        return geom, HydroParams(), kelvin_helmholtz
    if name == "rt3d":
        nb = max(1, int(16 * scale))
        geom = Geometry(3, 16, 16, 16, nb, nb, nb,
                        bc=(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING))
        hp = HydroParams(order=5, useGravity=True, gravity=(0.0, 0.0, -0.1))
        return geom, hp, rayleigh_taylor
    if name == "rt2d":
        nb = max(1, int(16 * scale))
        geom = Geometry(2, 16, 16, 1, nb, nb, 1,
                        bc=(BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING, BC_OUTFLOW, BC_OUTFLOW))
        hp = HydroParams(useGravity=True, gravity=(0.0, -0.1, 0.0))
        return geom, hp, rayleigh_taylor
    if name == "sweep3d":
        nb = max(1, int(4 * scale))
        geom = Geometry(3, 16, 16, 16, nb, nb, nb, bc=(BC_PERIODIC,) * 6)
        return geom, HydroParams(gamma=5.0 / 3.0), noisy_gas
    raise KeyError(name)
