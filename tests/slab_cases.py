"""Slab-decomposition cases shared by the CPU (gloo, oracle ranks) and GPU
tests: small uniform grids whose cell widths are powers of two, so that a
slab's own geometry (its layers plus halo planes) has bit-identical cell
widths, and the oracle on a slab, fed halo planes from its neighbours,
must reproduce the oracle on the whole grid exactly."""
import numpy as np

from flashx_b200 import simulations as S
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, DENS, EINT, ENER, GAMC, GAME,
                                Geometry, HydroParams, NUNK, PRES, TEMP, VELX, VELY, VELZ)

# device variable order of the halo messages (fxb_halo_pack)
DEV_VARS = (DENS, VELX, VELY, VELZ, PRES, GAMC, GAME, EINT, ENER, TEMP)


def case(name):
    """(whole-grid Geometry, HydroParams, initial UNK of the whole grid)."""
    if name == "kh2d":        # periodic in y: every slab has two neighbours
        geom = Geometry(2, 8, 4, 1, 4, 12, 1, bbox=((0.0, 1.0), (0.0, 1.5), (0.0, 1.0)), bc=(BC_PERIODIC,) * 6)
        hp = HydroParams()
        return geom, hp, S.kelvin_helmholtz(geom, hp)
    if name == "sod2d":       # outflow in y: the end slabs have one neighbour
        geom = Geometry(2, 8, 4, 1, 4, 8, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams()
        return geom, hp, S.sod(geom, hp)
    if name == "gas3d":       # periodic in z, PPM
        geom = Geometry(3, 8, 8, 4, 2, 2, 4, bc=(BC_PERIODIC,) * 6)
        hp = HydroParams(gamma=5.0 / 3.0)
        return geom, hp, S.noisy_gas(geom, hp)
    if name == "rt3d":        # reflecting in z, gravity, WENO5
        geom = Geometry(3, 8, 8, 4, 2, 2, 4,
                        bc=(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING))
        hp = HydroParams(order=5, useGravity=True, gravity=(0.0, 0.0, -0.1))
        return geom, hp, S.rayleigh_taylor(geom, hp)
    raise KeyError(name)


def _axis_extent(geom):
    return (geom.nblocky, geom.nyb) if geom.ndim == 2 else (geom.nblockz, geom.nzb)


def sub_geometry(geom, first_plane, nplanes, bc_lo, bc_hi):
    """Geometry of planes [first_plane, first_plane + nplanes) of the slowest
    axis (whole block layers), with the given boundary handling there."""
    nlay, nb = _axis_extent(geom)
    assert first_plane % nb == 0 and nplanes % nb == 0
    ax = geom.ndim - 1
    d = geom.deltas()[ax]
    lo = geom.bbox[ax][0] + first_plane * d
    bbox = list(geom.bbox)
    bbox[ax] = (lo, lo + nplanes * d)
    bc = list(geom.bc)
    bc[2 * ax], bc[2 * ax + 1] = bc_lo, bc_hi
    kw = dict(bbox=tuple(bbox), bc=tuple(bc), nguard=geom.nguard)
    if geom.ndim == 2:
        return Geometry(2, geom.nxb, geom.nyb, 1, geom.nblockx, nplanes // nb, 1, **kw)
    return Geometry(3, geom.nxb, geom.nyb, geom.nzb, geom.nblockx, geom.nblocky, nplanes // nb, **kw)


class OracleSlab:
    """One rank's slab run by the oracle: its layers plus the halo planes as
    whole block layers of a grid of their own (outflow beyond a halo, which
    only feeds halo cells), packed and unpacked through the same message
    layout as the device: variable-major planes of the 10 device variables."""

    def __init__(self, O, geom, hp, dec, whole_unk):
        nlay, nb = _axis_extent(geom)
        self.geom, self.dec, self.nb = geom, dec, nb
        hl, hh = dec.halo_lo, dec.halo_hi
        assert hl % nb == 0 and hh % nb == 0, "oracle slabs need halos of whole block layers"
        ax = geom.ndim - 1
        first = dec.layer_lo * nb - hl
        self.nplanes = dec.interior_planes() + hl + hh
        bc_lo = BC_OUTFLOW if hl else geom.bc[2 * ax]
        bc_hi = BC_OUTFLOW if hh else geom.bc[2 * ax + 1]
        self.lgeom = sub_geometry(geom, first % (nlay * nb), self.nplanes, bc_lo, bc_hi)
        self.igeom = sub_geometry(geom, dec.layer_lo * nb, dec.interior_planes(), bc_lo, bc_hi)
        per = dec.per_layer
        layers = [(first // nb + i) % nlay for i in range(self.nplanes // nb)]
        self.unk = np.ascontiguousarray(np.concatenate([whole_unk[l * per:(l + 1) * per] for l in layers]))
        self.p = O.make_params(self.lgeom.as_dict(), hp)
        self.pi = O.make_params(self.igeom.as_dict(), hp)
        self.i0, self.i1 = (hl // nb) * per, (hl // nb + dec.layers[dec.rank][1] - dec.layers[dec.rank][0]) * per
        self.O = O

    # planes of the stored slab, slowest axis first: (planes, cells of a plane, NUNK)
    def _planes(self):
        return S.gather_global(self.lgeom, self.unk).reshape(self.nplanes, -1, NUNK)

    def _store(self, planes):
        shape = S.gather_global(self.lgeom, self.unk).shape
        self.unk[...] = S.scatter_global(self.lgeom, planes.reshape(shape))

    @staticmethod
    def message(planes):
        """(n, cells, NUNK) -> variable-major flat message of the device variables."""
        return np.ascontiguousarray(planes[:, :, list(DEV_VARS)].transpose(2, 0, 1)).reshape(-1)

    def pack(self, send_lo, n_lo, send_hi, n_hi):
        pl = self._planes()
        hl, n = self.dec.halo_lo, self.dec.interior_planes()
        import torch
        if n_lo:
            send_lo.copy_(torch.from_numpy(self.message(pl[hl:hl + n_lo])))
        if n_hi:
            send_hi.copy_(torch.from_numpy(self.message(pl[hl + n - n_hi:hl + n])))

    def unpack(self, recv_lo, recv_hi):
        pl = self._planes()
        hl, hh, n = self.dec.halo_lo, self.dec.halo_hi, self.dec.interior_planes()
        cells = pl.shape[1]
        for buf, sl in ((recv_lo, slice(0, hl)), (recv_hi, slice(hl + n, hl + n + hh))):
            if buf is None:
                continue
            m = buf.numpy().reshape(len(DEV_VARS), -1, cells)
            for k, v in enumerate(DEV_VARS):
                pl[sl, :, v] = m[k]
        self._store(pl)

    def interior(self):
        return np.ascontiguousarray(self.unk[self.i0:self.i1])

    def step(self, dt, dt_old):
        self.O.hydro_step(self.p, self.unk, dt, dt_old)

    def compute_dt(self):
        return self.O.compute_dt(self.pi, self.interior())

    def integrals(self):
        return self.O.integrals(self.pi, self.interior())


def whole_run(O, geom, hp, unk, nsteps):
    """The oracle on the whole grid: (final UNK, dt sequence)."""
    p = O.make_params(geom.as_dict(), hp)
    unk = unk.copy()
    dt = dt_old = 0.5 * O.compute_dt(p, unk)
    dts = [dt]
    for _ in range(nsteps):
        O.hydro_step(p, unk, dt, dt_old)
        dt_old, dt = dt, O.driver_dt(O.compute_dt(p, unk), dt)
        dts.append(dt)
    return unk, dts
