"""GPU tests of a slab of a uniform grid (fxb_init_slab, fxb_halo_pack,
fxb_halo_unpack; the guard-cell exchange of Grid/GridMain/UG/
Grid_fillGuardCells.F90:261-306) on one B200, without a second rank:

* a single slab that is its own neighbour across a periodic axis packs its
  boundary planes straight into its halos (the whole device path of an
  exchange, halo-aware kernels, dt and integrals over the slab's own
  cells), and must match the oracle on the whole grid bit for bit;
* one slab of a two-slab split whose neighbour is played by the oracle on
  the whole grid: before every step the device's packed planes must equal
  the oracle's, the oracle's neighbouring planes go into the halo, and the
  slab's cells and CFL dt must match the oracle bit for bit.

The exchange between ranks itself (message pairing, tags, periodic wrap) is
covered by the gloo tests in test_slab.py."""
import numpy as np
import pytest

import slab_cases as C
from flashx_b200 import simulations as S
from flashx_b200.hydro import HydroDevice
from flashx_b200.parallel import SlabDecomposition

pytestmark = pytest.mark.gpu
NSTEPS = 6


def _inner(geom, unk):
    g = geom.nguard
    return unk[:, g:-g, g:-g, g:-g] if geom.ndim == 3 else unk[:, :, g:-g, g:-g]


@pytest.mark.parametrize("name", ["kh2d", "gas3d"])
def test_self_exchanging_slab_matches_whole_grid_fp64(name, oracle, need_gpu):
    geom, hp, unk = C.case(name)
    dec = SlabDecomposition(geom, 1, 0, self_halo=True)
    assert dec.halo_lo > 0 and dec.halo_hi > 0
    whole, dts = C.whole_run(oracle, geom, hp, unk, NSTEPS)
    dev = HydroDevice(geom, hp, "fp64", slab=dec)
    dev.attach_unk(unk.copy())
    dt = dt_old = 0.5 * dev.Hydro_computeDt()
    got = [dt]
    for _ in range(NSTEPS):
        dev.Hydro(0.0, dt, dt_old)
        dt_old, dt = dt, oracle.driver_dt(dev.Hydro_computeDt(), dt)
        got.append(dt)
    assert got == dts
    out = np.zeros(geom.unk_shape)
    dev.sync_to_host(out)
    np.testing.assert_array_equal(_inner(geom, out), _inner(geom, whole))
    ref = oracle.integrals(oracle.make_params(geom.as_dict(), hp), whole)
    np.testing.assert_allclose(dev.integrals(), ref, rtol=1e-12, atol=1e-12)
    # the guard cells next to the halos come from the exchanged planes
    p = oracle.make_params(geom.as_dict(), hp)
    oracle.fill_guardcells(p, whole)
    np.testing.assert_array_equal(out[..., C.DEV_VARS], whole[..., C.DEV_VARS])
    dev.close()


class _OracleNeighbour:
    """Stands in for HaloExchange: checks the device's packed planes against
    the whole-grid oracle and fills the halos with the oracle's planes."""

    def __init__(self, dev, dec, geom):
        import torch
        self.dev, self.dec, self.geom = dev, dec, geom
        n = dev.lib.fxb_halo_doubles(1)
        cuda = torch.device("cuda")
        mk = lambda k: torch.empty(k * n, dtype=torch.float64, device=cuda) if k else None
        self.send = (mk(dec.send_lo), mk(dec.send_hi))
        self.recv = (mk(dec.halo_lo), mk(dec.halo_hi))
        self.whole = None
        self.checked = 0

    def _planes(self, lo, hi):
        g = S.gather_global(self.geom, self.whole)
        return g.reshape(g.shape[0], -1, g.shape[-1])[lo:hi] if self.geom.ndim == 3 else \
            g.reshape(g.shape[1], -1, g.shape[-1])[lo:hi]

    def __call__(self):
        import ctypes
        import torch
        lib, d, nb = self.dev.lib, self.dec, self.dec.nb
        ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
        assert lib.fxb_halo_pack(ptr(self.send[0]), d.send_lo, ptr(self.send[1]), d.send_hi) == 0
        torch.cuda.synchronize()
        lo, hi = d.layer_lo * nb, d.layer_hi * nb
        if d.send_lo:
            want = C.OracleSlab.message(self._planes(lo, lo + d.send_lo))
            np.testing.assert_array_equal(self.send[0].cpu().numpy(), want)
            self.checked += 1
        if d.send_hi:
            want = C.OracleSlab.message(self._planes(hi - d.send_hi, hi))
            np.testing.assert_array_equal(self.send[1].cpu().numpy(), want)
            self.checked += 1
        if d.halo_lo:
            self.recv[0].copy_(torch.from_numpy(C.OracleSlab.message(self._planes(lo - d.halo_lo, lo))))
        if d.halo_hi:
            self.recv[1].copy_(torch.from_numpy(C.OracleSlab.message(self._planes(hi, hi + d.halo_hi))))
        torch.cuda.synchronize()
        assert lib.fxb_halo_unpack(ptr(self.recv[0]), ptr(self.recv[1])) == 0


@pytest.mark.parametrize("name,rank", [("sod2d", 0), ("sod2d", 1), ("rt3d", 1)])
def test_slab_with_oracle_neighbour_fp64(name, rank, oracle, need_gpu):
    geom, hp, unk = C.case(name)
    dec = SlabDecomposition(geom, 2, rank)
    p = oracle.make_params(geom.as_dict(), hp)
    b0, b1 = dec.block_range()
    ip = oracle.make_params(C.sub_geometry(geom, dec.layer_lo * dec.nb, dec.interior_planes(),
                                           geom.bc[2 * dec.axis], geom.bc[2 * dec.axis + 1]).as_dict(), hp)
    dev = HydroDevice(geom, hp, "fp64", slab=dec)
    nbr = _OracleNeighbour(dev, dec, geom)
    dev.exchange = nbr
    dev.attach_unk(np.ascontiguousarray(unk[b0:b1]))
    whole = unk.copy()
    nbr.whole = whole
    dt = dt_old = 0.5 * oracle.compute_dt(p, whole)
    for _ in range(NSTEPS):
        dev.Hydro(0.0, dt, dt_old)                   # exchange, then the step
        oracle.hydro_step(p, whole, dt, dt_old)
        local = dev.Hydro_computeDt()
        assert local == oracle.compute_dt(ip, np.ascontiguousarray(whole[b0:b1]))
        dt_old, dt = dt, oracle.driver_dt(oracle.compute_dt(p, whole), dt)
    out = np.zeros((b1 - b0,) + geom.block_shape)
    dev.sync_to_host(out)
    np.testing.assert_array_equal(_inner(geom, out), _inner(geom, whole[b0:b1]))
    assert nbr.checked >= NSTEPS
    dev.close()
