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


def _slab_worker(name, rank, world, port, outdir):
    import os
    import sys
    import traceback
    root_dir = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root_dir, os.path.join(root_dir, "flash-x_b200"), os.path.join(root_dir, "tests"),
                    os.path.join(root_dir, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK="0")
    result = "ok"
    try:
        import torch
        from flashx_b200 import parallel as P
        from flashx_b200.hydro import driver_dt
        torch.cuda.set_device(0)
        P.init_from_env("gloo", timeout_s=120)
        geom, hp, unk = C.case(name)
        dec = SlabDecomposition(geom, world, rank)
        b0, b1 = dec.block_range()
        dev = HydroDevice(geom, hp, "fp64", slab=dec)
        dev.attach_unk(np.ascontiguousarray(unk[b0:b1]))
        dt = dt_old = 0.5 * P.allreduce_min(dev.Hydro_computeDt())
        dts = [dt]
        for _ in range(NSTEPS):
            dev.Hydro(0.0, dt, dt_old)
            dt_old, dt = dt, driver_dt(P.allreduce_min(dev.Hydro_computeDt()), dt, hp)
            dts.append(dt)
        out = np.zeros(dev.unk_shape)
        dev.sync_to_host(out)
        integ = P.allreduce_sum(dev.integrals())
        np.savez(os.path.join(outdir, f"{name}{rank}.npz"), out=out, b0=b0, b1=b1, dts=np.array(dts),
                 integ=np.array(integ))
        dev.close()
    except Exception as e:  # noqa: BLE001
        result = f"error: {type(e).__name__}: {e}\n{traceback.format_exc()}"
    with open(os.path.join(outdir, f"{name}{rank}.txt"), "w") as f:
        f.write(result)
    try:
        import torch.distributed as dist
        if dist.is_initialized() and result == "ok":
            dist.destroy_process_group()
    except Exception:
        pass


@pytest.mark.parametrize("name", ["kh2d", "sod2d", "rt3d"])
def test_two_slabs_on_one_gpu_match_whole_grid(name, oracle, need_gpu):
    """Two ranks, as two processes sharing the GPU and a gloo group (their
    halo planes cross through pinned host copies; no kernel of one waits for
    the other), each stepping its slab with the real exchange (KH: each rank
    is both neighbours of the other across the periodic axis): the slabs, the
    reduced dt sequence and integrals equal the oracle on the whole grid."""
    import multiprocessing as mp
    import os
    import socket
    import tempfile
    world = 2
    out = tempfile.mkdtemp()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_slab_worker, args=(name, r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert not p.is_alive(), "a rank did not finish"
    for r in range(world):
        with open(os.path.join(out, f"{name}{r}.txt")) as f:
            assert f.read() == "ok"
    geom, hp, unk = C.case(name)
    whole, dts = C.whole_run(oracle, geom, hp, unk, NSTEPS)
    ref = oracle.integrals(oracle.make_params(geom.as_dict(), hp), whole)
    for r in range(world):
        d = np.load(os.path.join(out, f"{name}{r}.npz"))
        assert list(d["dts"]) == dts
        b0, b1 = int(d["b0"]), int(d["b1"])
        np.testing.assert_array_equal(_inner(geom, d["out"])[..., C.DEV_VARS], _inner(geom, whole[b0:b1])[..., C.DEV_VARS])
        np.testing.assert_allclose(d["integ"], ref, rtol=1e-12, atol=1e-12)
