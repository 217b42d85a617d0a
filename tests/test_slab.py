"""CPU tests of the slab decomposition of a uniform grid over ranks
(flashx_b200.parallel.SlabDecomposition / HaloExchange, the one-axis case of
UG's process grid and its guard-cell exchange, Grid/GridMain/UG/
Grid_fillGuardCells.F90:261-306 and UG/gr_shiftData.F90:63-191).

The split itself is checked directly.  The exchange runs as gloo ranks
(world size 2 and 3) whose slabs are stepped by the oracle: after several
steps every rank's cells, and the common dt sequence, must equal the oracle
on the whole grid bit for bit, which holds only if the halos carry the right
planes from the right neighbour and are wide enough for one step's stencil."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from flashx_b200.params import BC_OUTFLOW, BC_PERIODIC, Geometry


def _geom2d(nby, bc=BC_PERIODIC, nyb=16):
    return Geometry(2, 16, nyb, 1, 4, nby, 1, bc=(bc,) * 6)


def test_layers_cover_the_grid_once():
    from flashx_b200.parallel import SlabDecomposition
    for nranks in (1, 2, 3, 5, 8):
        d = SlabDecomposition(_geom2d(8, nyb=16), nranks, 0)
        flat = [l for lo, hi in d.layers for l in range(lo, hi)]
        assert flat == list(range(8))
        sizes = [hi - lo for lo, hi in d.layers]
        assert max(sizes) - min(sizes) <= 1


def test_halo_widths_2d_tiles():
    from flashx_b200.parallel import SlabDecomposition
    # periodic: two halos, widened from NGUARD=4 to 8 so that 16-cell tiles fill the slab
    d = SlabDecomposition(_geom2d(8), 4, 1)
    assert d.halos == [(8, 8)] * 4
    assert (d.interior_planes() + d.halo_lo + d.halo_hi) % 16 == 0
    # outflow: the end slabs have one halo of 16 planes, the middle ones two of 8
    d = SlabDecomposition(_geom2d(8, BC_OUTFLOW), 3, 0)
    assert d.halos == [(0, 16), (8, 8), (16, 0)]
    # one rank: no halo unless it exchanges with itself across the periodic axis
    assert SlabDecomposition(_geom2d(8), 1, 0).halos == [(0, 0)]
    assert SlabDecomposition(_geom2d(8), 1, 0, self_halo=True).halos == [(8, 8)]
    assert SlabDecomposition(_geom2d(8, BC_OUTFLOW), 1, 0, self_halo=True).halos == [(0, 0)]


def test_halo_widths_3d_and_message_pairing():
    from flashx_b200.parallel import SlabDecomposition
    g = Geometry(3, 16, 16, 16, 2, 2, 6, bc=(BC_PERIODIC,) * 6)
    decs = [SlabDecomposition(g, 3, r) for r in range(3)]
    for d in decs:
        assert (d.halo_lo, d.halo_hi) == (4, 4)
        assert d.block_range() == (d.layer_lo * 4, d.layer_hi * 4)
    # what a rank sends down fills its lower neighbour's upper halo, and up its upper neighbour's lower halo
    for d in decs:
        assert d.send_lo == decs[d.lo_rank].halo_hi
        assert d.send_hi == decs[d.hi_rank].halo_lo
        assert decs[d.lo_rank].hi_rank == d.rank and decs[d.hi_rank].lo_rank == d.rank


def test_decomposition_rejects_bad_splits():
    from flashx_b200.parallel import SlabDecomposition
    with pytest.raises(ValueError):
        SlabDecomposition(_geom2d(4), 5, 0)          # more ranks than block layers
    with pytest.raises(ValueError):
        SlabDecomposition(_geom2d(8, nyb=4), 8, 0)   # 8-plane halos from 4-plane neighbours
    with pytest.raises(ValueError):
        SlabDecomposition(_geom2d(8), 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


NSTEPS = 6


def _worker(rank, world, port, outdir, name):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "flash-x_b200"), os.path.join(root, "tests")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    result = "ok"
    try:
        from flashx_b200 import parallel as P
        from oracle import fx_oracle as O
        import slab_cases as C
        P.init_from_env("gloo", timeout_s=60)
        geom, hp, unk = C.case(name)
        dec = P.SlabDecomposition(geom, world, rank, tile=1)
        sl = C.OracleSlab(O, geom, hp, dec, unk)
        plane = sl.lgeom.nxb * sl.lgeom.nblockx * (sl.lgeom.nyb * sl.lgeom.nblocky if geom.ndim == 3 else 1)
        ex = P.HaloExchange(dec, len(C.DEV_VARS) * plane, sl.pack, sl.unpack)
        dt = dt_old = 0.5 * P.allreduce_min(sl.compute_dt())
        dts = [dt]
        for _ in range(NSTEPS):
            ex()
            sl.step(dt, dt_old)
            dt_old, dt = dt, O.driver_dt(P.allreduce_min(sl.compute_dt()), dt)
            dts.append(dt)
        sums = P.allreduce_sum(sl.integrals())
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), interior=sl.interior(), dts=np.array(dts),
                 sums=np.array(sums), b0=dec.block_range()[0], b1=dec.block_range()[1])
    except Exception as e:  # noqa: BLE001
        import traceback
        result = f"error: {type(e).__name__}: {e}\n{traceback.format_exc()}"
    with open(os.path.join(outdir, f"result{rank}.txt"), "w") as f:
        f.write(result)
    try:
        import torch.distributed as dist
        if dist.is_initialized() and result == "ok":
            dist.destroy_process_group()
    except Exception:
        pass


@pytest.mark.parametrize("name,world", [("kh2d", 3), ("sod2d", 2), ("gas3d", 2), ("rt3d", 3)])
def test_slabs_reproduce_the_whole_grid_gloo(name, world, oracle):
    import slab_cases as C
    out = tempfile.mkdtemp()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out, name)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        if p.is_alive():
            p.kill()
            pytest.fail("slab worker did not finish")
    res = [open(os.path.join(out, f"result{r}.txt")).read() for r in range(world)]
    assert res == ["ok"] * world, res
    geom, hp, unk = C.case(name)
    whole, dts = C.whole_run(oracle, geom, hp, unk, NSTEPS)
    g = geom.nguard
    inner = (slice(None), slice(g, -g) if geom.ndim == 3 else slice(None), slice(g, -g), slice(g, -g))
    covered = 0
    for r in range(world):
        z = np.load(os.path.join(out, f"rank{r}.npz"))
        b0, b1 = int(z["b0"]), int(z["b1"])
        assert np.array_equal(z["dts"], np.array(dts)), (r, z["dts"], dts)
        np.testing.assert_array_equal(z["interior"][inner], whole[b0:b1][inner])
        covered += b1 - b0
        sums = z["sums"]
    assert covered == geom.nblocks
    # the integrals summed over ranks equal the whole grid's (up to summation order)
    ref = oracle.integrals(oracle.make_params(geom.as_dict(), hp), whole)
    np.testing.assert_allclose(sums, ref, rtol=1e-12, atol=1e-12)
