"""CPU tests of checkpoint, restart and comparison (flashx_b200.checkpoint;
the datasets of Flash-X's IO_writeCheckpoint / IO_readCheckpoint in an .npz
container, and sfocu-style comparison): round trips of uniform and AMR
states, restarts that continue bit for bit, and the comparison report."""
import os
import tempfile

import numpy as np
import pytest

from flashx_b200 import amr as A
from flashx_b200 import checkpoint as C
from flashx_b200 import simulations as S
from flashx_b200.params import BC_PERIODIC, DENS, Geometry, HydroParams


def _tmp(name):
    return os.path.join(tempfile.mkdtemp(), name)


def _inner(geom, unk):
    g = geom.nguard
    return unk[:, g:-g, g:-g, g:-g] if geom.ndim == 3 else unk[:, :, g:-g, g:-g]


def test_uniform_round_trip_and_scalars():
    geom, hp, init = S.config("kh2d", scale=1 / 32)
    hp = HydroParams(order=5, RiemannSolver="HLL", use_avisc=True, cvisc=0.2)
    unk = init(geom, hp)
    path = _tmp("kh.npz")
    C.write_checkpoint(path, geom, hp, unk, time=0.125, dt=1e-3, dtold=9e-4, nstep=42)
    ck = C.read_checkpoint(path)
    assert ck["geom"] == geom and ck["hp"] == hp
    assert (ck["nstep"], ck["time"], ck["dt"], ck["dtold"]) == (42, 0.125, 1e-3, 9e-4)
    np.testing.assert_array_equal(_inner(geom, ck["unk"]), _inner(geom, unk))
    assert C.restart_mesh(ck) is None
    z = np.load(path)
    assert list(z["dens"].shape) == [geom.nblocks, 1, geom.nyb, geom.nxb]
    assert np.all(z["node type"] == 1) and np.all(z["refine level"] == 1)


def test_amr_round_trip():
    geom = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams()
    mesh, unk = A.levelset_problem(geom, hp, maxlev=2)
    path = _tmp("amr.npz")
    C.write_checkpoint(path, geom, hp, unk, mesh=mesh, time=1.0, dt=0.1, dtold=0.1, nstep=3)
    ck = C.read_checkpoint(path)
    m2 = C.restart_mesh(ck)
    assert np.array_equal(m2.levels, mesh.levels) and np.array_equal(m2.bcoords, mesh.bcoords)
    np.testing.assert_array_equal(_inner(geom, ck["unk"]), _inner(geom, unk))
    z = np.load(path)
    lv = z["refine level"]
    assert np.allclose(z["block size"][:, 0], 1.0 / (2 * 2.0 ** (lv - 1)))


def test_compare_reports_differences():
    geom, hp, init = S.config("sod2d", scale=1 / 8)
    unk = init(geom, hp)
    a, b = _tmp("a.npz"), _tmp("b.npz")
    C.write_checkpoint(a, geom, hp, unk)
    C.write_checkpoint(b, geom, hp, unk)
    assert all(r["max_abs"] == 0 for r in C.compare(a, b).values())
    u2 = unk.copy()
    g = geom.nguard
    u2[1, 0, g + 3, g + 5, DENS] += 1e-3
    C.write_checkpoint(b, geom, hp, u2)
    r = C.compare(a, b)
    assert abs(r["dens"]["max_abs"] - 1e-3) < 1e-15 and r["pres"]["max_abs"] == 0
    g3 = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
    mesh, u3 = A.levelset_problem(g3, hp, maxlev=2)
    C.write_checkpoint(b, g3, hp, u3, mesh=mesh)
    with pytest.raises(ValueError):
        C.compare(a, b)


def test_restart_continues_bit_for_bit(oracle):
    """Six oracle steps in one run equal three steps, a checkpoint, a restart
    from the file and three more steps."""
    geom, hp, init = S.config("kh2d", scale=1 / 32)
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)

    def steps(u, dt, dt_old, n):
        for _ in range(n):
            oracle.hydro_step(p, u, dt, dt_old)
            dt_old, dt = dt, oracle.driver_dt(oracle.compute_dt(p, u), dt)
        return dt, dt_old

    dt0 = 0.5 * oracle.compute_dt(p, unk)
    u_all = unk.copy()
    steps(u_all, dt0, dt0, 6)
    u = unk.copy()
    dt, dt_old = steps(u, dt0, dt0, 3)
    path = _tmp("restart.npz")
    C.write_checkpoint(path, geom, hp, u, time=0.0, dt=dt, dtold=dt_old, nstep=3)
    ck = C.read_checkpoint(path)
    u2 = ck["unk"]
    steps(u2, ck["dt"], ck["dtold"], 3)
    np.testing.assert_array_equal(_inner(geom, u2), _inner(geom, u_all))
