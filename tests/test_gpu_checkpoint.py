"""GPU restart: a run checkpointed from the device mirror (fxb_sync_to_host
into the Flash-X checkpoint datasets) and restarted on a fresh device
continues bit for bit, on a uniform grid and on an AMR mesh."""
import os
import tempfile

import numpy as np
import pytest

from flashx_b200 import amr as A
from flashx_b200 import checkpoint as C
from flashx_b200 import simulations as S
from flashx_b200.hydro import HydroDevice, driver_dt
from flashx_b200.params import BC_PERIODIC, Geometry, HydroParams

pytestmark = pytest.mark.gpu


def _run(dev, hp, dt, dt_old, n):
    for _ in range(n):
        dev.Hydro(0.0, dt, dt_old)
        dt_old, dt = dt, driver_dt(dev.Hydro_computeDt(), dt, hp)
    return dt, dt_old


@pytest.mark.parametrize("amr", [False, True])
def test_restart_from_checkpoint_continues_bit_for_bit(need_gpu, amr):
    if amr:
        geom = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
        hp = HydroParams()
        mesh, unk = A.levelset_problem(geom, hp, maxlev=2)
    else:
        geom, hp, init = S.config("kh2d", scale=1 / 16)
        mesh, unk = None, init(geom, hp)
    shape = unk.shape
    dev = HydroDevice(geom, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    dt0 = 0.5 * dev.Hydro_computeDt()
    _run(dev, hp, dt0, dt0, 6)
    ref = np.zeros(shape)
    dev.sync_to_host(ref)
    dev.attach_unk(unk.copy())
    dt, dt_old = _run(dev, hp, dt0, dt0, 3)
    mid = np.zeros(shape)
    dev.sync_to_host(mid)
    dev.close()
    path = os.path.join(tempfile.mkdtemp(), "chk.npz")
    C.write_checkpoint(path, geom, hp, mid, mesh=mesh, dt=dt, dtold=dt_old, nstep=3)
    ck = C.read_checkpoint(path)
    dev2 = HydroDevice(ck["geom"], ck["hp"], "fp64", mesh=C.restart_mesh(ck))
    dev2.attach_unk(ck["unk"])
    _run(dev2, ck["hp"], ck["dt"], ck["dtold"], 3)
    out = np.zeros(shape)
    dev2.sync_to_host(out)
    dev2.close()
    g = geom.nguard
    inner = (slice(None), slice(g, -g) if geom.ndim == 3 else slice(None), slice(g, -g), slice(g, -g))
    np.testing.assert_array_equal(out[inner], ref[inner])
