"""GPU parity at the benchmark configurations' stated sizes: the CUDA path
(through the C ABI) against the CPU oracle on the same seeded inputs.

* Configuration 1, 2-D Sod at 45 degrees on 256^2 (16x16 blocks of 16^2,
  outflow), driven to t = 0.2 by the Flash-X driver's dt control: the GPU's
  own Hydro_computeDt sequence equals the oracle's, the state is <= 1e-12
  relative per zone after step 1 and <= 1e-10 in L1 density after step 100
  (both bit-identical, as the FP64 path is built with -fmad=false), and at
  t = 0.2 the density, pressure and normal velocity along the diagonal are
  within the exact-solution bounds of Sod/shocktube.pro.
* Configuration 2, Kelvin-Helmholtz 2048^2: one step, bit for bit.
* Configuration 3, Rayleigh-Taylor 256^3 (WENO5 + HLLC, gravity, full CTU,
  periodic x/y, reflecting z): one step, bit for bit.
* Configuration 4, the AMR benchmark mesh (5,230 leaves of 16^3 on levels
  1-4): one step with guard fill, prolongation, restriction and flux
  correction, bit for bit; and three steps in batches of at most 700
  leaves (eight batches, leaves next to refined faces updated in a second
  pass) equal to the one-batch steps bit for bit.

The host needs about 14 GB for the two largest cases (two UNK copies each).
"""
import math

import numpy as np
import pytest

from exact_sod import sod_exact
from flashx_b200 import simulations as S
from flashx_b200.hydro import HydroDevice, driver_dt, initial_dt
from flashx_b200.params import DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ

pytestmark = pytest.mark.gpu

HYDRO_VARS = [DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ]
REL_TOL_ONE_STEP = 1e-12
L1_TOL_100 = 1e-10


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def test_sod_256_to_t02(oracle, need_gpu):
    geom, hp, init = S.config("sod2d", scale=1.0)
    assert geom.nblockx * geom.nxb == 256
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    ref = unk.copy()
    dev = HydroDevice(geom, hp, "fp64")
    dev.attach_unk(unk.copy())
    # Driver_verifyInitDt, then Driver_computeDt every step; the last step
    # lands on t = 0.2 as the driver's tmax clamp does
    dt_o = initial_dt(oracle.compute_dt(p, ref), hp)
    dt_g = initial_dt(dev.Hydro_computeDt(), hp)
    assert dt_g == dt_o
    t, n, dt_old = 0.0, 0, dt_o
    out = np.zeros(geom.unk_shape)
    while t < 0.2:
        dt = min(dt_o, 0.2 - t)
        oracle.hydro_step(p, ref, dt, dt_old)
        dev.Hydro(t + dt, dt, dt_old)
        t += dt
        n += 1
        if n in (1, 100):
            dev.sync_to_host(out)
            g, r = S.gather_global(geom, out)[..., HYDRO_VARS], S.gather_global(geom, ref)[..., HYDRO_VARS]
            if n == 1:
                assert np.max(_rel(g, r)) <= REL_TOL_ONE_STEP
            else:
                assert np.mean(np.abs(g[..., 0] - r[..., 0])) / np.mean(np.abs(r[..., 0])) <= L1_TOL_100
            assert np.array_equal(g, r), f"step {n}: FP64 path differs from the oracle"
        dt_old = dt
        c_o, c_g = oracle.compute_dt(p, ref), dev.Hydro_computeDt()
        assert c_g == c_o, f"step {n}: CFL dt {c_g} != oracle {c_o}"
        dt_o = oracle.driver_dt(c_o, dt_old)
        assert driver_dt(c_g, dt_old, hp) == dt_o
    assert abs(t - 0.2) < 1e-12 and n > 100
    dev.sync_to_host(out)
    g = S.gather_global(geom, out)[0]
    assert np.array_equal(g[..., HYDRO_VARS], S.gather_global(geom, ref)[0][..., HYDRO_VARS])
    dev.close()
    # the exact solution along the diagonal (Sod/shocktube.pro, soderror.pro)
    N = g.shape[0]
    idx = np.arange(N)
    x = (idx + 0.5) / N
    xi = (2 * x - 1.0) / math.sqrt(2.0) + 0.5
    rho_ex, u_ex, p_ex = sod_exact(xi, 0.2)
    rho, pres = g[idx, idx, DENS], g[idx, idx, PRES]
    vn = (g[idx, idx, VELX] + g[idx, idx, VELY]) / math.sqrt(2.0)
    keep = (xi > 0.05) & (xi < 0.95)
    l1 = lambda a, b: np.mean(np.abs(a[keep] - b[keep]))
    assert l1(rho, rho_ex) < 0.006
    assert l1(pres, p_ex) < 0.006
    assert l1(vn, u_ex) < 0.012
    mid = (xi > 0.74) & (xi < 0.80)
    assert np.allclose(rho[mid], 0.26557, atol=5e-3)
    assert np.allclose(pres[mid], 0.30313, atol=3e-3)


def test_kh_2048_one_step(oracle, need_gpu):
    geom, hp, init = S.config("kh2d", scale=1.0)
    assert geom.ncells == 2048 * 2048
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dev = HydroDevice(geom, hp, "fp64")
    dev.attach_unk(unk)
    dt = dev.Hydro_computeDt()
    assert dt == oracle.compute_dt(p, unk)
    dt = 0.5 * dt
    dev.Hydro(dt, dt, dt)
    oracle.hydro_step(p, unk, dt, dt)            # unk becomes the oracle's state
    out = np.zeros(geom.unk_shape)
    dev.sync_to_host(out)
    dev.close()
    g, r = S.gather_global(geom, out)[..., HYDRO_VARS], S.gather_global(geom, unk)[..., HYDRO_VARS]
    assert np.max(_rel(g, r)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r)


def test_rt_256_one_step(oracle, need_gpu):
    geom, hp, init = S.config("rt3d", scale=1.0)
    assert geom.ncells == 256 ** 3 and hp.order == 5 and hp.useGravity
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dev = HydroDevice(geom, hp, "fp64")
    dev.attach_unk(unk)
    dt = dev.Hydro_computeDt()
    assert dt == oracle.compute_dt(p, unk)
    dt = 0.5 * dt
    dev.Hydro(dt, dt, dt)
    out = np.zeros(geom.unk_shape)
    dev.sync_to_host(out)
    dev.close()
    oracle.hydro_step(p, unk, dt, dt)
    g = geom.nguard
    a = out[:, g:-g, g:-g, g:-g, :][..., HYDRO_VARS]
    b = unk[:, g:-g, g:-g, g:-g, :][..., HYDRO_VARS]
    assert np.max(_rel(a, b)) <= REL_TOL_ONE_STEP
    assert np.array_equal(a, b)


def test_amr_benchmark_mesh_one_step(oracle, need_gpu):
    from flashx_b200 import amr as A
    from flashx_b200.params import BC_PERIODIC, Geometry, HydroParams
    geom = Geometry(3, 16, 16, 16, 4, 4, 4, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams()
    mesh, unk = A.levelset_problem(geom, hp, maxlev=4)
    assert mesh.nleaf == 5230 and sorted(set(int(l) for l in mesh.levels)) == [1, 2, 3, 4]
    am = oracle.Amr(oracle.make_params(geom.as_dict(), hp), mesh.levels, mesh.bcoords)
    dev = HydroDevice(geom, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk)
    dt = dev.Hydro_computeDt()
    assert dt == am.compute_dt(unk)
    dt = 0.5 * dt
    dev.Hydro(dt, dt, dt)
    out = unk.copy()
    dev.sync_to_host(out)
    dev.close()
    am.hydro_step(unk, dt)
    g = geom.nguard
    a = out[:, g:-g, g:-g, g:-g, :][..., HYDRO_VARS]
    b = unk[:, g:-g, g:-g, g:-g, :][..., HYDRO_VARS]
    assert np.max(_rel(a, b)) <= REL_TOL_ONE_STEP
    assert np.array_equal(a, b)


def test_amr_benchmark_mesh_in_batches(need_gpu, monkeypatch):
    """The multi-batch step (FXB_AMR_MAX_BATCH caps the leaves per batch) on
    the benchmark mesh gives the one-batch state bit for bit, in both
    precisions; the tuning log shows the batch size in use."""
    from flashx_b200 import amr as A
    from flashx_b200.params import BC_PERIODIC, Geometry, HydroParams
    geom = Geometry(3, 16, 16, 16, 4, 4, 4, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams()
    mesh, unk = A.levelset_problem(geom, hp, maxlev=4)
    for prec in ("fp64", "mixed"):
        outs = []
        for cap in (None, "700"):
            if cap:
                monkeypatch.setenv("FXB_AMR_MAX_BATCH", cap)
            else:
                monkeypatch.delenv("FXB_AMR_MAX_BATCH", raising=False)
            monkeypatch.setenv("FXB_AMR_PERSISTENT", "0")
            dev = HydroDevice(geom, hp, prec, mesh=mesh)
            dev.attach_unk(unk.copy())
            if cap:
                assert "700 blocks" in dev.tuning()
            dt = 0.5 * dev.Hydro_computeDt()
            for _ in range(3):
                dev.Hydro(0.0, dt, dt)
            out = np.zeros(unk.shape)
            dev.sync_to_host(out)
            dev.close()
            outs.append(out)
        g = geom.nguard
        assert np.array_equal(outs[0][:, g:-g, g:-g, g:-g], outs[1][:, g:-g, g:-g, g:-g])
