"""GPU parity of the shock detector (hy_shockDetectBlk.F90, shockDetect) and
the hybrid Riemann solver (RiemannSolver = hybrid: HLL on faces next to a
marked cell, HLLC elsewhere; hy_getFaceFlux.F90:364-383), uniform grids: the
CUDA path through the C ABI against the oracle on the same seeded inputs.

FP64 is expected bit for bit (-fmad=false; REL_TOL = 1e-12 per value is
checked first), the SHOK slot of the synced UNK included (interior and guard
cells); the mixed path stays within 1e-5 L1 density of FP64.
"""
import numpy as np
import pytest

from flashx_b200 import simulations as S
from flashx_b200.hydro import FlashXError, FXB_EUNSUPPORTED, HydroDevice
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, DENS, EINT, ENER, GAMC, GAME,
                                Geometry, HydroParams, PRES, SHOK, TEMP, VELX, VELY, VELZ)

pytestmark = pytest.mark.gpu

HYDRO_VARS = [DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ]
REL_TOL = 1e-12
L1_TOL_MIXED = 1e-5


def _run(oracle, geom, hp, unk, steps, precision="fp64"):
    p = oracle.make_params(geom.as_dict(), hp)
    dt = 0.3 * oracle.compute_dt(p, unk)
    ref = unk.copy()
    for _ in range(steps):
        oracle.hydro_step(p, ref, dt, dt)
    dev = HydroDevice(geom, hp, precision)
    dev.attach_unk(unk.copy())
    for _ in range(steps):
        dev.Hydro(0.0, dt, dt)
    out = unk.copy()
    dev.sync_to_host(out)
    dev.close()
    return ref, out


def _check(geom, out, ref):
    a, b = S.gather_global(geom, out)[..., HYDRO_VARS], S.gather_global(geom, ref)[..., HYDRO_VARS]
    assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)) <= REL_TOL
    assert np.array_equal(a, b)


@pytest.mark.parametrize("case", ["sod2d_outflow", "sod2d_reflect", "blast2d_periodic_weno", "sod3d_outflow",
                                  "blast3d_mixed_bc"])
def test_hybrid_solver_fp64(oracle, need_gpu, case):
    if case == "sod2d_outflow":
        geom, hp, steps = Geometry(2, 16, 16, 1, 4, 4, 1, bc=(BC_OUTFLOW,) * 6), HydroParams(RiemannSolver="hybrid"), 25
        unk = S.sod(geom, hp)
    elif case == "sod2d_reflect":
        geom, hp, steps = (Geometry(2, 16, 16, 1, 4, 3, 1, bc=(BC_REFLECTING,) * 6),
                           HydroParams(RiemannSolver="hybrid", order=2), 25)
        unk = S.sod(geom, hp)
    elif case == "blast2d_periodic_weno":
        geom, hp, steps = (Geometry(2, 16, 16, 1, 3, 3, 1, bc=(BC_PERIODIC,) * 6),
                           HydroParams(RiemannSolver="hybrid", order=5), 20)
        unk = S.sod(geom, hp, p_l=10.0, p_r=0.1)
    elif case == "sod3d_outflow":
        geom, hp, steps = (Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6),
                           HydroParams(RiemannSolver="hybrid"), 10)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    else:
        geom, hp, steps = (Geometry(3, 16, 16, 16, 1, 2, 1, bc=(BC_PERIODIC, BC_PERIODIC, BC_REFLECTING,
                                                                BC_REFLECTING, BC_OUTFLOW, BC_OUTFLOW)),
                           HydroParams(RiemannSolver="hybrid", order=5), 10)
        unk = S.sod(geom, hp, p_l=10.0, p_r=0.1, xangle=30.0, yangle=70.0, posn=0.6)
    ref, out = _run(oracle, geom, hp, unk, steps)
    _check(geom, out, ref)
    assert np.array_equal(out[..., SHOK], ref[..., SHOK])      # the flags, guard cells included
    assert ref[..., SHOK].sum() > 0                               # the detector marked cells
    hllc, _ = _run(oracle, geom, HydroParams(order=hp.order), unk, steps)
    assert not np.array_equal(S.gather_global(geom, hllc)[..., DENS], S.gather_global(geom, ref)[..., DENS])


def test_shock_detector_alone_keeps_hllc(oracle, need_gpu):
    """shockDetect with HLLC: the flags reach UNK, the solution is HLLC's."""
    geom = Geometry(2, 16, 16, 1, 4, 4, 1, bc=(BC_OUTFLOW,) * 6)
    hp = HydroParams(shockDetect=True)
    unk = S.sod(geom, hp)
    ref, out = _run(oracle, geom, hp, unk, 25)
    _check(geom, out, ref)
    assert np.array_equal(out[..., SHOK], ref[..., SHOK]) and ref[..., SHOK].sum() > 0
    plain, _ = _run(oracle, geom, HydroParams(), unk, 25)
    assert np.array_equal(S.gather_global(geom, plain)[..., HYDRO_VARS], S.gather_global(geom, ref)[..., HYDRO_VARS])


@pytest.mark.parametrize("ndim", [2, 3])
def test_hybrid_solver_mixed_close_to_fp64(oracle, need_gpu, ndim):
    if ndim == 2:
        geom = Geometry(2, 16, 16, 1, 4, 4, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams(RiemannSolver="hybrid")
        unk = S.sod(geom, hp)
    else:
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams(RiemannSolver="hybrid", order=5)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    _, a = _run(oracle, geom, hp, unk, 15, "mixed")
    _, b = _run(oracle, geom, hp, unk, 15)
    x, y = S.gather_global(geom, a)[..., DENS], S.gather_global(geom, b)[..., DENS]
    assert np.mean(np.abs(x - y)) / np.mean(np.abs(y)) <= L1_TOL_MIXED


def test_shock_detector_rejected_on_amr_meshes(need_gpu):
    from flashx_b200 import amr as A
    root = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams(RiemannSolver="hybrid")
    mesh, _ = A.levelset_problem(root, hp, 2)
    with pytest.raises(FlashXError) as ei:
        HydroDevice(root, hp, mesh=mesh)
    assert ei.value.code == FXB_EUNSUPPORTED
