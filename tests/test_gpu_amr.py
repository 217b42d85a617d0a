"""GPU parity tests of the AMR path (3-D): the CUDA library through its C ABI
against the oracle's AMR step on the same seeded mixed-level meshes.

The FP64 path is built with -fmad=false and is expected to reproduce the
oracle bit for bit (guard fill with restriction, prolongation and Eos, flux
correction, update); the tolerance REL_TOL_ONE_STEP = 1e-12 per zone is
checked first, equality second.  The mixed path must stay within 1e-5 L1
density of the FP64 path.
"""
import os

import numpy as np
import pytest

from flashx_b200 import amr as A
from flashx_b200.hydro import FlashXError, HydroDevice
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, DENS, EINT, ENER, GAMC, GAME,
                                Geometry, HydroParams, PRES, TEMP, VELX, VELY, VELZ)

pytestmark = pytest.mark.gpu

HYDRO_VARS = [DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ]
REL_TOL_ONE_STEP = 1e-12
L1_TOL_MIXED = 1e-5


def _interior(geom, u):
    g = geom.nguard
    return u[:, g:-g, g:-g, g:-g, :][..., HYDRO_VARS]


def _case(bc=(BC_PERIODIC,) * 6, maxlev=2, nroot=4, order=5, flattening=False, grav=None):
    hp = HydroParams(order=order, use_flattening=flattening)
    if grav is not None:
        hp = HydroParams(order=order, useGravity=True, gravity=grav)
    root = Geometry(3, 8, 8, 8, nroot, nroot, nroot, bc=bc)
    mesh, unk = A.levelset_problem(root, hp, maxlev)
    assert len(set(mesh.levels)) == maxlev
    return root, hp, mesh, unk


def _oracle(O, root, hp, mesh, unk, dts):
    am = O.Amr(O.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    u = unk.copy()
    for dt in dts:
        am.hydro_step(u, dt)
    return am, u


def _gpu(root, hp, mesh, unk, dts, precision="fp64"):
    dev = HydroDevice(root, hp, precision, mesh=mesh)
    dev.attach_unk(unk.copy())
    t = 0.0
    for i, dt in enumerate(dts):
        dev.Hydro(t + dt, dt, dts[i - 1] if i else dt)
        t += dt
    out = unk.copy()
    dev.sync_to_host(out)
    return dev, out


@pytest.mark.parametrize("bc,maxlev,order,flat", [
    ((BC_PERIODIC,) * 6, 2, 2, False),
    ((BC_PERIODIC,) * 6, 2, 5, False),
    ((BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING), 2, 3, False),
    ((BC_PERIODIC,) * 6, 3, 5, False),
    ((BC_PERIODIC,) * 6, 2, 3, True),
])
def test_amr_step_fp64_matches_oracle(oracle, need_gpu, bc, maxlev, order, flat):
    root, hp, mesh, unk = _case(bc, maxlev, order=order, flattening=flat)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    _, ref = _oracle(oracle, root, hp, mesh, unk, [dt, dt])
    dev, out = _gpu(root, hp, mesh, unk, [dt, dt])
    g, r = _interior(root, out), _interior(root, ref)
    assert np.max(np.abs(g - r) / np.maximum(np.abs(r), 1e-300)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r), "FP64 AMR path is expected to be bit-identical to the oracle"
    dev.close()


@pytest.mark.parametrize("order", [5, 2])
def test_amr_gravity_matches_oracle(oracle, need_gpu, order):
    """Constant gravity on a mesh of two levels (reflecting in z): the
    flux-corrected update with both gravity half steps, bit-identical to the
    oracle over two steps; the mixed path within the L1 bound."""
    bc = (BC_PERIODIC,) * 4 + (BC_REFLECTING,) * 2
    root, hp, mesh, unk = _case(bc, 2, order=order, grav=(0.02, 0.01, -0.1))
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    _, ref = _oracle(oracle, root, hp, mesh, unk, [dt, dt])
    dev, out = _gpu(root, hp, mesh, unk, [dt, dt])
    dev.close()
    g, r = _interior(root, out), _interior(root, ref)
    assert np.max(np.abs(g - r) / np.maximum(np.abs(r), 1e-300)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r), "FP64 AMR path is expected to be bit-identical to the oracle"
    dev, mixed = _gpu(root, hp, mesh, unk, [dt, dt], "mixed")
    dev.close()
    a, b = _interior(root, mixed)[..., 0], g[..., 0]
    assert np.mean(np.abs(a - b)) / np.mean(b) <= L1_TOL_MIXED


def test_amr_guard_fill_matches_oracle(oracle, need_gpu):
    root, hp, mesh, unk = _case(maxlev=3)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    ref = unk.copy()
    am.fill_guardcells(ref)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    out = unk.copy()
    dev.Grid_fillGuardCells(out)
    np.testing.assert_array_equal(out[..., HYDRO_VARS], ref[..., HYDRO_VARS])
    assert am.compute_dt(unk) == dev.Hydro_computeDt()
    dev.close()


def test_amr_masked_fill_and_doeos(oracle, need_gpu):
    """Grid_fillGuardCells on an AMR mesh with a mask: the selected variables
    equal the oracle's fill and nothing else is written; doEos=False skips
    Eos_guardCells on the guard regions next to other levels
    (Paramesh4/Grid_fillGuardCells.F90:531-548), which leaves densities and
    interiors as they are and changes pressures only in guard cells."""
    from flashx_b200.params import NUNK
    root, hp, mesh, unk = _case(maxlev=3)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    ref = unk.copy()
    am.fill_guardcells(ref)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    out = np.full(unk.shape, -7.0)
    dev.Grid_fillGuardCells(out, mask=["dens", "pres"])
    sel, rest = [DENS, PRES], [v for v in range(NUNK) if v not in (DENS, PRES)]
    np.testing.assert_array_equal(out[..., sel], ref[..., sel])
    assert np.all(out[..., rest] == -7.0)
    noeos = np.full(unk.shape, -7.0)
    dev.Grid_fillGuardCells(noeos, mask=["dens", "pres"], doEos=False)
    np.testing.assert_array_equal(noeos[..., DENS], ref[..., DENS])
    np.testing.assert_array_equal(_interior(root, noeos)[..., [0, 5]], _interior(root, ref)[..., [0, 5]])
    assert np.any(noeos[..., PRES] != ref[..., PRES])
    dev.close()


@pytest.mark.parametrize("persistent", ["0", "1"])
def test_amr_batches_agree(oracle, need_gpu, monkeypatch, persistent):
    """Batched launches: leaves processed in several batches (guard fill,
    fluxes, then a second pass for the leaves whose fluxes are corrected)
    give the one-batch result.  Persistent kernel: 37 scratch slots (CTAs)
    for all leaves give the same result."""
    root, hp, mesh, unk = _case(maxlev=2)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    _, ref = _oracle(oracle, root, hp, mesh, unk, [dt])
    monkeypatch.setenv("FXB_AMR_MAX_BATCH", "37")
    monkeypatch.setenv("FXB_AMR_PERSISTENT", persistent)
    dev, out = _gpu(root, hp, mesh, unk, [dt])
    np.testing.assert_array_equal(_interior(root, out), _interior(root, ref))
    dev.close()


@pytest.mark.parametrize("precision,cluster", [("fp64", "1"), ("fp64", "4"), ("fp64", "8"), ("mixed", "2")])
def test_amr_persistent_kernel_equals_batched_launches(oracle, need_gpu, monkeypatch, precision, cluster):
    """One persistent kernel per step (device work queue: restriction by level,
    then the leaves finest first, each leaf's whole pipeline in one CTA, bounded
    waits for finer neighbours' boundary fluxes) against the batched launches:
    bit for bit in FP64 (both equal the oracle), within round-off of the FP64
    guard-fill arithmetic (compiled with FMA in the mixed kernels) in mixed
    precision; one kernel launch per step."""
    root, hp, mesh, unk = _case(maxlev=3, order=3)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    outs = {}
    monkeypatch.setenv("FXB_AMR_CLUSTER", cluster)          # CTAs per leaf (a thread-block cluster)
    for flag in ("0", "1"):
        monkeypatch.setenv("FXB_AMR_PERSISTENT", flag)
        dev, out = _gpu(root, hp, mesh, unk, [dt, dt, dt], precision)
        outs[flag] = _interior(root, out)
        if flag == "1":
            assert dev.last_timing()[1] == 1
            dtn, dto = dev.advance(4, dt, dt)              # graph-captured persistent steps
            assert dtn > 0 and dto > 0
        dev.close()
    if precision == "fp64":
        _, ref = _oracle(oracle, root, hp, mesh, unk, [dt, dt, dt])
        np.testing.assert_array_equal(outs["1"], _interior(root, ref))
        np.testing.assert_array_equal(outs["1"], outs["0"])
    else:
        a, b = outs["1"][..., 0], outs["0"][..., 0]
        assert np.mean(np.abs(a - b)) / np.mean(b) <= 1e-7


def test_amr_persistent_wait_timeout_reports_status(oracle, need_gpu, monkeypatch):
    """The persistent kernel's waits are bounded: with a test hook that makes
    every leaf next to finer leaves wait on a flag that nothing sets, the wait
    runs out (~0.5 ms), the kernel raises its abort flag, every CTA leaves, and
    the host reads FXB_ETIMEOUT; the next solver instance on the same context
    steps exactly like the oracle."""
    from flashx_b200.hydro import FXB_ETIMEOUT
    root, hp, mesh, unk = _case(maxlev=2)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    monkeypatch.setenv("FXB_TEST_WAIT_TIMEOUT", "1")
    monkeypatch.setenv("FXB_AMR_PERSISTENT", "1")
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    assert "step form: persistent" in dev.tuning()
    dev.Hydro(0.0, dt, dt)
    with pytest.raises(FlashXError) as ei:
        dev.Hydro_computeDt()
    assert ei.value.code == FXB_ETIMEOUT
    dev.close()
    monkeypatch.delenv("FXB_TEST_WAIT_TIMEOUT")
    monkeypatch.delenv("FXB_AMR_PERSISTENT")
    _, ref = _oracle(oracle, root, hp, mesh, unk, [dt])
    dev, out = _gpu(root, hp, mesh, unk, [dt])
    np.testing.assert_array_equal(_interior(root, out), _interior(root, ref))
    dev.close()


def test_amr_advance_graph_and_conservation(oracle, need_gpu):
    root, hp, mesh, unk = _case(maxlev=2)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    I0 = dev.integrals()
    dt = 0.5 * dev.Hydro_computeDt()
    dt1, dto1 = dev.advance(5, dt, dt)
    I1 = dev.integrals()
    out = unk.copy()
    dev.sync_to_host(out)
    dev.close()
    # the same five steps through the oracle with the driver's dt sequence
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    u = unk.copy()
    d, do = dt, dt
    for _ in range(5):
        am.hydro_step(u, d)
        d, do = oracle.driver_dt(am.compute_dt(u), d), d
    assert d == dt1 and do == dto1
    np.testing.assert_array_equal(_interior(root, out), _interior(root, u))
    assert abs(I1[0] - I0[0]) <= 1e-13 * I0[0]
    assert abs(I1[4] - I0[4]) <= 1e-13 * I0[4]


def test_amr_mixed_precision_close_to_fp64(need_gpu):
    root, hp, mesh, unk = _case(maxlev=2)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    dt = 0.5 * dev.Hydro_computeDt()
    dev.close()
    _, a = _gpu(root, hp, mesh, unk, [dt] * 4, "fp64")
    _, b = _gpu(root, hp, mesh, unk, [dt] * 4, "mixed")
    ra, rb = _interior(root, a)[..., 0], _interior(root, b)[..., 0]
    assert np.mean(np.abs(ra - rb)) / np.mean(np.abs(ra)) <= L1_TOL_MIXED


def test_amr_rejects_unbalanced_mesh(need_gpu):
    hp = HydroParams()
    root = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
    leaves = [(1, (i, j, k)) for k in range(2) for j in range(2) for i in range(2) if (i, j, k) != (0, 0, 0)]
    kids = [(2, (i, j, k)) for k in range(2) for j in range(2) for i in range(2)]
    leaves += [c for c in kids if c[1] != (1, 1, 1)]
    leaves += [(3, (2 + i, 2 + j, 2 + k)) for k in range(2) for j in range(2) for i in range(2)]
    mesh = A.mesh_from_levels(root, leaves)
    with pytest.raises(FlashXError, match="more than one level"):
        HydroDevice(root, hp, "fp64", mesh=mesh)


def test_amr_compute_dt_location(need_gpu):
    from test_gpu_parity import _expected_loc
    root, hp, mesh, unk = _case(maxlev=2)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    dt, loc = dev.Hydro_computeDt(location=True)
    dl = [mesh.deltas(int(l)) for l in mesh.levels]
    assert loc == _expected_loc(root, unk, mesh.levels, dl)
    assert loc[3] == int(mesh.levels[loc[4] - 1])
    dev.close()


@pytest.mark.parametrize("bc,maxlev,crit,max_refine", [
    ((BC_PERIODIC,) * 6, 3, [("dens", 0.8, 0.2, 0.01)], 4),
    ((BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING), 2,
     [("pres", 0.5, 0.05, 0.01), ("dens", 0.3, 0.1, 0.02)], 2),
])
def test_mark_refine_derefine_matches_oracle(oracle, need_gpu, bc, maxlev, crit, max_refine):
    """Grid_markRefineDerefine: the error estimates of every leaf bit for bit
    (guard fill of leaves and parents, Eos for the pressure criterion, the
    domain-boundary ranges) and the refine/derefine marks."""
    root, hp, mesh, unk = _case(bc, maxlev)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    names = {"dens": DENS, "pres": PRES}
    ref_flags, ref_err = am.mark_refine_derefine(unk, [(names[c[0]],) + tuple(c[1:]) for c in crit], max_refine)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    flags, err = dev.Grid_markRefineDerefine(crit, max_refine)
    assert np.array_equal(err, ref_err)
    assert np.array_equal(flags, ref_flags)
    assert set(np.unique(flags)) <= {-1, 0, 1} and np.any(err > 0)
    dev.close()


@pytest.mark.parametrize("bc,maxlev", [
    ((BC_PERIODIC,) * 6, 3),
    ((BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING), 2),
])
def test_regrid_matches_oracle(oracle, need_gpu, bc, maxlev):
    """Grid_updateRefinement: marks from the device, the tree update on the
    host (amr.refine_derefine), the data movement on the device (fxb_regrid:
    copies, restriction of derefined parents, prolongation of new children,
    Eos) bit for bit equal to the oracle's; first the marks of a density
    criterion, then every finest-level leaf derefined; two steps on the
    final mesh."""
    root, hp, mesh, unk = _case(bc, maxlev, order=3)
    p = oracle.make_params(root.as_dict(), hp)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    flags, _ = dev.Grid_markRefineDerefine([("dens", 0.3, 0.05, 0.01)], maxlev + 1)
    am, ref = oracle.Amr(p, mesh.levels, mesh.bcoords), unk.copy()
    m1 = dev.Grid_updateRefinement(flags, lrefine_max=maxlev + 1)
    old = {(int(l), tuple(int(v) for v in c)) for l, c in zip(mesh.levels, mesh.bcoords)}
    new = {(int(l), tuple(int(v) for v in c)) for l, c in zip(m1.levels, m1.bcoords)}
    assert any((l - 1, tuple(v // 2 for v in c)) in old for l, c in new - old), "no leaf was refined"
    am1 = oracle.Amr(p, m1.levels, m1.bcoords)
    ref = am.regrid(ref, am1)
    got = np.zeros(m1.unk_shape)
    dev.sync_to_host(got)
    assert np.array_equal(_interior(root, got), _interior(root, ref))
    top = int(max(m1.levels))
    m2 = dev.Grid_updateRefinement([-1 if l == top else 0 for l in m1.levels], lrefine_max=maxlev + 1)
    assert m2.nleaf < m1.nleaf
    am2 = oracle.Amr(p, m2.levels, m2.bcoords)
    ref = am1.regrid(ref, am2)
    got = np.zeros(m2.unk_shape)
    dev.sync_to_host(got)
    assert np.array_equal(_interior(root, got), _interior(root, ref))
    dt = 0.5 * am2.compute_dt(ref)
    assert dev.Hydro_computeDt() == am2.compute_dt(ref)
    for _ in range(2):
        am2.hydro_step(ref, dt)
        dev.Hydro(0.0, dt, dt)
    dev.sync_to_host(got)
    assert np.array_equal(_interior(root, got), _interior(root, ref))
    dev.close()


def test_regrid_rejects_two_levels_and_keeps_the_mesh(oracle, need_gpu):
    """A new leaf whose parent was not an old leaf (two levels at once) is
    refused with FXB_EARG; the registered mesh and its data stay usable."""
    from flashx_b200.hydro import mesh_blocks
    root, hp, mesh, unk = _case((BC_PERIODIC,) * 6, 2, order=3)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    lv = [(int(l), tuple(int(v) for v in c)) for l, c in zip(mesh.levels, mesh.bcoords)]
    first = next(lc for lc in lv if lc[0] == 1)
    bad = set(lv) - {first}
    kids = [(2, (2 * first[1][0] + i, 2 * first[1][1] + j, 2 * first[1][2] + k))
            for k in (0, 1) for j in (0, 1) for i in (0, 1)]
    bad.update(kids[1:])
    bad.update((3, (2 * kids[0][1][0] + i, 2 * kids[0][1][1] + j, 2 * kids[0][1][2] + k))
               for k in (0, 1) for j in (0, 1) for i in (0, 1))
    bm = A.AmrMesh(root, sorted(bad))
    with pytest.raises(FlashXError) as e:
        from flashx_b200 import hydro as H
        H._check(dev.lib.fxb_regrid(mesh_blocks(bm.levels, bm.bcoords), bm.nleaf))
    assert e.value.code == 1
    out = unk.copy()
    dev.sync_to_host(out)
    assert np.array_equal(_interior(root, out), _interior(root, unk))
    dt = 0.5 * dev.Hydro_computeDt()
    am, ref = _oracle(oracle, root, hp, mesh, unk, [dt])
    dev.Hydro(0.0, dt, dt)
    dev.sync_to_host(out)
    assert np.array_equal(_interior(root, out), _interior(root, ref))
    dev.close()


def _rough_gas(X, Y, Z):
    """Density varying by e^1.2 from cell to cell, velocities of order one, p = 1."""
    rho = np.exp(1.2 * np.sin(311.0 * X + 17.0 * Y) * np.cos(173.0 * Y - 29.0 * Z + 3.0 * X))
    vx, vy, vz = np.sin(251.0 * Y + 7.0 * Z), np.cos(199.0 * Z - 11.0 * X), np.sin(277.0 * X + 5.0 * Y)
    return rho, vx, vy, vz, np.ones_like(rho)


@pytest.mark.parametrize("opts,order,bc", [
    (dict(use_avisc=True), 3, (BC_PERIODIC,) * 6),
    (dict(use_avisc=True, cvisc=0.3), 5, (BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING,
                                          BC_REFLECTING)),
    (dict(use_hybridOrder=True), 3, (BC_PERIODIC,) * 6),
    (dict(use_hybridOrder=True, hybridOrderKappa=0.05), 5, (BC_REFLECTING,) * 6),
    (dict(use_hybridOrder=True, use_avisc=True), 2, (BC_PERIODIC,) * 6),
])
def test_amr_avisc_and_hybrid_order_match_oracle(oracle, need_gpu, opts, order, bc):
    """Artificial viscosity (the guard-filled blocks then carry the total
    energy) and hybrid order (DivU and flags per leaf from a guard fill of
    every guard cell) on a two-level mesh, FP64 bit for bit, two steps; the
    options change the solution."""
    hyb = opts.get("use_hybridOrder", False)
    hp = HydroParams(order=order, gamma=3.0 if hyb else 1.4, **opts)
    root = Geometry(3, 8, 8, 8, 4, 4, 4, bc=bc)
    mesh, unk = A.levelset_problem(root, hp, 2)
    if hyb:     # steep converging cells, where face states break the shock density bounds
        unk = A.fill_leaves(mesh, hp, _rough_gas)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    _, ref = _oracle(oracle, root, hp, mesh, unk, [dt, dt])
    dev, out = _gpu(root, hp, mesh, unk, [dt, dt])
    g, r = _interior(root, out), _interior(root, ref)
    assert np.max(np.abs(g - r) / np.maximum(np.abs(r), 1e-300)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r)
    dev.close()
    _, plain = _oracle(oracle, root, HydroParams(order=order, gamma=hp.gamma), mesh, unk, [dt, dt])
    assert not np.array_equal(r, _interior(root, plain))


def test_amr_avisc_mixed_close_to_fp64(need_gpu):
    root, hp, mesh, unk = _case(maxlev=2)
    hp = HydroParams(order=5, use_avisc=True, use_hybridOrder=True)
    dev = HydroDevice(root, hp, "fp64", mesh=mesh)
    dev.attach_unk(unk.copy())
    dt = 0.5 * dev.Hydro_computeDt()
    dev.close()
    _, a = _gpu(root, hp, mesh, unk, [dt] * 5, "mixed")
    _, b = _gpu(root, hp, mesh, unk, [dt] * 5)
    x, y = _interior(root, a)[..., 0], _interior(root, b)[..., 0]
    assert np.mean(np.abs(x - y)) / np.mean(np.abs(y)) <= L1_TOL_MIXED
