"""CPU tests of the AMR part of the oracle (PARAMESH guard fill, restriction,
prolongation, Eos on non-same-level guard regions, flux correction).

Known answers used: a mesh refined to one uniform level must reproduce the
uniform-grid oracle bit for bit (same-level copies and boundary conditions);
prolongation reproduces linear data; a coarse guard cell next to a finer
region holds the conserved-form average of the fine cells; a uniform flow
stays uniform across fine/coarse boundaries; mass, momentum and energy are
conserved on periodic mixed-level meshes, which needs the flux correction.
"""
import numpy as np
import pytest

from flashx_b200 import amr as A
from flashx_b200 import simulations as S
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, DENS, EINT, ENER, GAMC, GAME,
                                Geometry, HydroParams, PRES, TEMP, VELX, VELY, VELZ)


def _uniform_level_case(O, ndim, bc, order, steps=2, grav=None, **opts):
    hp = HydroParams(order=order, **opts) if grav is None else HydroParams(order=order, useGravity=True, gravity=grav)
    nz = 8 if ndim == 3 else 1
    root = Geometry(ndim, 8, 8, nz, 2, 2, 2 if ndim == 3 else 1, bc=bc)
    fine = Geometry(ndim, 8, 8, nz, 4, 4, 4 if ndim == 3 else 1, bc=bc)
    mesh = A.build_mesh(root, 2, lambda l, c, g: True)
    assert set(mesh.levels) == {2}
    unk_ug = S.noisy_gas(fine, hp)
    slot = [(c[2] * fine.nblocky + c[1]) * fine.nblockx + c[0] for c in mesh.bcoords]
    unk_amr = np.ascontiguousarray(unk_ug[slot])
    pu = O.make_params(fine.as_dict(), hp)
    am = O.Amr(O.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * O.compute_dt(pu, unk_ug)
    assert am.compute_dt(unk_amr) == O.compute_dt(pu, unk_ug)
    for _ in range(steps):
        O.hydro_step(pu, unk_ug, dt, dt)
        am.hydro_step(unk_amr, dt)
    g = fine.nguard
    sl = (slice(g, -g) if ndim == 3 else slice(None), slice(g, -g), slice(g, -g))
    for l, b in enumerate(slot):
        np.testing.assert_array_equal(unk_amr[l][sl], unk_ug[b][sl])


@pytest.mark.parametrize("ndim,bc,order", [
    (2, (BC_PERIODIC,) * 6, 3),
    (2, (BC_OUTFLOW, BC_REFLECTING, BC_REFLECTING, BC_OUTFLOW, 0, 0), 5),
    (3, (BC_PERIODIC,) * 4 + (BC_REFLECTING,) * 2, 5),
])
def test_uniform_level_mesh_equals_uniform_grid(oracle, ndim, bc, order):
    _uniform_level_case(oracle, ndim, bc, order)


@pytest.mark.parametrize("ndim,order", [(2, 3), (3, 5), (3, 2)])
def test_gravity_on_amr_meshes(oracle, ndim, order):
    """Constant gravity on AMR meshes: hy_gravityStep's n+1 half step runs on
    every leaf after the flux-corrected update, before energyFix and Eos
    (hy_updateSolution.F90 defers them under GRAVITY).  A single-level mesh
    reproduces the uniform grid bit for bit, and a uniform gas on a mesh of
    three levels falls freely (v = n dt g, rho and p unchanged)."""
    refl = (BC_PERIODIC,) * 2 + (BC_REFLECTING,) * 2 + (0, 0) if ndim == 2 else \
        (BC_PERIODIC,) * 4 + (BC_REFLECTING,) * 2
    g = (0.02, -0.1, 0.0) if ndim == 2 else (0.02, 0.01, -0.1)
    _uniform_level_case(oracle, ndim, refl, order, grav=g)

    hp = HydroParams(order=order, useGravity=True, gravity=g)
    nz = 8 if ndim == 3 else 1
    root = Geometry(ndim, 8, 8, nz, 4, 4, 4 if ndim == 3 else 1, bc=(BC_PERIODIC,) * 6)
    mesh = A.build_mesh(root, 3, lambda l, c, gm: (l == 1 and c[0] in (1, 2) and c[1] == 1) or
                        (l == 2 and c[0] == 3 and c[1] == 3))
    assert len(set(mesh.levels)) == 3

    def fields(X, Y, Z):
        one = np.ones_like(X)
        return 1.3 * one, 0.0 * one, 0.0 * one, 0.0 * one, 0.7 * one
    unk = A.fill_leaves(mesh, hp, fields)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    for _ in range(3):
        am.hydro_step(unk, dt)
    ng = root.nguard
    inner = unk[:, ng:-ng, ng:-ng, ng:-ng, :] if ndim == 3 else unk[:, :, ng:-ng, ng:-ng, :]
    for q, v in enumerate((VELX, VELY, VELZ)):
        assert np.allclose(inner[..., v], 3 * dt * g[q], rtol=1e-12, atol=1e-15)
    assert np.max(np.abs(inner[..., DENS] - 1.3)) < 1e-13
    assert np.max(np.abs(inner[..., PRES] - 0.7)) < 1e-12


def test_tree_validation(oracle):
    hp = HydroParams()
    root = Geometry(2, 8, 8, 1, 2, 2, 1, bc=(BC_PERIODIC,) * 6)
    p = oracle.make_params(root.as_dict(), hp)
    roots = [(1, (i, j, 0)) for j in range(2) for i in range(2)]
    oracle.Amr(p, [l for l, _ in roots], [c for _, c in roots]).close()
    # refine root (0,0) twice in its corner: level 3 next to level 1 -> unbalanced
    leaves = [lc for lc in roots if lc[1] != (0, 0, 0)]
    kids = [(2, (i, j, 0)) for j in range(2) for i in range(2)]
    leaves += [k for k in kids if k[1] != (1, 1, 0)]
    leaves += [(3, (2 + i, 2 + j, 0)) for j in range(2) for i in range(2)]
    with pytest.raises(ValueError, match="balanced"):
        oracle.Amr(p, [l for l, _ in leaves], [c for _, c in leaves])
    # a missing child -> incomplete
    bad = [lc for lc in roots if lc[1] != (0, 0, 0)] + kids[:3]
    with pytest.raises(ValueError, match="incomplete"):
        oracle.Amr(p, [l for l, _ in bad], [c for _, c in bad])
    # a leaf and its child both listed -> overlap
    bad = roots + kids
    with pytest.raises(ValueError, match="overlap"):
        oracle.Amr(p, [l for l, _ in bad], [c for _, c in bad])


def _two_level_2d(bc=(BC_OUTFLOW,) * 6):
    """4x4 root blocks of 8^2; the central 2x2 roots refined once."""
    root = Geometry(2, 8, 8, 1, 4, 4, 1, bc=bc)
    mesh = A.build_mesh(root, 2, lambda l, c, g: 1 <= c[0] <= 2 and 1 <= c[1] <= 2)
    return root, mesh


def _guard_positions(mesh, l):
    """(k, j, i) guard indices and level-l global cell indices of leaf l."""
    g = mesh.geom
    ng = g.nguard
    c = mesh.bcoords[l]
    out = []
    for j in range(g.nyb + 2 * ng):
        for i in range(g.nxb + 2 * ng):
            li, lj = i - ng, j - ng
            if 0 <= li < g.nxb and 0 <= lj < g.nyb:
                continue
            out.append((0, j, i, c[0] * g.nxb + li, c[1] * g.nyb + lj))
    return out


def test_prolongation_reproduces_linear_data(oracle):
    hp = HydroParams()
    root, mesh = _two_level_2d()
    a0, ax, ay = 0.1, 0.3, -0.2

    def fields(X, Y, Z):
        rho = np.full_like(X, 2.0)
        return rho, a0 + ax * X + ay * Y, 0.05 + 0.1 * X, 0.0 * X, np.full_like(X, 1.0)
    unk = A.fill_leaves(mesh, hp, fields)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    am.fill_guardcells(unk)
    checked = 0
    for l in range(mesh.nleaf):
        if mesh.levels[l] != 2:
            continue
        dx = mesh.deltas(2)[0]
        N = root.nblockx * root.nxb * 2
        for k, j, i, gx, gy in _guard_positions(mesh, l):
            # only cells whose interpolation stencil stays inside the domain
            if not (2 <= gx < N - 2 and 2 <= gy < N - 2):
                continue
            x, y = (gx + 0.5) * dx, (gy + 0.5) * dx
            assert abs(unk[l, k, j, i, VELX] - (a0 + ax * x + ay * y)) < 1e-14
            assert abs(unk[l, k, j, i, DENS] - 2.0) < 1e-15
            checked += 1
    assert checked > 100


def test_coarse_guard_cells_hold_restricted_average(oracle):
    hp = HydroParams()
    root, mesh = _two_level_2d()

    def fields(X, Y, Z):
        rho = 1.0 + 0.5 * np.sin(7.0 * X) * np.cos(5.0 * Y)
        return rho, 0.2 * np.cos(3.0 * Y), 0.1 * X, 0.0 * X, 1.0 + 0.1 * X * Y
    unk = A.fill_leaves(mesh, hp, fields)
    ref = unk.copy()
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    am.fill_guardcells(unk)
    ng = root.nguard
    # fine leaves by level-2 block coordinates
    fine = {tuple(mesh.bcoords[l][:2]): l for l in range(mesh.nleaf) if mesh.levels[l] == 2}
    checked = 0
    for l in range(mesh.nleaf):
        if mesh.levels[l] != 1:
            continue
        for k, j, i, gx, gy in _guard_positions(mesh, l):
            fx, fy = 2 * gx, 2 * gy
            key = (fx // root.nxb, fy // root.nyb)
            if key not in fine or gx < 0 or gy < 0:
                continue
            f = fine[key]
            li, lj = fx - key[0] * root.nxb + ng, fy - key[1] * root.nyb + ng
            cells = ref[f, 0, lj:lj + 2, li:li + 2, :]
            rho = cells[..., DENS].mean()
            mx = (cells[..., DENS] * cells[..., VELX]).mean()
            assert abs(unk[l, k, j, i, DENS] - rho) < 1e-15 * rho
            assert abs(unk[l, k, j, i, VELX] - mx / rho) < 1e-14
            checked += 1
    assert checked >= 32


def test_uniform_flow_stays_uniform(oracle):
    hp = HydroParams()
    root = Geometry(2, 8, 8, 1, 4, 4, 1, bc=(BC_PERIODIC,) * 6)
    mesh = A.build_mesh(root, 3, lambda l, c, g: (l == 1 and c[0] in (1, 2) and c[1] == 1) or
                        (l == 2 and c[0] == 3 and c[1] == 3))
    assert len(set(mesh.levels)) == 3

    def fields(X, Y, Z):
        one = np.ones_like(X)
        return 1.3 * one, 0.4 * one, -0.25 * one, 0.0 * one, 0.7 * one
    unk = A.fill_leaves(mesh, hp, fields)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    for _ in range(4):
        am.hydro_step(unk, dt)
    ng = root.nguard
    inner = unk[:, :, ng:-ng, ng:-ng, :]
    assert np.max(np.abs(inner[..., DENS] - 1.3)) < 1e-13
    assert np.max(np.abs(inner[..., VELX] - 0.4)) < 1e-13
    assert np.max(np.abs(inner[..., VELY] + 0.25)) < 1e-13
    assert np.max(np.abs(inner[..., PRES] - 0.7)) < 1e-13


@pytest.mark.parametrize("ndim,bc,order,opts", [
    (2, (BC_PERIODIC,) * 6, 3, dict(use_avisc=True)),
    (3, (BC_PERIODIC,) * 4 + (BC_REFLECTING,) * 2, 5, dict(use_avisc=True, cvisc=0.3)),
    (2, (BC_OUTFLOW, BC_REFLECTING, BC_REFLECTING, BC_OUTFLOW, 0, 0), 3, dict(use_hybridOrder=True)),
    (3, (BC_PERIODIC,) * 6, 5, dict(use_hybridOrder=True, hybridOrderKappa=0.05)),
    (3, (BC_PERIODIC,) * 6, 2, dict(use_hybridOrder=True, use_avisc=True)),
])
def test_uniform_level_mesh_equals_uniform_grid_options(oracle, ndim, bc, order, opts):
    """Artificial viscosity and hybrid order on a mesh refined to one level
    reproduce the uniform-grid oracle bit for bit: the AMR step reads their
    guard cells (transverse velocity differences, DivU four cells out) from
    the guard fill as the uniform grid does from its neighbours."""
    _uniform_level_case(oracle, ndim, bc, order, **opts)


@pytest.mark.parametrize("ndim,maxlev,opts", [(2, 3, {}), (3, 2, {}), (3, 2, dict(use_avisc=True)),
                                              (3, 2, dict(use_hybridOrder=True))])
def test_amr_conserves_on_periodic_mesh(oracle, ndim, maxlev, opts):
    hp = HydroParams(order=3 if ndim == 2 else 5, **opts)
    nz = 8 if ndim == 3 else 1
    root = Geometry(ndim, 8, 8, nz, 4, 4, 4 if ndim == 3 else 1, bc=(BC_PERIODIC,) * 6)
    mesh, unk = A.levelset_problem(root, hp, maxlev)
    assert len(set(mesh.levels)) == maxlev
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    I0 = am.integrals(unk)
    dt = 0.5 * am.compute_dt(unk)
    for _ in range(3):
        am.hydro_step(unk, dt)
    I1 = am.integrals(unk)
    tol = 1e-13 if opts else 1e-14      # rounding of the mesh sums; the options change the fluxes' operands
    assert abs(I1[0] - I0[0]) <= tol * abs(I0[0])            # mass
    assert abs(I1[4] - I0[4]) <= tol * abs(I0[4])            # total energy
    for q in (1, 2, 3):                                        # momentum
        assert abs(I1[q] - I0[q]) <= tol * I0[0]


def test_eos_regions_follow_neighbour_levels(oracle):
    hp = HydroParams()
    root, mesh = _two_level_2d(bc=(BC_PERIODIC,) * 6)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    for l in range(mesh.nleaf):
        finer, eos = am.leaf_flags(l)
        c = mesh.bcoords[l]
        if mesh.levels[l] == 1 and tuple(c[:2]) == (0, 0):
            # the root at the corner touches the refined 2x2 only diagonally
            assert finer == [0] * 6
            assert sum(eos) == 1 and eos[(1 * 3 + 2) * 3 + 2] == 1
        if mesh.levels[l] == 1 and tuple(c[:2]) == (1, 0):
            assert finer[3] == 1 and sum(finer) == 1
