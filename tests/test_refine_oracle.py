"""CPU tests of the oracle's refinement marking (Grid_markRefineDerefine:
the second-derivative error of gr_estimateBlkError.F90 and the marks of
Paramesh4/gr_markRefineDerefine.F90).

Known answers: on a single-level periodic mesh every leaf's guard cells are
same-level copies, so the error of each leaf is restated here with numpy from
the periodically padded global field and must agree bit for bit; constant
fields have zero error (derefine everywhere, across levels too: prolongation
and restriction keep a constant); a density step refines
the blocks it crosses up to the maximum level, and every other leaf is kept
or derefined by its own and its parent's error."""
import numpy as np
import pytest

from flashx_b200 import amr as A
from flashx_b200 import simulations as S
from flashx_b200.params import BC_OUTFLOW, BC_PERIODIC, DENS, PRES, Geometry, HydroParams


def _error_numpy(ext, dx, filt, lowb=(0, 0, 0), highb=(0, 0, 0), g=4):
    """gr_estimateBlkError on one guard-filled block ext[k, j, i] (Cartesian, 3-D)."""
    d = [0.5 / x for x in dx]
    E = ext
    du = np.zeros((3,) + E.shape)
    dua = np.zeros((3,) + E.shape)
    s = (slice(1, -1),) * 3
    du[0][s] = (E[1:-1, 1:-1, 2:] - E[1:-1, 1:-1, :-2]) * d[0]
    dua[0][s] = (np.abs(E[1:-1, 1:-1, 2:]) + np.abs(E[1:-1, 1:-1, :-2])) * d[0]
    du[1][s] = (E[1:-1, 2:, 1:-1] - E[1:-1, :-2, 1:-1]) * d[1]
    dua[1][s] = (np.abs(E[1:-1, 2:, 1:-1]) + np.abs(E[1:-1, :-2, 1:-1])) * d[1]
    du[2][s] = (E[2:, 1:-1, 1:-1] - E[:-2, 1:-1, 1:-1]) * d[2]
    dua[2][s] = (np.abs(E[2:, 1:-1, 1:-1]) + np.abs(E[:-2, 1:-1, 1:-1])) * d[2]
    n = E.shape[2] - 2 * g
    lo = [g if lowb[a] else 2 for a in range(3)]
    hi = [g + n - 1 if highb[a] else E.shape[2] - 3 for a in range(3)]
    k0, j0, i0 = slice(lo[2], hi[2] + 1), slice(lo[1], hi[1] + 1), slice(lo[0], hi[0] + 1)
    num = np.zeros((hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1))
    den = np.zeros_like(num)
    # terms in the reference's order: (1,x) (1,y) (2,x) (2,y) (1,z) (2,z) (3,x) (3,y) (3,z)
    for c, ax in ((0, 0), (0, 1), (1, 0), (1, 1), (0, 2), (1, 2), (2, 0), (2, 1), (2, 2)):
        sh = [0, 0, 0]
        sh[2 - ax] = 1
        def at(arr, o):
            return arr[slice(lo[2] + o * sh[0], hi[2] + 1 + o * sh[0]),
                       slice(lo[1] + o * sh[1], hi[1] + 1 + o * sh[1]),
                       slice(lo[0] + o * sh[2], hi[0] + 1 + o * sh[2])]
        d2 = (at(du[c], 1) - at(du[c], -1)) * d[ax]
        d3 = (np.abs(at(du[c], 1)) + np.abs(at(du[c], -1))) * d[ax]
        d4 = (at(dua[c], 1) + at(dua[c], -1)) * d[ax]
        num = num + d2 * d2
        t = d3 + filt * d4
        den = den + t * t
    with np.errstate(divide="ignore", invalid="ignore"):
        q = np.where(den != 0.0, num / den, 0.0)
    err = np.max(q)
    if np.any((den == 0.0) & (num != 0.0)):
        err = max(err, np.finfo(float).max)
    return np.sqrt(err)


def _single_level(oracle, field):
    hp = HydroParams()
    n = 8
    root = Geometry(3, n, n, n, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
    mesh = A.build_mesh(root, 2, lambda l, c, g: True)
    unk = A.fill_leaves(mesh, hp, field)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    return hp, root, mesh, unk, am


def test_single_level_error_matches_numpy_restatement(oracle):
    def field(X, Y, Z):
        r = 1.0 + 0.5 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) + 0.3 * np.tanh((Z - 0.5) / 0.05)
        return r, 0.1 + 0 * X, 0 * X, 0 * X, 1.0 + 0 * X
    hp, root, mesh, unk, am = _single_level(oracle, field)
    flags, err = am.mark_refine_derefine(unk, [(DENS, 0.8, 0.2, 0.01)], max_refine=4)
    n, g = 8, 4
    # global level-2 density, periodically padded
    glob = np.zeros((32, 32, 32))
    for l, c in enumerate(mesh.bcoords):
        glob[c[2] * n:(c[2] + 1) * n, c[1] * n:(c[1] + 1) * n, c[0] * n:(c[0] + 1) * n] = \
            unk[l, g:-g, g:-g, g:-g, DENS]
    pad = np.pad(glob, g, mode="wrap")
    dx = mesh.deltas(2)
    for l, c in enumerate(mesh.bcoords):
        ext = pad[c[2] * n:c[2] * n + n + 2 * g, c[1] * n:c[1] * n + n + 2 * g, c[0] * n:c[0] * n + n + 2 * g]
        assert err[l] == _error_numpy(ext, dx, 0.01), l
    assert err.max() > 0.0


def test_constant_fields_derefine(oracle):
    for bc in (BC_OUTFLOW, BC_PERIODIC):
        field = lambda X, Y, Z: (2.0 + 0 * X, 0 * X, 0 * X, 0 * X, 1.0 + 0 * X)
        hp = HydroParams()
        root = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(bc,) * 6)
        mesh = A.build_mesh(root, 3, lambda l, c, g: l == 1 and c == (0, 0, 0))
        assert set(mesh.levels) == {1, 2}
        unk = A.fill_leaves(mesh, hp, field)
        am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
        flags, err = am.mark_refine_derefine(unk, [(DENS, 0.8, 0.2, 0.01)], max_refine=4)
        assert np.all(err == 0.0)
        assert np.all(flags == -1)


def test_density_step_refines_the_blocks_it_crosses(oracle):
    hp = HydroParams()
    root = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_OUTFLOW,) * 6)
    mesh = A.build_mesh(root, 2, lambda l, c, g: True)

    def field(X, Y, Z):
        return np.where(X < 0.3, 1.0, 10.0), 0 * X, 0 * X, 0 * X, 1.0 + 0 * X
    unk = A.fill_leaves(mesh, hp, field)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    flags, err = am.mark_refine_derefine(unk, [(DENS, 0.8, 0.2, 0.01)], max_refine=4)
    for l, c in enumerate(mesh.bcoords):
        # level-2 blocks of 8 cells: x in [0, 0.25) and [0.25, 0.5) hold or neighbour the step
        if c[0] in (0, 1):
            assert flags[l] == 1 and err[l] > 0.8, (c, err[l])
        else:
            assert err[l] == 0.0
    # at the maximum level nothing is refined; the step's blocks stay, the rest derefine
    flags2, _ = am.mark_refine_derefine(unk, [(DENS, 0.8, 0.2, 0.01)], max_refine=2)
    assert np.all(flags2[[c[0] in (0, 1) for c in mesh.bcoords]] == 0)
    assert not np.any(flags2 == 1)


def test_pressure_criterion_uses_the_guard_cell_eos(oracle):
    """pres is an Eos output: its guard cells are recomputed by the Eos where
    they were interpolated, so the marks differ from an unfilled pressure
    only through those cells; with p uniform the error vanishes."""
    hp = HydroParams()
    root = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
    mesh = A.build_mesh(root, 3, lambda l, c, g: l == 1 and c == (1, 1, 1))
    def field(X, Y, Z):
        return 1.0 + 0.5 * X, 0.1 + 0 * X, 0 * X, 0 * X, 2.5 + 0 * X
    unk = A.fill_leaves(mesh, hp, field)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    flags, err = am.mark_refine_derefine(unk, [(PRES, 0.8, 0.2, 0.01), (DENS, 0.8, 0.2, 0.01)], max_refine=4)
    fp, ep = am.mark_refine_derefine(unk, [(PRES, 0.8, 0.2, 0.01)], max_refine=4)
    assert np.all(ep < 1e-10)
