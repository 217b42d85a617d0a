"""CPU tests of regridding during a run: the host tree update restated from
PARAMESH's amr_refine_derefine (flashx_b200.amr.refine_derefine) and the
oracle's data movement of Grid_updateRefinement (fxo_amr_regrid: copies,
restriction of derefined parents, conserved-form prolongation of new
children, Eos).  The device's data movement (fxb_regrid) is compared with
this oracle in tests/test_gpu_amr.py."""
import numpy as np
import pytest

from flashx_b200 import amr as A
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, DENS, EINT, ENER, Geometry, HydroParams, PRES,
                                VELX, VELY, VELZ)


def _geom(bc=BC_OUTFLOW, nb=4, n=8):
    return Geometry(3, n, n, n, nb, nb, nb, bc=(bc,) * 6)


def _leafset(mesh):
    return {(int(l), tuple(int(v) for v in c)) for l, c in zip(mesh.levels, mesh.bcoords)}


def _flags(mesh, marks):
    return [marks.get((int(l), tuple(int(v) for v in c)), 0) for l, c in zip(mesh.levels, mesh.bcoords)]


def _uniform(g):
    return A.build_mesh(g, 1, lambda *a: False)


def test_refine_one_leaf_and_propagate():
    g = _geom()
    m = _uniform(g)
    m2 = A.refine_derefine(m, _flags(m, {(1, (1, 1, 1)): 1}), lrefine_max=3)
    s = _leafset(m2)
    assert (1, (1, 1, 1)) not in s and len(s) == 64 - 1 + 8
    # refining a level-2 leaf next to level-1 leaves refines them too (proper nesting)
    m3 = A.refine_derefine(m2, _flags(m2, {(2, (2, 2, 2)): 1}), lrefine_max=3)
    s3 = _leafset(m3)
    assert (3, (4, 4, 4)) in s3
    for c in [(0, 0, 0), (0, 1, 1), (1, 0, 0), (0, 0, 1)]:
        assert (1, c) not in s3, c          # the 26 neighbours of (1,1,1) at level 1 were refined
    assert A.is_balanced(g, s3)


def test_derefine_rules():
    g = _geom()
    u = _uniform(g)
    m = A.refine_derefine(u, _flags(u, {(1, (1, 1, 1)): 1, (1, (0, 1, 1)): 1}), lrefine_max=3)
    kids = [lc for lc in _leafset(m) if lc[0] == 2 and all(v // 2 == 1 for v in lc[1])]
    assert len(kids) == 8
    # all eight siblings derefine: the parent comes back
    back = A.refine_derefine(m, _flags(m, {k: -1 for k in kids}), lrefine_max=3)
    assert (1, (1, 1, 1)) in _leafset(back) and len(_leafset(back)) == len(_leafset(m)) - 7
    # one sibling missing: nothing happens
    back = A.refine_derefine(m, _flags(m, {k: -1 for k in kids[1:]}), lrefine_max=3)
    assert _leafset(back) == _leafset(m)
    # at lrefine_min nothing derefines (and the coarser leaves are refined up to it)
    back = A.refine_derefine(m, _flags(m, {k: -1 for k in kids}), lrefine_min=2, lrefine_max=3)
    assert all(k in _leafset(back) for k in kids)
    assert min(l for l, _ in _leafset(back)) == 2
    # a same-level neighbour that refines blocks the derefinement
    marks = {k: -1 for k in kids}
    nbr = [lc for lc in _leafset(m) if lc[0] == 2 and lc[1] == (1, 2, 2)][0]   # a child of (0,1,1)
    marks[nbr] = 1
    m4 = A.refine_derefine(m, _flags(m, marks), lrefine_max=3)
    assert all(k in _leafset(m4) for k in kids)
    assert A.is_balanced(g, _leafset(m4))


def test_lrefine_max_stops_refinement():
    g = _geom()
    m = _uniform(g)
    assert _leafset(A.refine_derefine(m, [1] * 64, lrefine_max=1)) == _leafset(m)


def test_random_marks_keep_the_mesh_balanced():
    rng = np.random.default_rng(5)
    g = _geom(BC_PERIODIC)
    m = A.build_mesh(g, 3, lambda lev, c, gg: (c[0] + c[1] + c[2]) % 3 == 0)
    for _ in range(6):
        flags = rng.choice([-1, 0, 1], size=m.nleaf, p=[0.5, 0.35, 0.15])
        new = A.refine_derefine(m, flags, lrefine_max=4)
        s_old, s_new = _leafset(m), _leafset(new)
        assert A.is_balanced(g, s_new)
        for lev, c in s_new - s_old:
            par = (lev - 1, tuple(v // 2 for v in c))
            # a new leaf is a child of an old leaf, or a parent whose children were all old leaves
            kids = {(lev + 1, (2 * c[0] + i, 2 * c[1] + j, 2 * c[2] + k))
                    for k in (0, 1) for j in (0, 1) for i in (0, 1)}
            assert par in s_old or kids <= s_old
        m = new


def _linear_problem(g, hp, mesh):
    """rho, p linear in x, y, z and a constant velocity: conserved variables
    linear, so multilinear prolongation reproduces them."""
    def fields(X, Y, Z):
        rho = 1.0 + 0.3 * X + 0.2 * Y + 0.1 * Z
        p = 2.0 + 0.1 * X - 0.2 * Y + 0.3 * Z
        return rho, 0.1 + 0 * X, -0.2 + 0 * X, 0.05 + 0 * X, p
    return A.fill_leaves(mesh, hp, fields), fields


def _interior(unk, g):
    n = g.nguard
    return unk[:, n:-n, n:-n, n:-n, :]


def test_oracle_regrid_prolongs_linear_fields_exactly(oracle):
    g = _geom()
    hp = HydroParams()
    m = _uniform(g)
    unk, fields = _linear_problem(g, hp, m)
    p = oracle.make_params(g.as_dict(), hp)
    old = oracle.Amr(p, m.levels, m.bcoords)
    m2 = A.refine_derefine(m, _flags(m, {(1, (1, 1, 1)): 1, (1, (2, 1, 2)): 1}), lrefine_max=2)
    new = oracle.Amr(p, m2.levels, m2.bcoords)
    u2 = old.regrid(unk, new)
    want = A.fill_leaves(m2, hp, fields)
    got, ref = _interior(u2, g), _interior(want, g)
    for v in (DENS, VELX, VELY, VELZ, PRES, EINT, ENER):
        np.testing.assert_allclose(got[..., v], ref[..., v], rtol=2e-14, atol=2e-15)
    # refining and derefining back: restriction of the prolonged linear data is the original
    kids = {lc: -1 for lc in _leafset(m2) if lc[0] == 2}
    m3 = A.refine_derefine(m2, _flags(m2, kids), lrefine_max=2)
    assert _leafset(m3) == _leafset(m)
    u3 = new.regrid(u2, oracle.Amr(p, m3.levels, m3.bcoords))
    np.testing.assert_allclose(_interior(u3, g)[..., DENS], _interior(unk, g)[..., DENS], rtol=2e-14)


def test_oracle_regrid_identity_and_mass(oracle):
    g = _geom(BC_PERIODIC)
    hp = HydroParams()
    rho_fn = A.levelset_density(g, 3)
    m = A.build_mesh(g, 3, A.gradient_refine(g, rho_fn))
    unk = A.fill_leaves(m, hp, lambda X, Y, Z: (rho_fn(X, Y, Z), 0 * X + 0.1, 0 * X, 0 * X, 0 * X + 1.0))
    p = oracle.make_params(g.as_dict(), hp)
    old = oracle.Amr(p, m.levels, m.bcoords)
    # no marks: the same leaves, Eos applied
    same = old.regrid(unk, oracle.Amr(p, m.levels, m.bcoords))
    np.testing.assert_array_equal(_interior(same, g)[..., DENS], _interior(unk, g)[..., DENS])
    # derefining every complete group: total mass unchanged (restriction averages)
    flags = [-1 if l == 3 else 0 for l in m.levels]
    m2 = A.refine_derefine(m, flags, lrefine_max=3)
    assert m2.nleaf < m.nleaf
    u2 = old.regrid(unk, oracle.Amr(p, m2.levels, m2.bcoords))
    mass0 = old.integrals(unk)[0]
    mass1 = oracle.Amr(p, m2.levels, m2.bcoords).integrals(u2)[0]
    assert abs(mass1 - mass0) <= 1e-13 * abs(mass0)


def test_oracle_regrid_rejects_two_levels(oracle):
    g = _geom()
    hp = HydroParams()
    m = _uniform(g)
    unk, _ = _linear_problem(g, hp, m)
    p = oracle.make_params(g.as_dict(), hp)
    m2 = A.build_mesh(g, 3, lambda lev, c, gg: c == (1, 1, 1) or (lev == 2 and c == (2, 2, 2)))
    with pytest.raises(RuntimeError):
        oracle.Amr(p, m.levels, m.bcoords).regrid(unk, oracle.Amr(p, m2.levels, m2.bcoords))


@pytest.mark.parametrize("ndim,bc", [(3, BC_PERIODIC), (3, BC_OUTFLOW), (2, BC_PERIODIC), (2, BC_OUTFLOW)])
def test_library_tree_update_matches_the_restatement(ndim, bc):
    """fxb_refine_derefine (C++, host only) returns the same leaves, in the
    same Morton order, as amr.refine_derefine for random marks."""
    from flashx_b200.hydro import refine_derefine as native
    rng = np.random.default_rng(11 + ndim)
    g = Geometry(ndim, 8, 8, 8 if ndim == 3 else 1, 3, 2, 2 if ndim == 3 else 1, bc=(bc,) * 6)
    m = A.build_mesh(g, 3, lambda lev, c, gg: (c[0] + 2 * c[1] + c[2]) % 3 == 0)
    for _ in range(5):
        flags = rng.choice([-1, 0, 1], size=m.nleaf, p=[0.45, 0.35, 0.2])
        for lmin, lmax in ((1, 4), (2, 3)):
            a = A.refine_derefine(m, flags, lmin, lmax)
            b = native(m, flags, lmin, lmax)
            assert np.array_equal(a.levels, b.levels) and np.array_equal(a.bcoords, b.bcoords)
        m = A.refine_derefine(m, flags, 1, 4)
