"""Block-structured AMR meshes in the PARAMESH layout used by Flash-X.

A mesh is a forest of octrees (quadtrees in 2-D) over the root block grid
nblockx x nblocky x nblockz of a Geometry.  Level 1 holds the root blocks;
a block at level l has block coordinates c in [0, nblock * 2**(l-1)) and
covers the cells c * n .. c * n + n - 1 of the level-l cell index space; its
cell size is the root cell size halved l-1 times
(FX/Grid/GridMain/AMR/Paramesh4/gr_initSpecific.F90:169-184).  The leaf list
(level, block coordinates) in Morton order is what the C ABI's
fxb_register_blocks takes and what Flash-X's LEAF tile iterator produces.

Refinement follows the Flash-X/PARAMESH rule that neighbouring leaves,
across faces, edges and corners, differ by at most one level
(PARAMESH's proper nesting with diagonals = .true.); `build_mesh` refines
where a criterion asks for it and then refines coarse neighbours until that
holds.  `refine_derefine` is the tree update of a regrid during a run
(PARAMESH's amr_refine_derefine) from per-leaf refine/derefine marks; the
device moves the data to the new leaves (fxb_regrid).
"""
import math

import numpy as np

from .params import (DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ,
                     BC_PERIODIC, Geometry, HydroParams, NUNK)
from . import simulations as S


def _morton_key(level, c, maxlev):
    """Interleave the block coordinates scaled to the finest level."""
    sh = maxlev - level
    x, y, z = (int(v) << sh for v in c)
    key = 0
    for b in range(21):
        key |= ((x >> b) & 1) << (3 * b) | ((y >> b) & 1) << (3 * b + 1) | ((z >> b) & 1) << (3 * b + 2)
    return (key, level)


class AmrMesh:
    """Leaf blocks of a balanced block-structured mesh."""

    def __init__(self, geom: Geometry, leaves):
        self.geom = geom
        self.maxlev = max(l for l, _ in leaves)
        order = sorted(leaves, key=lambda lc: _morton_key(lc[0], lc[1], self.maxlev))
        self.levels = np.array([l for l, _ in order], dtype=np.int32)
        self.bcoords = np.array([list(c) for _, c in order], dtype=np.int32).reshape(-1, 3)

    @property
    def nleaf(self):
        return len(self.levels)

    @property
    def unk_shape(self):
        g = self.geom
        return (self.nleaf,) + g.unk_shape[1:]

    def ncells(self):
        g = self.geom
        return self.nleaf * g.nxb * (g.nyb if g.ndim >= 2 else 1) * (g.nzb if g.ndim == 3 else 1)

    def deltas(self, level):
        d = list(self.geom.deltas())
        for a in range(self.geom.ndim):
            for _ in range(level - 1):
                d[a] = d[a] / 2.0
        return tuple(d)

    def leaf_centres(self, leaf):
        """Cell-centre coordinates (xc, yc, zc) of one leaf's interior."""
        g = self.geom
        lev = int(self.levels[leaf])
        c = self.bcoords[leaf]
        dx, dy, dz = self.deltas(lev)
        (x0, _), (y0, _), (z0, _) = g.bbox
        xc = x0 + (c[0] * g.nxb + np.arange(g.nxb) + 0.5) * dx
        yc = y0 + (c[1] * g.nyb + np.arange(g.nyb) + 0.5) * dy if g.ndim >= 2 else np.zeros(1)
        zc = z0 + (c[2] * g.nzb + np.arange(g.nzb) + 0.5) * dz if g.ndim == 3 else np.zeros(1)
        return xc, yc, zc

    def level_counts(self):
        return {int(l): int(np.sum(self.levels == l)) for l in np.unique(self.levels)}


def _nb(geom, level, d):
    n0 = (geom.nblockx, geom.nblocky, geom.nblockz)[d]
    if d >= geom.ndim:
        return 1
    return n0 << (level - 1)


def _covering_leaf(leaves, level, c):
    """Leaf covering block position c at `level`: (level', coords) or None
    when the region is refined beyond `level`."""
    lev, cc = level, tuple(c)
    while lev >= 1:
        if (lev, cc) in leaves:
            return lev, cc
        lev -= 1
        cc = tuple(v // 2 for v in cc)
    return None


def _neighbour_positions(geom, level, c):
    K3 = 1 if geom.ndim == 3 else 0
    out = []
    for dk in range(-K3, K3 + 1):
        for dj in (-1, 0, 1):
            for di in (-1, 0, 1):
                if di == dj == dk == 0:
                    continue
                p = [c[0] + di, c[1] + dj, c[2] + dk]
                ok = True
                for d in range(3):
                    nb = _nb(geom, level, d)
                    if p[d] < 0 or p[d] >= nb:
                        if geom.bc[2 * d + (p[d] >= nb)] != BC_PERIODIC:
                            ok = False
                            break
                        p[d] %= nb
                if ok:
                    out.append(tuple(p))
    return out


def _children(geom, level, c):
    K3 = 1 if geom.ndim == 3 else 0
    return [(level + 1, (2 * c[0] + i, 2 * c[1] + j, 2 * c[2] + k))
            for k in range(K3 + 1) for j in range(2) for i in range(2)]


def build_mesh(geom: Geometry, maxlev, refine):
    """Refine the root blocks level by level where refine(level, coords, mesh_geom)
    returns True (coords = block coordinates at that level), then refine
    coarse neighbours until every leaf's neighbours are within one level."""
    leaves = set()
    for k in range(_nb(geom, 1, 2)):
        for j in range(_nb(geom, 1, 1)):
            for i in range(_nb(geom, 1, 0)):
                leaves.add((1, (i, j, k)))
    for lev in range(1, maxlev):
        marked = [lc for lc in leaves if lc[0] == lev and refine(lev, lc[1], geom)]
        for lc in marked:
            leaves.discard(lc)
            leaves.update(_children(geom, *lc))
        _balance(geom, leaves)
    return AmrMesh(geom, sorted(leaves))


def _balance(geom, leaves):
    changed = True
    while changed:
        changed = False
        for lev, c in sorted(leaves, key=lambda lc: -lc[0]):
            if (lev, c) not in leaves:
                continue
            for p in _neighbour_positions(geom, lev, c):
                cov = _covering_leaf(leaves, lev, p)
                if cov is not None and cov[0] < lev - 1:
                    leaves.discard(cov)
                    leaves.update(_children(geom, *cov))
                    changed = True


def is_balanced(geom, leaves):
    """Every leaf's neighbours (faces, edges, corners) within one level."""
    leaves = set(leaves)
    for lev, c in leaves:
        for p in _neighbour_positions(geom, lev, c):
            cov = _covering_leaf(leaves, lev, p)
            if cov is not None and cov[0] < lev - 1:
                return False
    return True


def refine_derefine(mesh: AmrMesh, flags, lrefine_min=1, lrefine_max=None):
    """PARAMESH's tree update (PM4_package/source/mpi_amr_refine_derefine.F90)
    for leaf marks flags[leaf] = 1 refine, -1 derefine, 0 neither (what
    Grid_markRefineDerefine / fxb_mark_refine_derefine returns, in the mesh's
    leaf order).  Returns the new AmrMesh.

    * level limits (mpi_amr_refine_derefine.F90:157-163): no refinement at
      lrefine_max, no derefinement at lrefine_min, refinement below it;
    * amr_check_refine: a leaf one level coarser than a refining neighbour
      (faces, edges, corners) refines too, until nothing changes, and is no
      longer derefined;
    * amr_check_derefine (mpi_amr_check_derefine.F90): a leaf derefines only
      if it is not a root block, none of its same-level neighbours is a parent
      or refines, and all its siblings are leaves that derefine as well; the
      siblings are then replaced by their parent.
    """
    g = mesh.geom
    lmax = lrefine_max if lrefine_max is not None else mesh.maxlev + 1
    order = [(int(l), tuple(int(v) for v in c)) for l, c in zip(mesh.levels, mesh.bcoords)]
    leaves = set(order)
    flags = [int(f) for f in flags]
    if len(flags) != len(order):
        raise ValueError("one mark per leaf")
    refine = {lc: f == 1 for lc, f in zip(order, flags)}
    derefine = {lc: f == -1 for lc, f in zip(order, flags)}
    for lc in order:
        if lc[0] >= lmax:
            refine[lc] = False
        if lc[0] == lrefine_min:
            derefine[lc] = False
        if lc[0] < lrefine_min:
            refine[lc] = True
    changed = True
    while changed:
        changed = False
        for lc in order:
            if not refine[lc]:
                continue
            lev, c = lc
            for p in _neighbour_positions(g, lev, c):
                cov = _covering_leaf(leaves, lev, p)
                if cov is not None and cov[0] < lev and not refine[cov]:
                    refine[cov] = True
                    derefine[cov] = False
                    changed = True
    nch = 8 if g.ndim == 3 else 4
    groups = {}
    for lc in order:
        lev, c = lc
        if not derefine[lc] or refine[lc] or lev == 1:
            continue
        blocked = False
        for p in _neighbour_positions(g, lev, c):
            same = (lev, p)
            if same in leaves:
                blocked = refine[same]
            else:
                blocked = _covering_leaf(leaves, lev, p) is None   # a parent at this level
            if blocked:
                break
        if not blocked:
            groups.setdefault((lev - 1, tuple(v // 2 for v in c)), []).append(lc)
    new = set(leaves)
    for lc in order:
        if refine[lc]:
            new.discard(lc)
            new.update(_children(g, *lc))
    for par, kids in groups.items():
        if len(kids) == nch:
            new.difference_update(kids)
            new.add(par)
    return AmrMesh(g, sorted(new))


def mesh_from_levels(geom: Geometry, leaves):
    return AmrMesh(geom, leaves)


# ------------------------------------------------------------------ AMR problem
def _levelset(geom, nmodes=8, amp=0.08, seed_stream=20):
    """Seeded interface z = 0.5 + sum of random-phase Fourier modes in x, y
    (y = 0.5 + modes in x in 2-D)."""
    a, b = S.uniform01(np.arange(nmodes, dtype=np.uint64), stream=seed_stream)
    c, d = S.uniform01(np.arange(nmodes, dtype=np.uint64), stream=seed_stream + 1)
    kx = 1.0 + np.floor(3.0 * a)
    ky = 1.0 + np.floor(3.0 * b)
    ph = 2.0 * math.pi * c
    am = amp * (0.5 + d) / nmodes * 2.0

    def phi(X, Y, Z):
        s = np.zeros_like(X)
        for m in range(nmodes):
            arg = kx[m] * X + ky[m] * Y if geom.ndim == 3 else kx[m] * X
            s = s + am[m] * np.sin(2.0 * math.pi * arg + ph[m])
        if geom.ndim == 3:
            return Z - 0.5 - s
        return Y - 0.5 - s
    return phi


def levelset_density(geom, maxlev, rho_lo=1.0, rho_hi=10.0, cells=2.0):
    """Density 1 below and 10 above the seeded interface, smoothed by tanh
    over `cells` cells of the finest level."""
    phi = _levelset(geom)
    dfine = min(geom.deltas()[:geom.ndim]) / 2.0 ** (maxlev - 1)
    w = cells * dfine

    def rho(X, Y, Z):
        return rho_lo + (rho_hi - rho_lo) * 0.5 * (1.0 + np.tanh(phi(X, Y, Z) / w))
    return rho


def gradient_refine(geom, rho_fn, threshold=0.1):
    """Refine a block where max |grad rho| / rho * dx over its cells exceeds
    the threshold, sampled at the block's own resolution (central
    differences, as gr_estimateError's first-derivative test)."""
    def refine(level, c, g):
        nx, ny, nz = g.nxb, (g.nyb if g.ndim >= 2 else 1), (g.nzb if g.ndim == 3 else 1)
        d = list(g.deltas())
        d = [v / 2.0 ** (level - 1) for v in d]
        (x0, _), (y0, _), (z0, _) = g.bbox
        xc = x0 + (c[0] * nx + np.arange(-1, nx + 1) + 0.5) * d[0]
        yc = y0 + (c[1] * ny + np.arange(-1, ny + 1) + 0.5) * d[1]
        zc = z0 + (c[2] * nz + np.arange(-1, nz + 1) + 0.5) * d[2] if g.ndim == 3 else np.zeros(1)
        Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
        r = rho_fn(X, Y, Z)
        kk = slice(1, -1) if g.ndim == 3 else slice(None)
        rc = r[kk, 1:-1, 1:-1]
        err = np.abs(r[kk, 1:-1, 2:] - r[kk, 1:-1, :-2]) * 0.5 / rc
        err = np.maximum(err, np.abs(r[kk, 2:, 1:-1] - r[kk, :-2, 1:-1]) * 0.5 / rc)
        if g.ndim == 3:
            err = np.maximum(err, np.abs(r[2:, 1:-1, 1:-1] - r[:-2, 1:-1, 1:-1]) * 0.5 / rc)
        return bool(np.max(err) > threshold)
    return refine


def fill_leaves(mesh: AmrMesh, hp: HydroParams, fields):
    """Leaf UNK (nleaf, k, j, i, var) from fields(X, Y, Z) -> (rho, vx, vy, vz, p)
    evaluated at each leaf's cell centres; guard cells zeroed."""
    g = mesh.geom
    unk = np.zeros(mesh.unk_shape)
    gk = g.nguard if g.ndim == 3 else 0
    gj = g.nguard if g.ndim >= 2 else 0
    gi = g.nguard
    for l in range(mesh.nleaf):
        xc, yc, zc = mesh.leaf_centres(l)
        Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
        rho, vx, vy, vz, p = fields(X, Y, Z)
        f = S._finish(hp, rho, vx, vy, vz, p)
        unk[l, gk:gk + Z.shape[0], gj:gj + Z.shape[1], gi:gi + Z.shape[2], :] = f
    return unk


def levelset_problem(geom: Geometry, hp: HydroParams, maxlev, threshold=0.1):
    """AMR benchmark problem: the seeded level-set density interface
    (rho 1 vs 10, tanh over 2 finest cells), p = 2.5, advected by a uniform
    velocity (0.25, 0.125, 0.0625) with a small vortical perturbation.
    Returns (mesh, leaf UNK)."""
    rho_fn = levelset_density(geom, maxlev)
    mesh = build_mesh(geom, maxlev, gradient_refine(geom, rho_fn, threshold))

    def fields(X, Y, Z):
        rho = rho_fn(X, Y, Z)
        s = 0.02 * np.sin(2.0 * math.pi * X) * np.sin(2.0 * math.pi * Y)
        vx = 0.25 + s
        vy = 0.125 - s
        vz = 0.0625 + 0.0 * X if geom.ndim == 3 else 0.0 * X
        p = np.full_like(rho, 2.5)
        return rho, vx, vy, vz, p
    return mesh, fill_leaves(mesh, hp, fields)


def stack_copies(mesh: AmrMesh, copies):
    """`copies` copies of a mesh stacked along the slowest axis (z in 3-D, y
    in 2-D), that axis' extent and root blocks multiplied: the mesh of a
    weak-scaling run split over `copies` ranks.  The copies are whole
    root-block layers, which the Morton order visits one after the other, so
    copy c is the leaf range [c n, (c + 1) n) of the result, its leaves in
    the order of `mesh` (a rank owning that range holds `mesh`'s leaf UNK).
    Returns (geometry, mesh)."""
    import dataclasses
    g = mesh.geom
    ax = g.ndim - 1
    key = ("nblockx", "nblocky", "nblockz")[ax]
    bbox = list(g.bbox)
    lo, hi = bbox[ax]
    bbox[ax] = (lo, lo + copies * (hi - lo))
    whole = dataclasses.replace(g, bbox=tuple(bbox), **{key: getattr(g, key) * copies})
    nroot = getattr(g, key)
    lev = mesh.levels.astype(np.int64)
    leaves = []
    for c in range(copies):
        b = mesh.bcoords.astype(np.int64).copy()
        b[:, ax] += c * (nroot << (lev - 1))
        leaves += [(int(l), tuple(int(v) for v in bc)) for l, bc in zip(lev, b)]
    out = AmrMesh(whole, leaves)
    n = mesh.nleaf
    for c in range(copies):
        b = out.bcoords[c * n:(c + 1) * n].astype(np.int64)
        b[:, ax] -= c * (nroot << (out.levels[c * n:(c + 1) * n].astype(np.int64) - 1))
        if not (np.array_equal(b, mesh.bcoords) and np.array_equal(out.levels[c * n:(c + 1) * n], mesh.levels)):
            raise ValueError("stack_copies: the copies are not contiguous in Morton order")
    return whole, out
