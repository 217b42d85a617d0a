"""AMR meshes split over ranks (CPU, gloo): the Morton-range decomposition,
its ghost and flux-ghost sets, and oracle ranks that exchange leaf data once
per step and reproduce the single-process AMR step bit for bit, dt sequence
included.  Every leaf a rank neither owns nor receives is set to NaN before
the run, so a dependency the ghost set misses shows up in the result."""
import os
import socket
import tempfile

import multiprocessing as mp
import numpy as np
import pytest

from flashx_b200 import amr as A
from flashx_b200.params import BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, Geometry, HydroParams

NSTEPS = 5


def _case(name):
    if name == "amr2d":
        root = Geometry(2, 8, 8, 1, 16, 16, 1, bc=(BC_PERIODIC,) * 4 + (BC_OUTFLOW,) * 2)
        hp = HydroParams(order=3)
        mesh, unk = A.levelset_problem(root, hp, 3)
    else:
        root = Geometry(3, 8, 8, 8, 4, 4, 4, bc=(BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW,
                                                   BC_REFLECTING, BC_REFLECTING))
        hp = HydroParams(order=5)
        mesh, unk = A.levelset_problem(root, hp, 2)
    return root, hp, mesh, unk


def test_decomposition_sets():
    from flashx_b200.parallel import AmrDecomposition
    root, hp, mesh, unk = _case("amr2d")
    for world in (1, 2, 3):
        decs = [AmrDecomposition(mesh, world, r) for r in range(world)]
        owned = np.concatenate([d.owned() for d in decs])
        assert np.array_equal(owned, np.arange(mesh.nleaf))          # contiguous Morton ranges, each leaf once
        for d in decs:
            gh = d.ghosts[d.rank]
            assert not np.any(d.owner[gh] == d.rank)
            fg = np.nonzero(d.roles == 2)[0]
            assert set(fg) <= set(gh)                               # flux ghosts are received
            assert np.all(np.asarray(mesh.levels)[fg] >= 2)
            for s, leaves in d.sends().items():                     # what one sends, the other receives
                assert np.array_equal(leaves, decs[s].recvs()[d.rank])
        if world == 1:
            assert len(decs[0].ghosts[0]) == 0 and not np.any(decs[0].roles == 2)
    # adjacency is symmetric and includes periodic neighbours
    d = AmrDecomposition(mesh, 2, 0)
    for i in range(mesh.nleaf):
        for j in d._touch[i]:
            assert i in d._touch[int(j)]
    # some leaves are neither owned nor received, so the NaN test below means something
    assert np.sum(d.roles == 1) + len(d.ghosts[0]) < mesh.nleaf


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, outdir, name):
    import sys
    root_dir = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root_dir, os.path.join(root_dir, "flash-x_b200"), os.path.join(root_dir, "tests")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    result = "ok"
    try:
        import torch
        from flashx_b200 import parallel as P
        from oracle import fx_oracle as O
        P.init_from_env("gloo", timeout_s=60)
        root, hp, mesh, unk = _case(name)
        am = O.Amr(O.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
        dec = P.AmrDecomposition(mesh, world, rank)
        u = unk.copy()
        known = np.zeros(mesh.nleaf, dtype=bool)
        known[dec.owned()] = True
        known[dec.ghosts[rank]] = True
        u[~known] = np.nan                       # never read: any use would leak NaN into the result
        shape = u.shape[1:]

        def pack(leaves, buf):
            buf.copy_(torch.from_numpy(np.ascontiguousarray(u[leaves]).reshape(-1)))

        def unpack(leaves, buf):
            u[leaves] = buf.numpy().reshape((len(leaves),) + shape)

        ex = P.AmrExchange(dec, int(np.prod(shape)), pack, unpack, device=torch.device("cpu"))
        dt = 0.5 * P.allreduce_min(am.compute_dt(u, dec.roles))
        dts = [dt]
        for _ in range(NSTEPS):
            ex()
            am.hydro_step(u, dt, roles=dec.roles)
            dt = O.driver_dt(P.allreduce_min(am.compute_dt(u, dec.roles)), dt)
            dts.append(dt)
        sums = P.allreduce_sum(am.integrals(u, dec.roles))
        own = dec.owned()
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), leaves=own, data=u[own], dts=np.array(dts),
                 sums=np.array(sums))
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


@pytest.mark.parametrize("name,world", [("amr2d", 2), ("amr2d", 3), ("amr3d", 2), ("amr3d", 3)])
def test_amr_ranks_reproduce_the_whole_mesh_gloo(name, world, oracle):
    out = tempfile.mkdtemp()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out, name)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        if p.is_alive():
            p.kill()
            pytest.fail("AMR rank did not finish")
    res = [open(os.path.join(out, f"result{r}.txt")).read() for r in range(world)]
    assert res == ["ok"] * world, res
    root, hp, mesh, unk = _case(name)
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    u = unk.copy()
    dt = 0.5 * am.compute_dt(u)
    dts = [dt]
    for _ in range(NSTEPS):
        am.hydro_step(u, dt)
        dt = oracle.driver_dt(am.compute_dt(u), dt)
        dts.append(dt)
    g = root.nguard
    inner = (slice(None),) + ((slice(g, -g),) if root.ndim == 3 else (slice(None),)) + (slice(g, -g), slice(g, -g))
    covered = 0
    for r in range(world):
        z = np.load(os.path.join(out, f"rank{r}.npz"))
        assert np.array_equal(z["dts"], np.array(dts)), (r, z["dts"], dts)
        np.testing.assert_array_equal(z["data"][inner], u[z["leaves"]][inner])
        covered += len(z["leaves"])
        sums = z["sums"]
    assert covered == mesh.nleaf
    np.testing.assert_allclose(sums, am.integrals(u), rtol=1e-12, atol=1e-12)


def _touch_brute_force(mesh):
    """Every pair of leaves tested: closed boxes (finest-cell units) that meet
    on every axis, periodic axes wrapped; face neighbours overlap with positive
    length on all axes but one."""
    g = mesh.geom
    nd = g.ndim
    L = int(mesh.maxlev)
    lev = np.asarray(mesh.levels, dtype=np.int64)
    sc = 1 << (L - lev)
    lo = np.asarray(mesh.bcoords, dtype=np.int64)[:, :nd] * sc[:, None]
    hi = lo + sc[:, None]
    ext = [b << (L - 1) for b in (g.nblockx, g.nblocky, g.nblockz)[:nd]]
    touch, face = [], []
    for i in range(mesh.nleaf):
        t, f = [], []
        for j in range(mesh.nleaf):
            if i == j:
                continue
            meet, nover = True, 0
            for a in range(nd):
                sh = (-ext[a], 0, ext[a]) if g.bc[2 * a] == BC_PERIODIC else (0,)
                meet &= any(lo[i, a] <= hi[j, a] + s and lo[j, a] + s <= hi[i, a] for s in sh)
                nover += any(lo[i, a] < hi[j, a] + s and lo[j, a] + s < hi[i, a] for s in sh)
            if meet:
                t.append(j)
                if nover == nd - 1:
                    f.append(j)
        touch.append(t)
        face.append(f)
    return touch, face


@pytest.mark.parametrize("ndim,nroot,maxlev,bc", [
    (2, 4, 3, (BC_PERIODIC,) * 4 + (BC_OUTFLOW,) * 2),
    (2, 2, 3, (BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW)),
    (2, 1, 3, (BC_PERIODIC,) * 4 + (BC_OUTFLOW,) * 2),
    (3, 2, 2, (BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW, BC_REFLECTING, BC_REFLECTING)),
    (3, 3, 2, (BC_PERIODIC,) * 6),
])
def test_adjacency_matches_all_pairs(ndim, nroot, maxlev, bc):
    """The root-block buckets of AmrDecomposition._adjacency find the same
    neighbours as testing every pair (one and two root blocks per periodic
    axis included, where a neighbour is reached across both sides)."""
    from flashx_b200.parallel import AmrDecomposition
    if ndim == 2:
        root = Geometry(2, 8, 8, 1, nroot, nroot, 1, bc=bc)
    else:
        root = Geometry(3, 8, 8, 8, nroot, nroot, nroot, bc=bc)
    mesh, _ = A.levelset_problem(root, HydroParams(), maxlev)
    touch, face = AmrDecomposition._adjacency(mesh)
    bt, bf = _touch_brute_force(mesh)
    for i in range(mesh.nleaf):
        assert list(touch[i]) == bt[i] and list(face[i]) == bf[i], f"leaf {i}"


@pytest.mark.parametrize("ndim", [2, 3])
def test_stacked_copies_step_like_the_single_mesh(ndim, oracle):
    """The weak-scaling mesh: `world` copies of a periodic mesh stacked along
    the slowest axis.  Copy r is rank r's Morton range, and the oracle's
    whole-mesh step of the stacked mesh leaves every copy equal, bit for bit,
    to the step of the single mesh (the copies join like the periodic
    boundary they replace)."""
    from flashx_b200.parallel import AmrDecomposition
    if ndim == 2:
        root = Geometry(2, 8, 8, 1, 4, 4, 1, bc=(BC_PERIODIC,) * 4 + (BC_OUTFLOW,) * 2)
        mesh, unk = A.levelset_problem(root, HydroParams(order=3), 3)
    else:
        root = Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
        mesh, unk = A.levelset_problem(root, HydroParams(order=3), 2)
    hp = HydroParams(order=3)
    world = 3
    whole, wmesh = A.stack_copies(mesh, world)
    n = mesh.nleaf
    assert wmesh.nleaf == world * n
    for r in range(world):
        d = AmrDecomposition(wmesh, world, r)
        assert np.array_equal(d.owned(), np.arange(r * n, (r + 1) * n))
    one = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    many = oracle.Amr(oracle.make_params(whole.as_dict(), hp), wmesh.levels, wmesh.bcoords)
    u1, uw = unk.copy(), np.concatenate([unk] * world, axis=0)
    dt = 0.5 * one.compute_dt(u1)
    assert many.compute_dt(uw) == one.compute_dt(u1)
    for _ in range(2):
        one.hydro_step(u1, dt)
        many.hydro_step(uw, dt)
    g = root.nguard
    sl = (slice(None), slice(g, -g) if ndim == 3 else slice(None), slice(g, -g), slice(g, -g))
    for r in range(world):
        assert np.array_equal(uw[r * n:(r + 1) * n][sl], u1[sl]), f"copy {r}"
