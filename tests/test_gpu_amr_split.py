"""GPU parity of one rank's share of an AMR mesh split over ranks
(flashx_b200.parallel.AmrDecomposition, PARAMESH's Morton distribution).

The device holds the whole mesh, the host UNK only the rank's own leaves;
the device knows the other ranks' leaves its step reads (every other leaf
is set to NaN on the device) and before every step receives their current
interiors through fxb_amr_unpack_leaves, here made from the oracle's
whole-mesh run instead of another rank.  Its own
leaves must then equal the whole-mesh oracle bit for bit after every step
(FP64, -fmad=false; REL_TOL = 1e-12 per value is checked first), and
Hydro_computeDt must equal the oracle's minimum over those leaves.
"""
import numpy as np
import pytest

from flashx_b200 import amr as A
from flashx_b200.hydro import FlashXError, HydroDevice, amr_leaf_message
from flashx_b200.parallel import AmrDecomposition
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, DENS, EINT, ENER, GAMC, GAME,
                                Geometry, HydroParams, PRES, TEMP, VELX, VELY, VELZ)

pytestmark = pytest.mark.gpu

HYDRO_VARS = [DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ]
REL_TOL = 1e-12


def _interior(geom, u):
    g = geom.nguard
    return u[:, g:-g, g:-g, g:-g, :][..., HYDRO_VARS]


class _OracleFeed:
    """Stands in for the other ranks: the ghost leaves' interiors of the
    oracle's current state, unpacked on the device."""

    def __init__(self, dev, geom, ghosts):
        self.dev, self.geom, self.ghosts, self.state, self.msg = dev, geom, ghosts, None, None

    def __call__(self):
        import torch
        msg = torch.from_numpy(amr_leaf_message(self.geom, self.state, self.ghosts)).cuda()
        torch.cuda.synchronize()
        self.dev.unpack_leaves(self.ghosts, msg)
        self.msg = msg        # kept alive until the next call


@pytest.mark.parametrize("world,rank,nroot,maxlev,bc,order", [
    (3, 2, 6, 3, (BC_PERIODIC,) * 6, 3),
    (4, 3, 6, 3, (BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING), 5),
    (4, 3, 8, 2, (BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING), 2),
])
@pytest.mark.parametrize("persistent", [None, "1"])
def test_split_rank_matches_whole_mesh(oracle, need_gpu, monkeypatch, world, rank, nroot, maxlev, bc, order,
                                       persistent):
    if persistent is not None:
        monkeypatch.setenv("FXB_AMR_PERSISTENT", persistent)
    hp = HydroParams(order=order)
    root = Geometry(3, 8, 8, 8, nroot, nroot, nroot, bc=bc)
    mesh, unk = A.levelset_problem(root, hp, maxlev)
    dec = AmrDecomposition(mesh, world, rank)
    own, ghosts = dec.owned(), dec.ghosts[rank]
    known = np.zeros(mesh.nleaf, dtype=bool)
    known[own] = True
    known[ghosts] = True
    assert not known.all(), "the case must leave some leaves unknown to the rank"
    assert maxlev == 2 or np.any(dec.roles == 2), "the case must have flux ghosts"
    am = oracle.Amr(oracle.make_params(root.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    dev = HydroDevice(root, hp, mesh=mesh, amr_split=dec)
    assert dev.unk_shape == (len(own),) + mesh.unk_shape[1:]
    feed = _OracleFeed(dev, root, ghosts)
    dev.exchange = feed
    dev.attach_unk(unk[own].copy())
    import torch
    unknown = np.nonzero(~known)[0]
    poison = torch.full((len(unknown) * dev.lib.fxb_amr_leaf_doubles(),), float("nan"), dtype=torch.float64,
                        device="cuda")
    torch.cuda.synchronize()
    dev.unpack_leaves(unknown, poison)
    u = unk.copy()
    t = 0.0
    for s in range(3):
        feed.state = u
        assert dev.Hydro_computeDt() == am.compute_dt(u, roles=dec.roles)
        dev.Hydro(t + dt, dt, dt)
        am.hydro_step(u, dt)
        t += dt
        feed.state = u
        out = np.zeros(dev.unk_shape)
        dev.sync_to_host(out)
        g, r = _interior(root, out), _interior(root, u)[own]
        assert np.max(np.abs(g - r) / np.maximum(np.abs(r), 1e-300)) <= REL_TOL
        assert np.array_equal(g, r), f"own leaves differ from the whole-mesh step after step {s + 1}"
    assert dev.Hydro_computeDt() == am.compute_dt(u, roles=dec.roles)
    ref = am.integrals(u, roles=dec.roles)
    got = dev.integrals()
    assert np.allclose(got, ref, rtol=1e-12, atol=0)
    dev.close()


def test_leaf_messages_round_trip(need_gpu):
    """fxb_amr_pack_leaves lays a message out as amr_leaf_message does, and
    fxb_amr_unpack_leaves stores it back."""
    import torch
    hp = HydroParams()
    root = Geometry(3, 8, 8, 8, 4, 4, 4, bc=(BC_PERIODIC,) * 6)
    mesh, unk = A.levelset_problem(root, hp, 2)
    dev = HydroDevice(root, hp, mesh=mesh)
    dev.attach_unk(unk.copy())
    leaves = np.array([5, 0, mesh.nleaf - 1, 17, 3])
    buf = torch.empty(len(leaves) * dev.lib.fxb_amr_leaf_doubles(), dtype=torch.float64, device="cuda")
    dev.pack_leaves(leaves, buf)
    torch.cuda.synchronize()
    assert np.array_equal(buf.cpu().numpy(), amr_leaf_message(root, unk, leaves))
    # store leaf 0's interior into leaves 1 and 2, then read the UNK back
    msg = torch.from_numpy(np.concatenate([amr_leaf_message(root, unk, [0])] * 2)).cuda()
    torch.cuda.synchronize()
    dev.unpack_leaves([1, 2], msg)
    out = np.zeros(mesh.unk_shape)
    dev.sync_to_host(out)
    i = _interior(root, out)
    assert np.array_equal(i[1], i[0]) and np.array_equal(i[2], i[0])
    with pytest.raises(FlashXError):
        dev.pack_leaves([mesh.nleaf], buf)
    dev.close()


def _split_worker(rank, world, port, outdir):
    import os
    import sys
    import traceback
    root_dir = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root_dir, os.path.join(root_dir, "flash-x_b200"), os.path.join(root_dir, "tests")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK="0", FXB_AMR_PERSISTENT="0", FXB_AMR_TUNE="0")
    result = "ok"
    try:
        import torch
        from flashx_b200 import parallel as P
        torch.cuda.set_device(0)
        P.init_from_env("gloo", timeout_s=120)
        root, hp, mesh, unk = _split_case()
        dec = AmrDecomposition(mesh, world, rank)
        dev = HydroDevice(root, hp, mesh=mesh, amr_split=dec)
        dev.attach_unk(unk[dec.owned()].copy())
        dt = 0.5 * P.allreduce_min(dev.Hydro_computeDt())
        for _ in range(3):
            dev.Hydro(0.0, dt, dt)
        dtn = P.allreduce_min(dev.Hydro_computeDt())
        out = np.zeros(dev.unk_shape)
        dev.sync_to_host(out)
        integ = P.allreduce_sum(dev.integrals())
        flags, _ = dev.Grid_markRefineDerefine([("dens", 0.3, 0.05, 0.01)], 3)
        m1 = dev.Grid_updateRefinement(flags, lrefine_max=3)
        dev.Hydro(0.0, dt, dt)
        out2 = np.zeros(dev.unk_shape)
        dev.sync_to_host(out2)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), own=dec.owned(), out=out, dt=dt, dtn=dtn,
                 integ=np.array(integ), flags=flags, own2=dev.split.owned(), out2=out2,
                 levels=m1.levels, bcoords=m1.bcoords)
        dev.close()
    except Exception as e:  # noqa: BLE001
        result = f"error: {type(e).__name__}: {e}\n{traceback.format_exc()}"
    with open(os.path.join(outdir, f"result{rank}.txt"), "w") as f:
        f.write(result)
    try:
        import torch.distributed as dist
        if dist.is_initialized() and result == "ok":
            dist.destroy_process_group()
    except Exception:
        pass


def _split_case():
    hp = HydroParams(order=3)
    root = Geometry(3, 8, 8, 8, 6, 6, 6, bc=(BC_PERIODIC,) * 6)
    mesh, unk = A.levelset_problem(root, hp, 2)
    return root, hp, mesh, unk


def test_two_ranks_on_one_gpu_reproduce_the_whole_mesh(oracle, need_gpu):
    """Two ranks, as two processes sharing the GPU and a gloo group (their
    leaf messages cross through pinned host copies; no kernel of one waits for
    the other): each steps its Morton half with the real per-step exchange,
    then both mark and regrid together and step again.  Every rank's own
    leaves, the reduced dt and integrals and the marks equal the whole-mesh
    oracle's, bit for bit (integrals to summation order)."""
    import multiprocessing as mp
    import socket
    import tempfile
    from flashx_b200.params import DENS as _D
    world = 2
    out = tempfile.mkdtemp()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert not p.is_alive(), "a rank did not finish"
    import os
    for r in range(world):
        with open(os.path.join(out, f"result{r}.txt")) as f:
            assert f.read() == "ok"
    ranks = [np.load(os.path.join(out, f"rank{r}.npz")) for r in range(world)]
    root, hp, mesh, unk = _split_case()
    p = oracle.make_params(root.as_dict(), hp)
    am = oracle.Amr(p, mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    assert all(float(d["dt"]) == dt for d in ranks)
    u = unk.copy()
    for _ in range(3):
        am.hydro_step(u, dt)
    assert all(float(d["dtn"]) == am.compute_dt(u) for d in ranks)
    for d in ranks:
        g, r = _interior(root, d["out"]), _interior(root, u)[d["own"]]
        assert np.array_equal(g, r)
        assert np.allclose(d["integ"], am.integrals(u), rtol=1e-12, atol=0)
    flags, _ = am.mark_refine_derefine(u, [(_D, 0.3, 0.05, 0.01)], 3)
    assert all(np.array_equal(d["flags"], flags) for d in ranks)
    m1 = A.refine_derefine(mesh, flags, 1, 3)
    assert all(np.array_equal(d["levels"], m1.levels) and np.array_equal(d["bcoords"], m1.bcoords) for d in ranks)
    am1 = oracle.Amr(p, m1.levels, m1.bcoords)
    u1 = am.regrid(u, am1)
    am1.hydro_step(u1, dt)
    for d in ranks:
        assert np.array_equal(_interior(root, d["out2"]), _interior(root, u1)[d["own2"]])
