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
