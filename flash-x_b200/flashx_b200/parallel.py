"""Multi-process driver logic: one process per GPU.

Flash-X advances every rank with one global time step: Driver_computeDt
reduces the per-rank CFL minimum with MPI_AllReduce(MIN)
(Driver/DriverMain/Driver_computeDt.F90:373,383) before the growth limit and
clamp, and IO_writeIntegralQuantities sums the conserved integrals with
MPI_Reduce(SUM) (IO/IOMain/IO_writeIntegralQuantities.F90:224).  Here those two
reductions run over torch.distributed (NCCL between GPUs, gloo on CPU).

`ReplicaDriver` advances one independent problem per rank with that common
dt.  `SlabDecomposition` splits one uniform block grid over the ranks along
its slowest axis and `HaloExchange` moves the guard planes between
neighbouring slabs before every step, as the UG Grid_fillGuardCells does with
MPI_SendRecv along each process axis (Grid/GridMain/UG/Grid_fillGuardCells.F90:
261-306, UG/gr_shiftData.F90:63-191).
"""
import datetime
import os

import numpy as np
import torch
import torch.distributed as dist

from .hydro import driver_dt, initial_dt
from .params import BC_PERIODIC


def init_from_env(backend, timeout_s=120):
    """init_process_group from RANK/WORLD_SIZE/MASTER_* (torchrun); returns
    (world, rank, local_rank); a no-op (1, 0, 0) without WORLD_SIZE > 1."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return 1, 0, int(os.environ.get("LOCAL_RANK", "0"))
    if not dist.is_initialized():
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist.get_world_size(), dist.get_rank(), int(os.environ.get("LOCAL_RANK", "0"))


def _device():
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def allreduce_min(x):
    """Driver_computeDt's MPI_AllReduce(MIN) of one FP64 value."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return float(t.item())


def allreduce_max(x):
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(values):
    """IO_writeIntegralQuantities' MPI_Reduce(SUM) of the integral vector."""
    vals = [float(v) for v in values]
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().tolist()


class ReplicaDriver:
    """Driver_evolveAll for one problem per rank with a common dt, or for the
    slabs of one grid (a HydroDevice built with a SlabDecomposition exchanges
    its halos inside Hydro, as Hydro's own Grid_fillGuardCells).

    `dev` exposes the hydro interface (Hydro, Hydro_computeDt), e.g.
    flashx_b200.hydro.HydroDevice.  Every rank makes the same collective
    calls in the same order, in warm-up, timing and error paths alike."""

    def __init__(self, dev, hp):
        self.dev, self.hp = dev, hp
        self.t = 0.0

    def first_dt(self):
        """Driver_verifyInitDt.F90:234-250 on the global CFL dt."""
        return initial_dt(allreduce_min(self.dev.Hydro_computeDt()), self.hp)

    def step(self, dt, dt_old):
        """Hydro, then Driver_computeDt; returns (dt_new, dt)."""
        self.t += dt
        self.dev.Hydro(self.t, dt, dt_old)
        dt_cfl = allreduce_min(self.dev.Hydro_computeDt())
        return driver_dt(dt_cfl, dt, self.hp), dt

    def run(self, nsteps, dt, dt_old):
        for _ in range(nsteps):
            dt, dt_old = self.step(dt, dt_old)
        return dt, dt_old


class SlabDecomposition:
    """Split of a uniform block grid over `nranks` ranks along its slowest
    axis (y in 2-D, z in 3-D): rank r holds the contiguous, balanced block
    layers `layers[r]` (every block of each layer, so its blocks are one
    contiguous range of the grid's block list) and halo planes below and
    above them.  A side facing another slab, or the periodic wrap, has a halo
    of at least NGUARD planes, widened until the stored extent (interior plus
    halos) is a multiple of `tile` (16 for the 2-D kernels' tiles); a
    physical boundary has none.  `self_halo` gives a single rank halos on a
    periodic axis that it fills from its own planes (the exchange without a
    neighbour).  Flash-X's UG places blocks on an iProcs x jProcs x kProcs
    process grid (UG/gr_createDomain.F90); this is its one-axis case."""

    def __init__(self, geom, nranks, rank, tile=None, self_halo=False):
        if not 0 <= rank < nranks:
            raise ValueError("rank outside [0, nranks)")
        self.ndim = geom.ndim
        self.axis = geom.ndim - 1
        nlay = geom.nblocky if geom.ndim == 2 else geom.nblockz
        self.nb = geom.nyb if geom.ndim == 2 else geom.nzb
        self.per_layer = geom.nblockx * (geom.nblocky if geom.ndim == 3 else 1)
        if nranks > nlay:
            raise ValueError(f"{nranks} ranks for {nlay} block layers")
        self.nranks, self.rank, self.nlay = nranks, rank, nlay
        self.tile = tile if tile is not None else (16 if geom.ndim == 2 else 1)
        self.nguard = geom.nguard
        periodic = geom.bc[2 * self.axis] == BC_PERIODIC
        self.layers = [(r * nlay // nranks, (r + 1) * nlay // nranks) for r in range(nranks)]
        wrap = periodic and (nranks > 1 or self_halo)
        self.halos = []
        for r, (lo, hi) in enumerate(self.layers):
            has_lo, has_hi = r > 0 or wrap, r < nranks - 1 or wrap
            self.halos.append(self._widths((hi - lo) * self.nb, has_lo, has_hi))
        for r in range(nranks):
            for side, nbr in ((0, self._nbr(r, -1)), (1, self._nbr(r, +1))):
                h = self.halos[r][side]
                if h and h > self.interior_planes(nbr):
                    raise ValueError(f"halo of {h} planes exceeds rank {nbr}'s {self.interior_planes(nbr)} planes")

    def _widths(self, interior, has_lo, has_hi):
        hl = self.nguard if has_lo else 0
        hh = self.nguard if has_hi else 0
        if (has_lo or has_hi) and self.tile > 1:
            while (interior + hl + hh) % self.tile:
                if has_hi and (not has_lo or hh <= hl):
                    hh += 1
                else:
                    hl += 1
        elif (interior + hl + hh) % self.tile:
            raise ValueError("a slab without halos must fill whole tiles")
        return hl, hh

    def _nbr(self, r, step):
        return (r + step) % self.nranks

    def interior_planes(self, r=None):
        lo, hi = self.layers[self.rank if r is None else r]
        return (hi - lo) * self.nb

    @property
    def layer_lo(self):
        return self.layers[self.rank][0]

    @property
    def layer_hi(self):
        return self.layers[self.rank][1]

    @property
    def halo_lo(self):
        return self.halos[self.rank][0]

    @property
    def halo_hi(self):
        return self.halos[self.rank][1]

    @property
    def lo_rank(self):
        return self._nbr(self.rank, -1) if self.halo_lo else None

    @property
    def hi_rank(self):
        return self._nbr(self.rank, +1) if self.halo_hi else None

    @property
    def send_lo(self):
        """Planes sent down: the lower neighbour's upper halo."""
        return self.halos[self.lo_rank][1] if self.halo_lo else 0

    @property
    def send_hi(self):
        """Planes sent up: the upper neighbour's lower halo."""
        return self.halos[self.hi_rank][0] if self.halo_hi else 0

    def block_range(self):
        """This rank's blocks: [b0, b1) of the whole grid's block list."""
        return self.layer_lo * self.per_layer, self.layer_hi * self.per_layer

    def local_blocks(self, unk):
        """This rank's part of a whole-grid UNK (a view)."""
        b0, b1 = self.block_range()
        return unk[b0:b1]


class HaloExchange:
    """One guard-plane exchange between slabs: pack this rank's boundary
    planes, send them to the neighbours and receive theirs (point-to-point,
    NCCL between GPUs, gloo on CPU), unpack into the halos.

    pack(send_lo, n_lo, send_hi, n_hi) and unpack(recv_lo, recv_hi) move
    planes between the state and flat FP64 tensors of
    `doubles_per_plane` x planes values (None where a count is 0).  Messages
    are matched per neighbour pair in issue order, downward planes (tag 0)
    before upward planes (tag 1), so two ranks that are each other's lower
    and upper neighbour (a periodic pair) pair them correctly.  A rank that
    is its own neighbour packs straight into its receive buffers.
    host_stage: the planes are packed in device memory but cross between the
    ranks through pinned host copies (a process group whose backend moves
    host memory, e.g. gloo between processes that share a GPU)."""

    def __init__(self, dec, doubles_per_plane, pack, unpack, device="cpu", stream=None, host_stage=False):
        self.dec, self.pack, self.unpack, self.stream = dec, pack, unpack, stream
        buf = lambda n: torch.empty(n * doubles_per_plane, dtype=torch.float64, device=device) if n else None
        self.send_lo, self.send_hi = buf(dec.send_lo), buf(dec.send_hi)
        self.recv_lo, self.recv_hi = buf(dec.halo_lo), buf(dec.halo_hi)
        self.own_neighbour = dec.nranks == 1
        self.host_stage = host_stage and not self.own_neighbour
        if self.host_stage:
            pin = lambda b: torch.empty(b.numel(), dtype=torch.float64, pin_memory=True) if b is not None else None
            self.h = {k: pin(getattr(self, k)) for k in ("send_lo", "send_hi", "recv_lo", "recv_hi")}

    def __call__(self):
        d = self.dec
        if not (d.halo_lo or d.halo_hi):
            return
        if self.stream is not None:
            with torch.cuda.stream(self.stream):
                self._run(d)
        else:
            self._run(d)

    def _run(self, d):
        if self.own_neighbour:
            self.pack(self.recv_hi, d.send_lo, self.recv_lo, d.send_hi)
        else:
            self.pack(self.send_lo, d.send_lo, self.send_hi, d.send_hi)
            b = {k: getattr(self, k) for k in ("send_lo", "send_hi", "recv_lo", "recv_hi")}
            if self.host_stage:
                for k in ("send_lo", "send_hi"):
                    if b[k] is not None:
                        self.h[k].copy_(b[k], non_blocking=True)
                torch.cuda.current_stream().synchronize()
                b = self.h
            ops = []
            if d.halo_lo:
                ops.append(dist.P2POp(dist.isend, b["send_lo"], d.lo_rank, tag=0))
            if d.halo_hi:
                ops.append(dist.P2POp(dist.irecv, b["recv_hi"], d.hi_rank, tag=0))
            if d.halo_hi:
                ops.append(dist.P2POp(dist.isend, b["send_hi"], d.hi_rank, tag=1))
            if d.halo_lo:
                ops.append(dist.P2POp(dist.irecv, b["recv_lo"], d.lo_rank, tag=1))
            for req in dist.batch_isend_irecv(ops):
                req.wait()
            if self.host_stage:
                for k in ("recv_lo", "recv_hi"):
                    if b[k] is not None:
                        getattr(self, k).copy_(b[k], non_blocking=True)
        self.unpack(self.recv_lo, self.recv_hi)


class AmrDecomposition:
    """A block-structured AMR mesh split over ranks along PARAMESH's Morton
    order (PM4_package/source/amr_morton_order.F90, amr_sort_morton.F90): the
    leaf list of an AmrMesh is Morton-ordered, and rank r owns the contiguous
    range [n r / world, n (r + 1) / world) of it.

    Every rank keeps the whole mesh and a full UNK; per step it exchanges
    the interiors of the leaves another rank's step reads, then steps:
      * role 1, its own leaves: guard fill, fluxes, boundary fluxes, flux
        correction, update (levelFlux/Hydro.F90:161-270);
      * role 2, "flux ghosts": the other ranks' leaves one level finer that
        share a face with an own leaf -- their fluxes are computed here too
        (from exchanged data, bit for bit what their owner computes), so that
        Grid_conserveFluxes on the own leaf needs no second exchange in the
        step (the reference's mpi_amr_flux_conserve.F90:87-132 sends them).
    A leaf's guard fill reads leaves within two steps of the "touching"
    relation (sharing a face, edge or corner, across levels and periodic
    boundaries): same-level neighbours, coarser neighbours and their
    neighbours for the prolongation stencil, finer neighbours through the
    restricted parent cells.  With flux ghosts one step away, every rank
    therefore receives the leaves within `hops` = 3 steps of its own."""

    def __init__(self, mesh, world, rank, hops=3):
        self.mesh, self.world, self.rank, self.hops = mesh, world, rank, hops
        n = mesh.nleaf
        if world < 1 or not 0 <= rank < world or n < world:
            raise ValueError("AmrDecomposition: need 1 <= world <= leaves and 0 <= rank < world")
        self.bounds = [n * r // world for r in range(world + 1)]
        self.owner = np.zeros(n, dtype=np.int64)
        for r in range(world):
            self.owner[self.bounds[r]:self.bounds[r + 1]] = r
        self._touch, self._face = self._adjacency(mesh)
        self.ghosts = [self._ghosts_of(r, hops) for r in range(world)]
        self.roles = self.roles_of(rank)

    @staticmethod
    def _adjacency(mesh):
        """Per leaf: the leaves it touches (face, edge or corner) and those it
        shares a face with; boxes in units of the finest cells, periodic axes
        wrapped.  A leaf lies inside its root block, so the leaves it touches
        lie in its own root block or in one touching it: each root block's
        leaves are tested against those of its (up to 3^ndim) neighbours."""
        import itertools
        g = mesh.geom
        nd = g.ndim
        L = int(mesh.maxlev)
        lev = np.asarray(mesh.levels, dtype=np.int64)
        scale = 1 << (L - lev)
        lo = np.asarray(mesh.bcoords, dtype=np.int64)[:, :nd] * scale[:, None]
        hi = lo + scale[:, None]
        nb = [g.nblockx, g.nblocky, g.nblockz][:nd]
        ext = np.array([b << (L - 1) for b in nb], dtype=np.int64)
        per = [g.bc[2 * a] == BC_PERIODIC for a in range(nd)]
        root = lo >> (L - 1)
        buckets = {}
        for i, rc in enumerate(map(tuple, root)):
            buckets.setdefault(rc, []).append(i)
        touch, face = [None] * mesh.nleaf, [None] * mesh.nleaf
        for rc, members in buckets.items():
            near = set()
            for off in itertools.product((-1, 0, 1), repeat=nd):
                c = []
                for a in range(nd):
                    v = rc[a] + off[a]
                    if per[a]:
                        v %= nb[a]
                    elif not 0 <= v < nb[a]:
                        break
                    c.append(v)
                else:
                    near.update(buckets.get(tuple(c), ()))
            A = np.asarray(members, dtype=np.int64)
            C = np.asarray(sorted(near), dtype=np.int64)
            contact = np.ones((len(A), len(C)), dtype=bool)     # closed boxes meet on every axis
            nover = np.zeros((len(A), len(C)), dtype=np.int64)   # axes where open intervals overlap
            for a in range(nd):
                shifts = (-ext[a], 0, ext[a]) if per[a] else (0,)
                cm = np.zeros_like(contact)
                om = np.zeros_like(contact)
                la, ha = lo[A, a][:, None], hi[A, a][:, None]
                for sh in shifts:
                    l2, h2 = lo[C, a][None, :] + sh, hi[C, a][None, :] + sh
                    cm |= (la <= h2) & (l2 <= ha)
                    om |= (la < h2) & (l2 < ha)
                contact &= cm
                nover += om
            contact &= A[:, None] != C[None, :]
            fmask = contact & (nover == nd - 1)
            for q, i in enumerate(A):
                touch[i] = C[contact[q]]
                face[i] = C[fmask[q]]
        return touch, face

    def _ghosts_of(self, r, hops):
        own = set(range(self.bounds[r], self.bounds[r + 1]))
        seen, front = set(own), set(own)
        for _ in range(hops):
            nxt = set()
            for l in front:
                nxt.update(int(x) for x in self._touch[l] if int(x) not in seen)
            seen |= nxt
            front = nxt
        return np.array(sorted(seen - own), dtype=np.int64)

    def flux_ghosts_of(self, r):
        """Other ranks' leaves one level finer sharing a face with a leaf of r."""
        lev = np.asarray(self.mesh.levels)
        out = set()
        for l in range(self.bounds[r], self.bounds[r + 1]):
            for x in self._face[l]:
                x = int(x)
                if self.owner[x] != r and lev[x] == lev[l] + 1:
                    out.add(x)
        return np.array(sorted(out), dtype=np.int64)

    def roles_of(self, r):
        roles = np.zeros(self.mesh.nleaf, dtype=np.uint8)
        roles[self.bounds[r]:self.bounds[r + 1]] = 1
        roles[self.flux_ghosts_of(r)] = 2
        return roles

    def owned(self, r=None):
        r = self.rank if r is None else r
        return np.arange(self.bounds[r], self.bounds[r + 1])

    def sends(self):
        """{peer: own leaves the peer reads}"""
        own = self.owned()
        return {s: np.intersect1d(own, self.ghosts[s]) for s in range(self.world)
                if s != self.rank and len(np.intersect1d(own, self.ghosts[s]))}

    def recvs(self):
        """{peer: leaves of the peer this rank reads}"""
        mine = self.ghosts[self.rank]
        return {s: mine[self.owner[mine] == s] for s in range(self.world)
                if s != self.rank and np.any(self.owner[mine] == s)}


class AmrExchange:
    """The step's one exchange of leaf data between the ranks of an
    AmrDecomposition (PARAMESH's mpi_amr_comm_setup + mpi_xchange_blocks for
    the guard fill, mpi_amr_comm_setup.F90:531): per peer one message with
    the leaves it reads, `leaf_doubles` values each, over
    torch.distributed.batch_isend_irecv (NCCL between GPUs, gloo on CPU).
    pack(leaves, buf) fills a message, unpack(leaves, buf) stores one.
    host_stage: the messages are packed in device memory but cross between
    the ranks through pinned host copies (a process group whose backend
    moves host memory, e.g. gloo between processes that share a GPU)."""

    def __init__(self, dec, leaf_doubles, pack, unpack, device=None, stream=None, host_stage=False):
        self.dec, self.n, self.pack, self.unpack = dec, int(leaf_doubles), pack, unpack
        self.device = device if device is not None else _device()
        self.stream = stream
        self.host_stage = host_stage
        self.sends, self.recvs = dec.sends(), dec.recvs()
        self.sbuf = {s: torch.empty(len(v) * self.n, dtype=torch.float64, device=self.device)
                     for s, v in self.sends.items()}
        self.rbuf = {s: torch.empty(len(v) * self.n, dtype=torch.float64, device=self.device)
                     for s, v in self.recvs.items()}
        if host_stage:
            self.shost = {s: torch.empty(b.numel(), dtype=torch.float64, pin_memory=True) for s, b in self.sbuf.items()}
            self.rhost = {s: torch.empty(b.numel(), dtype=torch.float64, pin_memory=True) for s, b in self.rbuf.items()}

    def __call__(self):
        if self.dec.world == 1:
            return
        ctx = torch.cuda.stream(self.stream) if self.stream is not None else _nullctx()
        with ctx:
            for s, leaves in self.sends.items():
                self.pack(leaves, self.sbuf[s])
            tx, rx = self.sbuf, self.rbuf
            if self.host_stage:
                for s in self.sends:
                    self.shost[s].copy_(self.sbuf[s], non_blocking=True)
                torch.cuda.current_stream().synchronize()
                tx, rx = self.shost, self.rhost
            ops = [dist.P2POp(dist.isend, tx[s], s) for s in sorted(self.sends)]
            ops += [dist.P2POp(dist.irecv, rx[s], s) for s in sorted(self.recvs)]
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            if self.host_stage:
                for s in self.recvs:
                    self.rbuf[s].copy_(self.rhost[s], non_blocking=True)
            for s, leaves in self.recvs.items():
                self.unpack(leaves, self.rbuf[s])


class _nullctx:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False
