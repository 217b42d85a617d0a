"""Multi-process driver logic: one process per GPU.

Flash-X advances every rank with one global time step: Driver_computeDt
reduces the per-rank CFL minimum with MPI_AllReduce(MIN)
(Driver/DriverMain/Driver_computeDt.F90:373,383) before the growth limit and
clamp, and IO_writeIntegralQuantities sums the conserved integrals with
MPI_Reduce(SUM) (IO/IOMain/IO_writeIntegralQuantities.F90:224).  Here those two
reductions run over torch.distributed (NCCL between GPUs, gloo on CPU).

`ReplicaDriver` advances one independent problem per rank (weak scaling) with
that common dt.  A decomposition of one domain across GPUs additionally needs
the guard-cell exchange between ranks, which this module does not provide.
"""
import datetime
import os

import torch
import torch.distributed as dist

from .hydro import driver_dt, initial_dt


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
    """Driver_evolveAll for one problem per rank with a common dt.

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
