"""CPU tests of the multi-process driver logic (world_size 2, gloo):
the common dt (Driver_computeDt's MPI_AllReduce MIN), summed integrals, the
replica driver taking identical dt sequences on every rank, and a rank that
fails mid-run being noticed by the other rank instead of hanging it."""
import os
import socket
import tempfile

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class FakeDevice:
    """Stands in for HydroDevice: a CFL rate that differs per rank and
    evolves with the steps taken."""

    def __init__(self, rank):
        self.rank = rank
        self.calls = []
        self.rate = 10.0 * (rank + 1)

    def Hydro(self, t, dt, dt_old):
        self.calls.append((t, dt, dt_old))
        self.rate *= 1.01 + 0.02 * self.rank

    def Hydro_computeDt(self):
        return 0.8 / self.rate


def _worker(rank, world, port, outdir, mode):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "flash-x_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from flashx_b200 import parallel as P
    from flashx_b200.params import HydroParams
    result = "ok"
    try:
        P.init_from_env("gloo", timeout_s=20)
        if mode == "reduce":
            assert P.allreduce_min(1.0 + rank) == 1.0
            assert P.allreduce_max(1.0 + rank) == 2.0
            assert P.allreduce_sum([1.0, rank]) == [2.0, 1.0]
            dev = FakeDevice(rank)
            drv = P.ReplicaDriver(dev, HydroParams(dtinit=1e-3))
            dt = drv.first_dt()
            dt, dt_old = drv.run(25, dt, dt)
            with open(os.path.join(outdir, f"calls{rank}.txt"), "w") as f:
                f.write(repr(dev.calls))
        else:   # rank 1 aborts before the step's collective, as Driver_abort would
            dev = FakeDevice(rank)
            drv = P.ReplicaDriver(dev, HydroParams())
            dt = drv.first_dt()
            if rank == 1:
                raise RuntimeError("injected failure on rank 1")
            drv.run(5, dt, dt)
            result = "rank 0 finished although rank 1 failed"
    except Exception as e:  # noqa: BLE001
        result = f"error: {type(e).__name__}: {e}"
    with open(os.path.join(outdir, f"result{rank}.txt"), "w") as f:
        f.write(result)
    try:
        import torch.distributed as dist
        if dist.is_initialized() and result == "ok":
            dist.destroy_process_group()
    except Exception:
        pass


def _run(mode):
    out = tempfile.mkdtemp()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out, mode)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
            pytest.fail("worker did not finish")
    return out, [open(os.path.join(out, f"result{r}.txt")).read() for r in range(2)]


def test_common_dt_and_replica_driver_gloo():
    out, res = _run("reduce")
    assert res == ["ok", "ok"], res
    c0 = eval(open(os.path.join(out, "calls0.txt")).read())
    c1 = eval(open(os.path.join(out, "calls1.txt")).read())
    assert len(c0) == 25
    # both ranks advanced with exactly the same (t, dt, dtOld) sequence
    assert c0 == c1
    # dt grew by at most the tstep_change_factor of 2 per step
    assert all(b[1] <= 2.0 * a[1] + 1e-30 for a, b in zip(c0, c0[1:]))


def test_failed_rank_is_detected_not_hung():
    _, res = _run("fail")
    assert res[1].startswith("error: RuntimeError: injected failure")
    assert res[0].startswith("error:"), res[0]
