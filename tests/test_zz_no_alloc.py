"""GPU test of fxb_integrals_noalloc, the entry point for callers that cannot
allocate device memory (their GPU memory belongs to another runtime's pool,
or every byte they place on the GPU is accounted for).

It takes caller-owned device arrays and keeps its scratch in a fixed static
device array of the library, so it performs no cudaMalloc of its own.  The
test hands it device arrays of the same state the library's own mirror
holds and checks its sums against the existing fxb_integrals entry point, on
two calls in a row (the second call reuses the scratch the first one left
behind).  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from flashx_b200 import simulations as S
from flashx_b200.hydro import FXB_EARG, FXB_OK, FxbError, HydroDevice, load_library
from flashx_b200.params import DENS, EINT, ENER, VELX, VELY, VELZ

pytestmark = pytest.mark.gpu

RTOL = 1e-12   # different summation order than fxb_integrals: roundoff only


def test_integrals_without_allocation_match_fxb_integrals(need_gpu):
    import torch
    geom, hp, init = S.config("kh2d", scale=1 / 16)       # 128^2 periodic
    unk = init(geom, hp)
    dev = HydroDevice(geom, hp, "fp64")
    dev.attach_unk(unk.copy())
    dt = 0.5 * dev.Hydro_computeDt()
    dev.advance(3, dt, dt)                                 # a state that is not the initial one
    ref = dev.integrals()
    state = np.zeros(geom.unk_shape)
    dev.sync_to_host(state)
    g = S.gather_global(geom, state)[0]                     # (ny, nx, var)
    # caller-owned device arrays (the caller allocates them; the entry point does not)
    cols = {v: torch.tensor(np.ascontiguousarray(g[..., v]).ravel(), dtype=torch.float64, device="cuda")
            for v in (DENS, VELX, VELY, VELZ, ENER, EINT)}
    out = torch.full((7,), float("nan"), dtype=torch.float64, device="cuda")
    dx, dy, dz = geom.deltas()
    lib = load_library()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    for call in range(2):
        out.fill_(float("nan"))
        rc = lib.fxb_integrals_noalloc(ptr(cols[DENS]), ptr(cols[VELX]), ptr(cols[VELY]), ptr(cols[VELZ]),
                                       ptr(cols[ENER]), ptr(cols[EINT]), geom.ncells, dx * dy * dz,
                                       ptr(out), None)
        assert rc == FXB_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.allclose(got, ref, rtol=RTOL, atol=1e-14 * abs(ref[0])), (call, got, ref)
    # a size that is not a whole number of 4096-cell chunks (the last CTA sums
    # a partial chunk), on a non-default stream, against float64 NumPy sums
    n = geom.ncells - 1000
    dv = dx * dy * dz
    c = {v: np.ascontiguousarray(g[..., v]).ravel()[:n] for v in (DENS, VELX, VELY, VELZ, ENER, EINT)}
    rho, vx, vy, vz = c[DENS], c[VELX], c[VELY], c[VELZ]
    expect = np.array([np.sum(rho * dv), np.sum(rho * vx * dv), np.sum(rho * vy * dv), np.sum(rho * vz * dv),
                       np.sum(rho * c[ENER] * dv), np.sum(rho * c[EINT] * dv),
                       np.sum(0.5 * rho * (vx * vx + vy * vy + vz * vz) * dv)])
    side = torch.cuda.Stream()
    for call in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = lib.fxb_integrals_noalloc(ptr(cols[DENS]), ptr(cols[VELX]), ptr(cols[VELY]), ptr(cols[VELZ]),
                                       ptr(cols[ENER]), ptr(cols[EINT]), n, dv, ptr(out),
                                       ctypes.c_void_p(side.cuda_stream))
        assert rc == FXB_OK
        side.synchronize()
        got = out.cpu().numpy()
        assert np.allclose(got, expect, rtol=RTOL, atol=1e-14 * abs(expect[0])), (call, got, expect)
    # sizes beyond the static scratch are rejected with a clear error, before any launch
    rc = lib.fxb_integrals_noalloc(ptr(cols[DENS]), ptr(cols[VELX]), ptr(cols[VELY]), ptr(cols[VELZ]),
                                   ptr(cols[ENER]), ptr(cols[EINT]), 8192 * 4096 + 1, 1.0, ptr(out), None)
    assert rc == FXB_EARG
    err = FxbError()
    lib.fxb_last_error(ctypes.byref(err))
    assert b"static scratch capacity" in err.message
    dev.close()
