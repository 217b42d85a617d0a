"""CPU tests of the drop-in boundary: the C-ABI library loads and exports
every entry point include/flashx_b200.h declares, argument validation and
status codes behave like the reference's aborts, and the host-side mirror
builds the right block list and variable map.  No compute call runs here."""
import ctypes
import os
import re

import numpy as np
import pytest

from flashx_b200 import hydro as H
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, Geometry, HydroParams, UNK_VARS)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "flashx_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|long|void)\s*\*?\s*(fxb_\w+)\s*\(", src, re.M)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    assert set(H.ABI_SYMBOLS) == set(syms)


def test_library_exports_every_declared_symbol():
    lib = H.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def _init(hp=None, geom=None, vm=None, nunk=11, precision="fp64"):
    lib = H.load_library()
    hp = hp or HydroParams()
    geom = geom or Geometry(2, 16, 16, 1, 2, 2, 1)
    p = H.make_fxb_params(hp, precision)
    d = H.make_fxb_domain(geom)
    vm = vm if vm is not None else H.default_var_map()
    return lib.fxb_init(ctypes.byref(p), ctypes.byref(d), vm, nunk), p, d


def test_init_validation_codes():
    lib = H.load_library()
    rc, p, d = _init()
    # on a CPU-only host the device query fails last, after every argument check
    assert rc in (H.FXB_OK, H.FXB_ECUDA)
    # bad dimensionality, guard count, order, solver, var_map
    d.ndim = 1
    assert lib.fxb_init(ctypes.byref(p), ctypes.byref(d), H.default_var_map(), 11) == H.FXB_EUNSUPPORTED
    d.ndim = 2; d.nguard = 2
    assert lib.fxb_init(ctypes.byref(p), ctypes.byref(d), H.default_var_map(), 11) == H.FXB_EARG
    d.nguard = 4; p.order = 4
    assert lib.fxb_init(ctypes.byref(p), ctypes.byref(d), H.default_var_map(), 11) == H.FXB_EUNSUPPORTED
    p.order = 3
    for bad in (6, 9):      # HLLD is MHD-only; no solver 9
        p.riemann = bad
        assert lib.fxb_init(ctypes.byref(p), ctypes.byref(d), H.default_var_map(), 11) == H.FXB_EUNSUPPORTED
    p.riemann = 4
    vm = H.default_var_map(); vm[0] = 11
    assert lib.fxb_init(ctypes.byref(p), ctypes.byref(d), vm, 11) == H.FXB_EARG
    d.bc[0] = BC_PERIODIC; d.bc[1] = BC_OUTFLOW
    assert lib.fxb_init(ctypes.byref(p), ctypes.byref(d), H.default_var_map(), 11) == H.FXB_EARG
    err = H.FxbError()
    assert lib.fxb_last_error(ctypes.byref(err)) == H.FXB_EARG
    assert b"periodic" in err.message


def test_slab_validation_codes():
    """fxb_init_slab: a side facing another slab needs a halo of NGUARD to the
    slab's own planes, a non-periodic domain edge none, 2-D slabs fill 16-cell
    tiles (argument checks come before the device query)."""
    lib = H.load_library()
    p = H.make_fxb_params(HydroParams())
    geom = Geometry(2, 16, 16, 1, 2, 4, 1, bc=(BC_OUTFLOW,) * 6)
    d = H.make_fxb_domain(geom)
    vm = H.default_var_map()
    init = lambda *s: lib.fxb_init_slab(ctypes.byref(p), ctypes.byref(d), vm, 11, ctypes.byref(H.FxbSlab(*s)))
    assert init(0, 2, 0, 16) in (H.FXB_OK, H.FXB_ECUDA)
    assert init(1, 3, 8, 8) in (H.FXB_OK, H.FXB_ECUDA)
    assert init(2, 4, 16, 0) in (H.FXB_OK, H.FXB_ECUDA)
    assert init(0, 5, 0, 0) == H.FXB_EARG          # layers outside the grid
    assert init(2, 2, 8, 8) == H.FXB_EARG          # empty
    assert init(0, 2, 0, 0) == H.FXB_EARG          # no halo towards the next slab
    assert init(0, 2, 0, 2) == H.FXB_EARG          # halo thinner than NGUARD
    assert init(0, 2, 0, 40) == H.FXB_EARG         # halo wider than the slab
    assert init(0, 2, 8, 16) == H.FXB_EARG         # halo on an outflow boundary
    assert init(0, 2, 0, 4) == H.FXB_EUNSUPPORTED  # 32 + 4 rows do not fill 16-row tiles
    # use_upwindTVD: reset with NGUARD = 4 (Hydro_init.F90:137), refused with more guard cells
    p.upwind_tvd = 1
    assert init(0, 2, 0, 16) in (H.FXB_OK, H.FXB_ECUDA)
    d.nguard = 6
    assert init(0, 2, 0, 16) == H.FXB_EUNSUPPORTED
    d.nguard = 4
    p.upwind_tvd = 0
    d.bc[2] = d.bc[3] = BC_PERIODIC
    assert init(0, 4, 8, 8) in (H.FXB_OK, H.FXB_ECUDA)   # one slab exchanging with itself
    sub = H.leaf_blocks(geom, (1, 3))
    assert [tuple(b.bcoord) for b in sub] == [(0, 1, 0), (1, 1, 0), (0, 2, 0), (1, 2, 0)]
    lib.fxb_finalize()


def test_gravity_validation_2d_and_3d():
    """Constant gravity passes the argument checks on 2-D and 3-D grids; only
    its combination with flattening is refused (FXB_EUNSUPPORTED)."""
    lib = H.load_library()
    for geom, g in ((Geometry(2, 16, 16, 1, 2, 2, 1), (0.0, -0.1, 0.0)),
                    (Geometry(3, 16, 16, 16, 1, 1, 2), (0.0, 0.0, -0.1))):
        rc, p, d = _init(HydroParams(useGravity=True, gravity=g), geom)
        assert rc in (H.FXB_OK, H.FXB_ECUDA)
        p.flattening = 1
        assert lib.fxb_init(ctypes.byref(p), ctypes.byref(d), H.default_var_map(), 11) == H.FXB_EUNSUPPORTED
        err = H.FxbError()
        lib.fxb_last_error(ctypes.byref(err))
        assert b"gravity" in err.message
    lib.fxb_finalize()


def test_calls_before_init_are_rejected():
    lib = H.load_library()
    lib.fxb_finalize()
    out = ctypes.c_double()
    assert lib.fxb_compute_dt(ctypes.byref(out), None) == H.FXB_EARG
    assert lib.fxb_hydro_step(0.0, 1e-3, 1e-3) == H.FXB_EARG
    assert lib.fxb_eos() == H.FXB_EARG
    buf = (ctypes.c_double * 16)()
    for f in (lib.fxb_put_interior, lib.fxb_get_interior):
        assert f(None) == H.FXB_EARG
        assert f(buf) == H.FXB_EARG                  # nothing attached


def test_parameter_validation_mirrors_hydro_init():
    HydroParams().validate()
    HydroParams(use_flattening=True).validate()
    HydroParams(RiemannSolver="LLF").validate()
    HydroParams(RiemannSolver="Roe").validate()
    HydroParams(RiemannSolver="Roe", entropy=True, entropyFixMethod="Harten").validate()
    HydroParams(use_steepening=True).validate()
    HydroParams(order=2).validate()
    HydroParams(use_upwindTVD=True, use_avisc=True).validate()
    HydroParams(RiemannSolver="Marquina").validate()
    HydroParams(RiemannSolver="MarquinaModified").validate()
    HydroParams(RiemannSolver="hybrid").validate()
    HydroParams(shockDetect=True).validate()
    for bad in (dict(order=4), dict(order=6), dict(RiemannSolver="HLLD"), dict(shockLowerCFL=True), dict(entropyFixMethod="Einfeldt"),
                dict(slopeLimiter="superbee"),
                dict(transOrder=3),
                dict(use_flattening=True, useGravity=True),
                dict(hydroComputeDtOption=0)):
        with pytest.raises(ValueError):
            HydroParams(**bad).validate()


def test_var_map_and_block_list():
    vm = H.default_var_map()
    assert [UNK_VARS[vm[i]] for i in range(len(H.FXB_VARS))] == list(H.FXB_VARS)
    geom = Geometry(3, 16, 16, 16, 3, 2, 2)
    blocks = H.leaf_blocks(geom)
    coords = [tuple(b.bcoord) for b in blocks]
    assert len(coords) == 12 and len(set(coords)) == 12
    # Flash-X block order: x fastest
    assert coords[:4] == [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0)]


def test_unk_layout_round_trip():
    from flashx_b200 import simulations as S
    geom = Geometry(2, 16, 16, 1, 3, 2, 1)
    rng = np.random.default_rng(0)
    g = rng.random((1, 32, 48, 11))
    unk = S.scatter_global(geom, g)
    assert unk.shape == (6, 1, 24, 24, 11)
    assert np.array_equal(S.gather_global(geom, unk), g)
    # block 1 is bx=1, by=0: its first interior cell is global (x=16, y=0)
    assert np.array_equal(unk[1, 0, 4, 4], g[0, 0, 16])
