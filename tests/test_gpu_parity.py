"""GPU parity tests: the CUDA path (through the C ABI of libflashx_b200.so)
against the CPU oracle on the same seeded inputs.

Tolerances: the plain FP64 path must match to <= 1e-12 relative per zone
after one step and <= 1e-10 in L1 density after 100 steps; it is built
with -fmad=false and is expected to be bit-identical, which is asserted
separately.  The mixed path (FP32 reconstruction/Riemann, FP64 update) must
stay within 1e-5 L1 density of the FP64 path.
"""
import numpy as np
import pytest

from flashx_b200 import simulations as S
from flashx_b200.hydro import FlashXError, HydroDevice, driver_dt
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, DENS, EINT, ENER, GAMC, GAME,
                                Geometry, HydroParams, PRES, TEMP, VELX, VELY, VELZ, NUNK)

pytestmark = pytest.mark.gpu

HYDRO_VARS = [DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ]
REL_TOL_ONE_STEP = 1e-12     # per zone, after one step
L1_TOL_100 = 1e-10           # L1 density after 100 steps (relative to mean density)
L1_TOL_MIXED = 1e-5          # mixed vs FP64, L1 density (relative)


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def gpu_run(geom, hp, unk, dts, precision="fp64"):
    dev = HydroDevice(geom, hp, precision)
    dev.attach_unk(unk.copy())
    t = 0.0
    for i, dt in enumerate(dts):
        dev.Hydro(t + dt, dt, dts[i - 1] if i else dt)
        t += dt
    out = np.zeros(geom.unk_shape)
    dev.sync_to_host(out)
    return dev, out


def oracle_run(O, geom, hp, unk, dts):
    p = O.make_params(geom.as_dict(), hp)
    u = unk.copy()
    for i, dt in enumerate(dts):
        O.hydro_step(p, u, dt, dts[i - 1] if i else dt)
    return u


def oracle_dts(O, geom, hp, unk, n, first=None):
    """dt sequence the reference driver would take (Driver_computeDt growth limit)."""
    p = O.make_params(geom.as_dict(), hp)
    u = unk.copy()
    dt = first if first is not None else 0.5 * O.compute_dt(p, u)
    dts = []
    for i in range(n):
        dts.append(dt)
        O.hydro_step(p, u, dt, dts[i - 1] if i else dt)
        dt = O.driver_dt(O.compute_dt(p, u), dt)
    return dts, u


def compare(geom, a, b):
    ga, gb = S.gather_global(geom, a), S.gather_global(geom, b)
    return ga[..., HYDRO_VARS], gb[..., HYDRO_VARS]


def test_sod_one_step_fp64_matches_oracle(oracle, need_gpu):
    geom, hp, init = S.config("sod2d", scale=0.25)        # 64^2, outflow
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dt = 0.8 * oracle.compute_dt(p, unk)                  # a full CFL step, not dtinit
    ref = oracle_run(oracle, geom, hp, unk, [dt])
    _, out = gpu_run(geom, hp, unk, [dt])
    g, r = compare(geom, out, ref)
    assert np.max(_rel(g, r)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r), "FP64 path is expected to be bit-identical to the oracle"


@pytest.mark.parametrize("name", ["sod2d", "kh2d"])
def test_100_steps_fp64_l1(oracle, need_gpu, name):
    geom, hp, init = S.config(name, scale=0.25 if name == "sod2d" else 1 / 32)
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dts, ref = oracle_dts(oracle, geom, hp, unk, 100, first=0.5 * oracle.compute_dt(p, unk))
    _, out = gpu_run(geom, hp, unk, dts)
    g, r = compare(geom, out, ref)
    l1 = np.mean(np.abs(g[..., 0] - r[..., 0])) / np.mean(np.abs(r[..., 0]))
    assert l1 <= L1_TOL_100
    assert np.array_equal(g, r)


@pytest.mark.parametrize("opts", [
    dict(order=5), dict(order=5, wenoMethod="WENOZ"), dict(RiemannSolver="HLL"), dict(RiemannSolver="LLF"),
    dict(RiemannSolver="Roe"),
    dict(slopeLimiter="minmod"), dict(slopeLimiter="vanLeer"), dict(slopeLimiter="hybrid"),
    dict(slopeLimiter="limited", LimitedSlopeBeta=1.5), dict(charLimiting=False),
    dict(charLimiting=False, slopeLimiter="hybrid"), dict(use_auxEintEqn=False), dict(hy_fPresInMomFlux=0.5),
    dict(order=2), dict(order=2, RiemannSolver="Roe"), dict(order=2, charLimiting=False, slopeLimiter="hybrid"),
    dict(order=2, slopeLimiter="limited", LimitedSlopeBeta=1.5), dict(order=2, RiemannSolver="HLL",
                                                                      use_auxEintEqn=False),
    dict(use_avisc=True), dict(use_avisc=True, cvisc=0.3, order=2), dict(use_avisc=True, use_auxEintEqn=False),
])
def test_options_one_step_fp64(oracle, need_gpu, opts):
    geom = Geometry(2, 16, 16, 1, 3, 2, 1, bc=(BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_OUTFLOW, 1, 1))
    hp = HydroParams(**opts)
    unk = S.kelvin_helmholtz(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dts, ref = oracle_dts(oracle, geom, hp, unk, 3, first=0.5 * oracle.compute_dt(p, unk))
    _, out = gpu_run(geom, hp, unk, dts)
    g, r = compare(geom, out, ref)
    assert np.max(_rel(g, r)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r)


@pytest.mark.parametrize("flattening", [False, True])
def test_steepening_2d_fp64(oracle, need_gpu, flattening):
    """use_steepening (PPM contact steepening) on the 45-degree Sod problem,
    whose contact switches it on; with and without flattening."""
    geom, _, init = S.config("sod2d", scale=0.25)
    hp = HydroParams(use_steepening=True, use_flattening=flattening)
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dts, ref = oracle_dts(oracle, geom, hp, unk, 20, first=0.5 * oracle.compute_dt(p, unk))
    _, out = gpu_run(geom, hp, unk, dts)
    g, r = compare(geom, out, ref)
    assert np.array_equal(g, r)
    hp0 = HydroParams(use_flattening=flattening)
    _, ref0 = oracle_dts(oracle, geom, hp0, unk, 20, first=dts[0])
    assert not np.array_equal(ref, ref0)   # the steepening acted


@pytest.mark.parametrize("order", [2, 3, 5])
def test_flattening_2d_fp64(oracle, need_gpu, order):
    """use_flattening on the 45-degree Sod problem, where the shock switches it on."""
    geom, _, init = S.config("sod2d", scale=0.25)
    hp = HydroParams(order=order, use_flattening=True)
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dts, ref = oracle_dts(oracle, geom, hp, unk, 5, first=0.5 * oracle.compute_dt(p, unk))
    _, out = gpu_run(geom, hp, unk, dts)
    g, r = compare(geom, out, ref)
    assert np.max(_rel(g, r)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r)


@pytest.mark.parametrize("bc", [BC_OUTFLOW, BC_REFLECTING, BC_PERIODIC])
def test_fill_guardcells_matches_oracle(oracle, need_gpu, bc):
    geom = Geometry(2, 16, 16, 1, 2, 3, 1, bc=(bc,) * 6)
    hp = HydroParams()
    unk = S.kelvin_helmholtz(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    ref = unk.copy()
    oracle.fill_guardcells(p, ref)
    dev = HydroDevice(geom, hp)
    dev.attach_unk(unk.copy())
    out = np.zeros(geom.unk_shape)
    dev.Grid_fillGuardCells(out)
    assert np.array_equal(out[..., HYDRO_VARS], ref[..., HYDRO_VARS])


@pytest.mark.parametrize("bc", [BC_OUTFLOW, BC_REFLECTING, BC_PERIODIC])
def test_masked_fill_guardcells(oracle, need_gpu, bc):
    """Grid_fillGuardCells with a mask: only the selected variables cross
    PCIe and are written (equal to the oracle's fill); every other UNK entry
    keeps its host value."""
    from flashx_b200.hydro import COUNT_GC_DOUBLES, COUNT_GC_FILLS
    geom = Geometry(2, 16, 16, 1, 2, 3, 1, bc=(bc,) * 6)
    hp = HydroParams()
    unk = S.kelvin_helmholtz(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    ref = unk.copy()
    oracle.fill_guardcells(p, ref)
    dev = HydroDevice(geom, hp)
    dev.attach_unk(unk.copy())
    c0 = dev.counters()
    out = np.full(geom.unk_shape, -7.0)
    dev.Grid_fillGuardCells(out, mask=["dens", "pres", "velx"])
    c1 = dev.counters()
    sel = [DENS, PRES, VELX]
    rest = [v for v in range(NUNK) if v not in sel]
    assert np.array_equal(out[..., sel], ref[..., sel])
    assert np.all(out[..., rest] == -7.0)
    ncell = out.size // NUNK
    assert c1[COUNT_GC_FILLS] - c0[COUNT_GC_FILLS] == 1
    assert c1[COUNT_GC_DOUBLES] - c0[COUNT_GC_DOUBLES] == 3 * ncell
    # no mask: every hydro variable, as before
    out2 = np.full(geom.unk_shape, -7.0)
    dev.Grid_fillGuardCells(out2, doEos=False)
    assert np.array_equal(out2[..., HYDRO_VARS], ref[..., HYDRO_VARS])
    with pytest.raises(ValueError):
        dev.Grid_fillGuardCells(out2, mask=["shok"])
    dev.close()


@pytest.mark.parametrize("name", ["kh2d", "sweep3d"])
def test_compute_dt_once_per_step(oracle, need_gpu, name):
    """Driver_computeDt calls Hydro_computeDt once per leaf block
    (Driver_computeDt.F90:306): the first call after a state change reduces
    on the device, every later call returns the cached global dt (and
    dtMinLoc) without a launch or a host synchronisation."""
    from flashx_b200.hydro import COUNT_DT_CACHED, COUNT_DT_DEVICE
    geom, hp, init = S.config(name, scale=0.25 if name == "kh2d" else 0.5)
    unk = init(geom, hp)
    dev = HydroDevice(geom, hp, "fp64")
    dev.attach_unk(unk.copy())
    p = oracle.make_params(geom.as_dict(), hp)
    for step in range(3):
        c0 = dev.counters()
        dtcheck, loc = 1e30, None
        for _ in range(geom.nblocks):                        # Driver_computeDt's block loop
            dt_b, loc_b = dev.Hydro_computeDt(location=True)
            if dt_b < dtcheck:
                dtcheck, loc = dt_b, loc_b
        c1 = dev.counters()
        assert c1[COUNT_DT_DEVICE] - c0[COUNT_DT_DEVICE] == 1
        assert c1[COUNT_DT_CACHED] - c0[COUNT_DT_CACHED] == geom.nblocks - 1
        host = np.zeros(geom.unk_shape)
        dev.sync_to_host(host)
        assert dtcheck == oracle.compute_dt(p, host)
        assert loc == _expected_loc(geom, host)
        dev.Hydro(0.0, 0.5 * dtcheck, 0.5 * dtcheck)
    dev.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tma_window_equals_thread_loads(need_gpu, monkeypatch, precision):
    """The 2-D kernel stages interior windows by TMA and edge windows with
    per-thread loads; staging every window with per-thread loads (FXB_TMA=0)
    gives the same state bit for bit."""
    geom, hp, init = S.config("kh2d", scale=1 / 8)          # 256^2: 196 of 256 tiles interior
    unk = init(geom, hp)
    outs = []
    for flag in ("1", "0"):
        monkeypatch.setenv("FXB_TMA", flag)
        dev = HydroDevice(geom, hp, precision)
        dev.attach_unk(unk.copy())
        dt = 0.5 * dev.Hydro_computeDt()
        dev.advance(6, dt, dt)
        out = np.zeros(geom.unk_shape)
        dev.sync_to_host(out)
        dev.close()
        outs.append(out)
    assert np.array_equal(outs[0][..., HYDRO_VARS], outs[1][..., HYDRO_VARS])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("config", ["rt3d", "sweep3d"])
def test_ug_launch_shapes_give_identical_states(need_gpu, monkeypatch, precision, config):
    """The uniform-grid tuner only changes launch shapes: the defaults
    (FXB_UG_TUNE=0), the tuned shapes and forced odd ones (CTAs per SM per
    stage, lines per fused face-state tile) step to the same state bit for
    bit, and fxb_tuning reports the shapes in use."""
    geom, hp, init = S.config(config, scale=0.25 if config == "rt3d" else 0.5)
    unk = init(geom, hp)
    outs = []
    for env in ({"FXB_UG_TUNE": "0"}, {}, {"FXB_UG_CTA": "2,16,4,1", "FXB_UG_T1": "1,16,2"}):
        for k in ("FXB_UG_TUNE", "FXB_UG_CTA", "FXB_UG_T1"):
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        dev = HydroDevice(geom, hp, precision)
        dev.attach_unk(unk.copy())
        log = dev.tuning()
        assert log.startswith("uniform grid 3-D")
        if "FXB_UG_CTA" in env:
            assert "sigma 2, face states 16, fluxes 4, update 1" in log
            if precision == "mixed":
                assert "x/y/z: 1/16/2" in log
        dt = 0.5 * dev.Hydro_computeDt()
        dev.advance(4, dt, dt)
        out = np.zeros(geom.unk_shape)
        dev.sync_to_host(out)
        dev.close()
        outs.append(out)
    assert np.array_equal(outs[0][..., HYDRO_VARS], outs[1][..., HYDRO_VARS])
    assert np.array_equal(outs[0][..., HYDRO_VARS], outs[2][..., HYDRO_VARS])


def test_window_wait_timeout_reports_status(oracle, need_gpu, monkeypatch):
    """A window barrier that never completes (test hook: it expects 8 bytes
    more than the TMA box brings) ends each waiting tile after its bounded
    wait with ERR_TIMEOUT; the host reads FXB_ETIMEOUT, and the context stays
    usable: the next solver instance steps exactly like the oracle."""
    from flashx_b200.hydro import FXB_ETIMEOUT
    geom = Geometry(2, 16, 16, 1, 3, 3, 1, bc=(BC_PERIODIC,) * 6)   # one interior (TMA) tile
    hp = HydroParams()
    unk = S.kelvin_helmholtz(geom, hp)
    monkeypatch.setenv("FXB_TEST_WAIT_TIMEOUT", "1")
    dev = HydroDevice(geom, hp)
    dev.attach_unk(unk.copy())
    dt = 0.5 * dev.Hydro_computeDt()
    dev.Hydro(0.0, dt, dt)
    with pytest.raises(FlashXError) as ei:
        dev.Hydro_computeDt()
    assert ei.value.code == FXB_ETIMEOUT
    dev.close()
    monkeypatch.delenv("FXB_TEST_WAIT_TIMEOUT")
    p = oracle.make_params(geom.as_dict(), hp)
    ref = oracle_run(oracle, geom, hp, unk, [dt])
    _, out = gpu_run(geom, hp, unk, [dt])
    g, r = compare(geom, out, ref)
    assert np.array_equal(g, r)


def test_compute_dt_and_device_driver_loop(oracle, need_gpu):
    """Hydro_computeDt equals the oracle's; the graph-captured device driver
    loop (fxb_advance) reproduces the host-driven loop exactly."""
    geom, hp, init = S.config("kh2d", scale=1 / 32)
    unk = init(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dev = HydroDevice(geom, hp)
    dev.attach_unk(unk.copy())
    assert dev.Hydro_computeDt() == oracle.compute_dt(p, unk)
    dt = dt_old = 0.5 * dev.Hydro_computeDt()
    for _ in range(7):
        dev.Hydro(0.0, dt, dt_old)
        dt_old = dt
        dt = driver_dt(dev.Hydro_computeDt(), dt_old, hp)
    host = np.zeros(geom.unk_shape)
    dev.sync_to_host(host)
    dev2 = HydroDevice(geom, hp)
    dev2.attach_unk(unk.copy())
    d0 = 0.5 * dev2.Hydro_computeDt()
    dtn, dto = dev2.advance(7, d0, d0)
    dev2_out = np.zeros(geom.unk_shape)
    dev2.sync_to_host(dev2_out)
    assert (dtn, dto) == (dt, dt_old)
    assert np.array_equal(host[..., HYDRO_VARS], dev2_out[..., HYDRO_VARS])


def test_conservation_on_device(need_gpu):
    geom, hp, init = S.config("kh2d", scale=1 / 8)        # 256^2 periodic
    unk = init(geom, hp)
    dev = HydroDevice(geom, hp)
    dev.attach_unk(unk)
    I0 = dev.integrals()
    dt = 0.5 * dev.Hydro_computeDt()
    dev.advance(40, dt, dt)
    I1 = dev.integrals()
    assert abs(I1[0] - I0[0]) / I0[0] < 1e-13
    assert abs(I1[4] - I0[4]) / I0[4] < 1e-13


def test_mixed_precision_l1_vs_fp64(need_gpu):
    geom, hp, init = S.config("kh2d", scale=1 / 16)       # 128^2
    unk = init(geom, hp)
    outs = {}
    for prec in ("fp64", "mixed"):
        dev = HydroDevice(geom, hp, prec)
        dev.attach_unk(unk.copy())
        dt = 0.5 * dev.Hydro_computeDt() if prec == "fp64" else dts0
        if prec == "fp64":
            dts0 = dt
        dev.advance(50, dt, dt)
        o = np.zeros(geom.unk_shape)
        dev.sync_to_host(o)
        outs[prec] = S.gather_global(geom, o)
    a, b = outs["mixed"], outs["fp64"]
    l1 = np.mean(np.abs(a[..., DENS] - b[..., DENS])) / np.mean(b[..., DENS])
    assert l1 <= L1_TOL_MIXED


@pytest.mark.parametrize("opts", [dict(), dict(order=5), dict(order=2), dict(RiemannSolver="HLL")])
def test_gravity_2d_fp64(oracle, need_gpu, opts):
    """Constant gravity on a 2-D grid (the face-state half step of
    hy_getRiemannState.F90:843-885, the update's old-state half step of
    hy_unsplitUpdate.F90:1234-1245 and hy_gravityStepBlk's new-state half
    step): a Rayleigh-Taylor interface with gravity along both axes, three
    steps, bit-identical to the oracle; the mixed path within the L1 bound."""
    geom = Geometry(2, 16, 16, 1, 3, 2, 1, bc=(BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING, 1, 1))
    hp = HydroParams(useGravity=True, gravity=(0.02, -0.1, 0.0), **opts)
    unk = S.rayleigh_taylor(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dts, ref = oracle_dts(oracle, geom, hp, unk, 3, first=0.5 * oracle.compute_dt(p, unk))
    dev, out = gpu_run(geom, hp, unk, dts)
    dev.close()
    g, r = compare(geom, out, ref)
    assert np.max(_rel(g, r)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r)
    dev, mixed = gpu_run(geom, hp, unk, dts, "mixed")
    dev.close()
    a, b = S.gather_global(geom, mixed), S.gather_global(geom, out)
    assert np.mean(np.abs(a[..., DENS] - b[..., DENS])) / np.mean(b[..., DENS]) <= L1_TOL_MIXED


def test_negative_pressure_reports_status(need_gpu):
    """A state with negative pressure makes the eigen-system fail; the library
    returns FXB_ESOUND from the next synchronising call (no GPU fault)."""
    geom = Geometry(2, 16, 16, 1, 1, 1, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams()
    unk = S.kelvin_helmholtz(geom, hp)
    unk[0, 0, 10, 10, PRES] = -1.0
    unk[0, 0, 10, 10, GAMC] = 1.4
    dev = HydroDevice(geom, hp)
    dev.attach_unk(unk)
    dev.Hydro(0.0, 1e-4, 1e-4)
    with pytest.raises(FlashXError) as e:
        dev.Hydro_computeDt()
    assert e.value.code == 3


# ---------------------------------------------------------------- 3-D
@pytest.mark.parametrize("case", ["ppm_periodic", "sod_outflow", "rt_weno_gravity", "hll_noctu", "wenoz_reflect",
                                  "sod_flattening", "weno_flattening_reflect", "llf_sod", "roe_sod_reflect",
                                  "sod_steepening", "mh_sod", "mh_rt_gravity", "mh_roe_flattening_reflect",
                                  "mh_primitive_noctu", "avisc_sod", "avisc_weno_periodic"])
def test_3d_fp64_matches_oracle(oracle, need_gpu, case):
    """3-D path (full CTU corner coupling, gravity, WENO) against the oracle,
    three steps, bit for bit."""
    if case == "ppm_periodic":
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_PERIODIC,) * 6)
        hp = HydroParams(gamma=5.0 / 3.0)
        unk = S.noisy_gas(geom, hp)
    elif case == "sod_outflow":
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams()
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    elif case == "rt_weno_gravity":
        geom = Geometry(3, 16, 16, 16, 1, 1, 2, bbox=((0, 1), (0, 1), (0, 2)),
                        bc=(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING))
        hp = HydroParams(order=5, useGravity=True, gravity=(0.0, 0.0, -0.1))
        unk = S.rayleigh_taylor(geom, hp)
    elif case == "hll_noctu":
        geom = Geometry(3, 16, 16, 16, 1, 2, 1, bc=(BC_PERIODIC,) * 6)
        hp = HydroParams(RiemannSolver="HLL", use_3dFullCTU=False, slopeLimiter="minmod")
        unk = S.noisy_gas(geom, hp)
    elif case == "sod_steepening":
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams(use_steepening=True)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    elif case == "llf_sod":
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams(RiemannSolver="LLF")
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    elif case == "roe_sod_reflect":
        geom = Geometry(3, 16, 16, 16, 1, 2, 1, bc=(BC_REFLECTING,) * 6)
        hp = HydroParams(RiemannSolver="Roe", order=5)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    elif case == "sod_flattening":
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams(use_flattening=True)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    elif case == "avisc_sod":
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams(use_avisc=True)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    elif case == "avisc_weno_periodic":
        geom = Geometry(3, 16, 16, 16, 1, 1, 2, bc=(BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING,
                                                    BC_PERIODIC, BC_PERIODIC))
        hp = HydroParams(order=5, use_avisc=True, cvisc=0.2, gamma=5.0 / 3.0)
        unk = S.noisy_gas(geom, hp)
    elif case == "mh_sod":
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6)
        hp = HydroParams(order=2)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    elif case == "mh_rt_gravity":
        geom = Geometry(3, 16, 16, 16, 1, 1, 2, bbox=((0, 1), (0, 1), (0, 2)),
                        bc=(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING))
        hp = HydroParams(order=2, useGravity=True, gravity=(0.0, 0.0, -0.1))
        unk = S.rayleigh_taylor(geom, hp)
    elif case == "mh_roe_flattening_reflect":
        geom = Geometry(3, 16, 16, 16, 1, 2, 1, bc=(BC_REFLECTING,) * 6)
        hp = HydroParams(order=2, RiemannSolver="Roe", use_flattening=True)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    elif case == "mh_primitive_noctu":
        geom = Geometry(3, 16, 16, 16, 1, 2, 1, bc=(BC_PERIODIC,) * 6)
        hp = HydroParams(order=2, charLimiting=False, use_3dFullCTU=False, slopeLimiter="vanLeer")
        unk = S.noisy_gas(geom, hp)
    elif case == "weno_flattening_reflect":
        geom = Geometry(3, 16, 16, 16, 1, 1, 1, bc=(BC_REFLECTING,) * 6)
        hp = HydroParams(order=5, use_flattening=True)
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    else:
        geom = Geometry(3, 16, 16, 16, 1, 1, 1, bc=(BC_REFLECTING,) * 6)
        hp = HydroParams(order=5, wenoMethod="WENOZ")
        unk = S.sod(geom, hp, xangle=30.0, yangle=70.0, posn=0.6)
    p = oracle.make_params(geom.as_dict(), hp)
    dts, ref = oracle_dts(oracle, geom, hp, unk, 3, first=0.5 * oracle.compute_dt(p, unk))
    _, out = gpu_run(geom, hp, unk, dts)
    g, r = compare(geom, out, ref)
    assert np.max(_rel(g, r)) <= REL_TOL_ONE_STEP
    assert np.array_equal(g, r)


def test_3d_conservation_and_mixed(need_gpu):
    geom = Geometry(3, 16, 16, 16, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams(gamma=5.0 / 3.0)
    unk = S.noisy_gas(geom, hp)
    outs = {}
    for prec in ("fp64", "mixed"):
        dev = HydroDevice(geom, hp, prec)
        dev.attach_unk(unk.copy())
        I0 = dev.integrals()
        dt = 0.5 * dev.Hydro_computeDt() if prec == "fp64" else dt0
        dt0 = dt
        dev.advance(10, dt, dt)
        I1 = dev.integrals()
        assert abs(I1[0] - I0[0]) / I0[0] < 1e-13
        assert abs(I1[4] - I0[4]) / I0[4] < 1e-13
        o = np.zeros(geom.unk_shape)
        dev.sync_to_host(o)
        outs[prec] = S.gather_global(geom, o)
    a, b = outs["mixed"], outs["fp64"]
    assert np.mean(np.abs(a[..., DENS] - b[..., DENS])) / np.mean(b[..., DENS]) <= L1_TOL_MIXED


def _expected_loc(geom, unk, levels=None, deltas=None):
    """Flash-X dtMinLoc from a host UNK: first cell (block, k, j, i) of maximal rate."""
    g = geom.nguard
    k0 = g if geom.ndim == 3 else 0
    j0 = g if geom.ndim >= 2 else 0
    nk = geom.nzb if geom.ndim == 3 else 1
    nj = geom.nyb if geom.ndim >= 2 else 1
    best, loc = -1.0, None
    for b in range(unk.shape[0]):
        u = unk[b, k0:k0 + nk, j0:j0 + nj, g:g + geom.nxb, :]
        dx, dy, dz = deltas[b] if deltas is not None else geom.deltas()
        cs = np.sqrt(u[..., GAMC] * u[..., PRES] / u[..., DENS])
        r = (np.abs(u[..., VELX] - 0.) + cs) * (1.0 / dx)
        if geom.ndim > 1:
            r = np.maximum(r, (np.abs(u[..., VELY] - 0.) + cs) * (1.0 / dy))
        if geom.ndim > 2:
            r = np.maximum(r, (np.abs(u[..., VELZ] - 0.) + cs) * (1.0 / dz))
        m = r.max()
        if m > best:
            best = m
            k, j, i = np.unravel_index(np.argmax(r), r.shape)
            loc = [int(i) + g + 1, int(j) + j0 + 1, int(k) + k0 + 1,
                   int(levels[b]) if levels is not None else 1, b + 1]
    return loc


@pytest.mark.parametrize("name", ["kh2d", "sweep3d"])
def test_compute_dt_location(need_gpu, name):
    """fxb_compute_dt's limiting cell equals the first cell of maximal CFL rate,
    in Hydro_computeDt's index convention, before and after a step."""
    geom, hp, init = S.config(name, scale=0.25 if name == "kh2d" else 0.5)
    unk = init(geom, hp)
    dev = HydroDevice(geom, hp, "fp64")
    dev.attach_unk(unk.copy())
    dt, loc = dev.Hydro_computeDt(location=True)
    assert loc == _expected_loc(geom, unk)
    dev.Hydro(0.0, 0.5 * dt, 0.5 * dt)
    dt2, loc2 = dev.Hydro_computeDt(location=True)
    out = np.zeros(geom.unk_shape)
    dev.sync_to_host(out)
    assert loc2 == _expected_loc(geom, out)
    dev.close()


def _transonic_rarefaction(hp):
    """Toro's test 1 along x (rho, u, p = 1, 0.75, 1 | 0.125, 0, 0.1 at x = 0.3):
    its left rarefaction is sonic, so the acoustic eigenvalues change sign
    across faces and Roe's entropy fix acts."""
    geom = Geometry(2, 16, 16, 1, 4, 1, 1, bc=(BC_OUTFLOW,) * 4 + (BC_OUTFLOW, BC_OUTFLOW))
    nx, ny = geom.nxb * geom.nblockx, geom.nyb * geom.nblocky
    xc = (np.arange(nx) + 0.5) / nx
    X = np.broadcast_to(xc, (1, ny, nx))
    left = X < 0.3
    rho = np.where(left, 1.0, 0.125)
    vx = np.where(left, 0.75, 0.0)
    p = np.where(left, 1.0, 0.1)
    f = S._finish(hp, rho, vx, 0 * X, 0 * X, p)
    return geom, S.scatter_global(geom, f)


@pytest.mark.parametrize("entropy,method", [(False, "HartenHyman"), (True, "HartenHyman"), (True, "Harten")])
def test_roe_entropy_fix_fp64(oracle, need_gpu, entropy, method):
    hp = HydroParams(RiemannSolver="Roe", entropy=entropy, entropyFixMethod=method)
    geom, unk = _transonic_rarefaction(hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dts, ref = oracle_dts(oracle, geom, hp, unk, 5, first=0.5 * oracle.compute_dt(p, unk))
    _, out = gpu_run(geom, hp, unk, dts)
    g, r = compare(geom, out, ref)
    assert np.array_equal(g, r)
    if entropy:   # the fix changes the solution here
        hp0 = HydroParams(RiemannSolver="Roe")
        _, ref0 = oracle_dts(oracle, geom, hp0, unk, 5, first=dts[0])
        assert not np.array_equal(ref, ref0)


@pytest.mark.parametrize("ndim", [2, 3])
def test_muscl_hancock_mixed_close_to_fp64(need_gpu, ndim):
    """order = 2 in the FP32-reconstruction path stays within the mixed-precision
    tolerance of the FP64 path (20 steps)."""
    if ndim == 2:
        geom, _, init = S.config("kh2d", scale=1 / 16)
    else:
        geom = Geometry(3, 16, 16, 16, 2, 2, 2, bc=(BC_PERIODIC,) * 6)
        init = S.noisy_gas
    hp = HydroParams(order=2, gamma=1.4 if ndim == 2 else 5.0 / 3.0)
    unk = init(geom, hp)
    outs = []
    for prec in ("fp64", "mixed"):
        dev = HydroDevice(geom, hp, prec)
        dev.attach_unk(unk.copy())
        dt = 0.5 * dev.Hydro_computeDt()
        for _ in range(20):
            dev.Hydro(0.0, dt, dt)
        o = np.zeros(geom.unk_shape)
        dev.sync_to_host(o)
        outs.append(S.gather_global(geom, o)[..., DENS])
        dev.close()
    l1 = np.mean(np.abs(outs[1] - outs[0])) / np.mean(np.abs(outs[0]))
    assert 0 < l1 <= L1_TOL_MIXED


def rough_gas(geom, hp, sig=1.0, vmag=1.0):
    """Log-normal density (exp of a seeded normal field), velocities uniform in
    [-vmag, vmag], p = 1: steep, converging cells where hybrid order acts."""
    import math
    xc, yc, zc, _, _ = S.cell_coords(geom)
    shape = (len(zc), len(yc), len(xc))
    idx = np.arange(int(np.prod(shape)), dtype=np.uint64).reshape(shape)
    u1, u2 = S.uniform01(idx, stream=30)
    n1 = np.sqrt(-2.0 * np.log(1.0 - u1)) * np.cos(2.0 * math.pi * u2)
    u3, u4 = S.uniform01(idx, stream=31)
    rho = np.exp(sig * n1)
    vx, vy = vmag * (2 * u3 - 1), vmag * (2 * u4 - 1)
    vz = 0 * vx if geom.ndim == 2 else vmag * (2 * u1 - 1)
    return S.scatter_global(geom, S._finish(hp, rho, vx, vy, vz, np.ones_like(rho)))


@pytest.mark.parametrize("ndim,opts", [
    (2, dict()), (2, dict(hybridOrderKappa=0.3)), (2, dict(order=2)), (2, dict(order=5)),
    (3, dict()), (3, dict(order=2, hybridOrderKappa=0.2)),
])
def test_hybrid_order_fp64(oracle, need_gpu, ndim, opts):
    """use_hybridOrder (hy_dataReconstOneStep.F90:864-913) on a rough gas with
    gamma = 3, where face states break the shock density bounds: bit for bit,
    and different from the run without it."""
    if ndim == 2:
        geom = Geometry(2, 16, 16, 1, 2, 2, 1, bc=(BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_OUTFLOW, 1, 1))
    else:
        geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams(use_hybridOrder=True, gamma=3.0, **opts)
    unk = rough_gas(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    dts, ref = oracle_dts(oracle, geom, hp, unk, 3, first=0.5 * oracle.compute_dt(p, unk))
    _, out = gpu_run(geom, hp, unk, dts)
    g, r = compare(geom, out, ref)
    assert np.array_equal(g, r)
    hp0 = HydroParams(gamma=3.0, **opts)
    ref0 = oracle_run(oracle, geom, hp0, unk, dts)
    assert not np.array_equal(ref, ref0)   # the fallback acted
