"""CPU tests of the oracle (the checker the CUDA path is compared with).

The reference ships no golden vectors for this path (its Comparison-test
checkpoints live off-tree), so the oracle is pinned by known answers:
the exact Sod solution (Sod/shocktube.pro), hand Riemann problems, Eos
identities, guard-cell semantics and conservation, plus committed fixtures
that guard it against regressions (tests/golden/gen_golden.py).
"""
import math
import sys
import os

import numpy as np
import pytest

from flashx_b200 import simulations as S
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING, DENS, EINT, ENER, GAMC, GAME,
                                Geometry, HydroParams, PRES, SHOK, TEMP, VELX, VELY)
from exact_sod import sod_exact

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def run_oracle(O, geom, hp, unk, tmax=None, nsteps=None):
    p = O.make_params(geom.as_dict(), hp)
    dt_cfl = O.compute_dt(p, unk)
    dt = 0.1 * dt_cfl if hp.dtinit > 0.1 * dt_cfl else hp.dtinit
    dt_old = dt
    t, n = 0.0, 0
    while (tmax is None or t < tmax) and (nsteps is None or n < nsteps):
        if tmax is not None and t + dt > tmax:
            dt = tmax - t
        O.hydro_step(p, unk, dt, dt_old)
        t += dt
        n += 1
        dt_old = dt
        dt = O.driver_dt(O.compute_dt(p, unk), dt_old)
    return t, n


@pytest.mark.parametrize("order", [3, 2])
def test_sod_2d_matches_exact_solution(oracle, order):
    """2-D Sod at 45 degrees, 128^2: density along the diagonal vs the exact
    solution at t=0.2 (the analytic check of Sod/shocktube.pro, soderror.pro),
    with PPM and with MUSCL-Hancock (order 2, same bounds)."""
    geom = Geometry(2, 16, 16, 1, 8, 8, 1, bc=(BC_OUTFLOW,) * 6)
    hp = HydroParams(order=order)
    unk = S.sod(geom, hp)
    t, n = run_oracle(oracle, geom, hp, unk, tmax=0.2)
    assert abs(t - 0.2) < 1e-12 and n > 50
    g = S.gather_global(geom, unk)[0]
    N = g.shape[0]
    dx = 1.0 / N
    idx = np.arange(N)
    x = (idx + 0.5) * dx
    xi = (2 * x - 1.0) / math.sqrt(2.0) + 0.5          # coordinate along the tube normal
    rho_ex, u_ex, p_ex = sod_exact(xi, 0.2)
    rho = g[idx, idx, DENS]
    pres = g[idx, idx, PRES]
    vn = (g[idx, idx, VELX] + g[idx, idx, VELY]) / math.sqrt(2.0)
    keep = (xi > 0.05) & (xi < 0.95)
    l1 = lambda a, b: np.mean(np.abs(a[keep] - b[keep]))
    assert l1(rho, rho_ex) < 0.01
    assert l1(pres, p_ex) < 0.01
    assert l1(vn, u_ex) < 0.02
    # plateau values between contact and shock
    mid = (xi > 0.74) & (xi < 0.80)
    assert np.allclose(rho[mid], 0.26557, atol=5e-3)
    assert np.allclose(pres[mid], 0.30313, atol=3e-3)


def test_conservation_periodic_kh(oracle):
    """Mass, momentum and total energy are conserved to roundoff on a periodic domain."""
    geom = Geometry(2, 16, 16, 1, 4, 4, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams()
    unk = S.kelvin_helmholtz(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    I0 = oracle.integrals(p, unk)
    run_oracle(oracle, geom, hp, unk, nsteps=20)
    I1 = oracle.integrals(p, unk)
    assert abs(I1[0] - I0[0]) / I0[0] < 1e-13
    assert abs(I1[1] - I0[1]) < 1e-13 * I0[0]
    assert abs(I1[4] - I0[4]) / I0[4] < 1e-13


def test_eos_dens_ei_identities(oracle):
    geom = Geometry(2, 16, 16, 1, 2, 2, 1)
    hp = HydroParams()
    unk = S.kelvin_helmholtz(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    oracle.eos_interior(p, unk)
    g = S.gather_global(geom, unk)[0]
    assert np.allclose(g[..., PRES], (hp.gamma - 1) * g[..., DENS] * g[..., EINT], rtol=1e-14)
    assert np.allclose(g[..., GAME], hp.gamma, rtol=1e-14)
    assert np.all(g[..., GAMC] == hp.gamma)
    ekin = 0.5 * (g[..., VELX] ** 2 + g[..., VELY] ** 2)
    assert np.allclose(g[..., ENER], g[..., EINT] + ekin, rtol=1e-14)
    assert np.allclose(g[..., TEMP], g[..., EINT] * (hp.gamma - 1) / hp.gasConstant, rtol=1e-13)


def _state(rho, u, v, w, p, g=1.4):
    return np.array([rho, u, v, w, p, g, g, p / ((g - 1) * rho)])


def _phys_flux(V, d, g=1.4):
    rho, vel, p = V[0], V[1:4], V[4]
    E = 0.5 * rho * np.dot(vel, vel) + p / (g - 1)
    F = np.zeros(6)
    F[0] = rho * vel[d]
    F[1:4] = rho * vel[d] * vel
    F[1 + d] += p
    F[4] = (E + p) * vel[d]
    F[5] = p
    return F


def _cons(V):
    rho, vel, p, g = V[0], np.array(V[1:4]), V[4], V[6]
    return np.array([rho, *(rho * vel), 0.5 * rho * np.dot(vel, vel) + p / (g - 1), 0.0])


@pytest.mark.parametrize("solver", ["HLLC", "HLL", "LLF", "Roe"])
def test_riemann_known_answers(oracle, solver):
    geom = Geometry(2, 16, 16, 1, 1, 1, 1)
    hp = HydroParams(RiemannSolver=solver)
    p = oracle.make_params(geom.as_dict(), hp)
    # identical states: the physical flux
    V = _state(1.3, 0.2, -0.1, 0.05, 0.9)
    for d in range(3):
        F = oracle.riemann(p, d, V, V)
        assert np.allclose(F[:6], _phys_flux(V, d), rtol=1e-14, atol=1e-15)
    # supersonic to the right: HLL(C) give the upwind flux of the left state;
    # LLF (hy_LLF.F90) the mean flux less the largest |u| + c of the mean,
    # left and right states times the conserved jump
    VL, VR = _state(1.0, 5.0, 0, 0, 1.0), _state(0.5, 4.0, 0, 0, 0.3)
    F = oracle.riemann(p, 0, VL, VR)
    if solver == "Roe":
        # supersonic: every wave speed of the mean state is positive, so the
        # conserved fluxes are the left flux up to the mean-state linearisation
        # (the mass flux exactly); the pressure slot is the mean pressure
        assert F[0] == pytest.approx(_phys_flux(VL, 0)[0], rel=1e-15)
        assert np.allclose(F[:5], _phys_flux(VL, 0)[:5], rtol=0.01)
        assert F[5] == 0.5 * (VL[4] + VR[4])
    elif solver == "LLF":
        c = lambda V: np.sqrt(V[5] * V[4] / V[0])
        Va = 0.5 * (np.array(VL) + np.array(VR))
        smax = max(abs(Va[1]) + np.sqrt(Va[5] * Va[4] / Va[0]), abs(VL[1]) + c(VL), abs(VR[1]) + c(VR))
        want = 0.5 * (_phys_flux(VR, 0) + _phys_flux(VL, 0) - smax * (_cons(VR) - _cons(VL)))
        assert np.allclose(F[:6], want, rtol=1e-14)
    else:
        assert np.allclose(F[:6], _phys_flux(VL, 0), rtol=1e-14)
    # aux-eint fluxes follow the mass flux upwind (hy_getFaceFlux.F90:444-453)
    assert F[7] == pytest.approx(F[0] / VL[0]) and F[6] == pytest.approx(F[0] * VL[7])
    # stationary contact: HLLC and Roe resolve it exactly (zero mass flux), HLL and LLF diffuse it
    VL, VR = _state(1.0, 0, 0, 0, 1.0), _state(0.1, 0, 0, 0, 1.0)
    F = oracle.riemann(p, 0, VL, VR)
    if solver in ("HLLC", "Roe"):
        assert F[0] == 0.0 and F[1] == pytest.approx(1.0, rel=1e-15)
    else:
        assert F[0] > 1e-3
    # vacuum guard returns zero flux
    VL = _state(1e-40, 0, 0, 0, 1.0)
    F = oracle.riemann(p, 0, VL, VR)
    assert np.all(F[:6] == 0.0)
    # imaginary sound speed is an error (ierr=1)
    bad = _state(1.0, 0, 0, 0, 1.0)
    bad[5] = -1.4
    with pytest.raises(RuntimeError):
        oracle.riemann(p, 0, bad, VR)


@pytest.mark.parametrize("bc", [BC_OUTFLOW, BC_REFLECTING, BC_PERIODIC])
def test_guardcell_fill_semantics(oracle, bc):
    """Grid_fillGuardCells: outflow copies the first interior cell, reflecting
    mirrors and flips the normal velocity, periodic wraps
    (Grid_bcApplyToRegion.F90:458-531, UG/gr_shiftData.F90)."""
    geom = Geometry(2, 16, 16, 1, 2, 2, 1, bc=(bc,) * 6)
    rng = np.random.default_rng(1)
    unk = S.scatter_global(geom, rng.random((1, 32, 32, 11)) + 0.5)
    glob = S.gather_global(geom, unk)[0]
    p = oracle.make_params(geom.as_dict(), HydroParams())
    oracle.fill_guardcells(p, unk)
    blk0 = unk[0, 0]           # block at the low-x, low-y corner; (j, i, var), guard 4
    # low-x guard column i=3 (one cell outside) at interior row j=4..19
    col = blk0[4:20, 3, :]
    if bc == BC_OUTFLOW:
        assert np.array_equal(col, glob[0:16, 0, :])
    elif bc == BC_REFLECTING:
        ref = glob[0:16, 0, :].copy()
        ref[:, VELX] *= -1
        assert np.array_equal(col, ref)
    else:
        assert np.array_equal(col, glob[0:16, 31, :])
    # interior-block boundary: block 1 (bx=1) guard column i=3 holds block 0's last column
    assert np.array_equal(unk[1, 0][4:20, 3, :], glob[0:16, 15, :])
    # corner guard (3,3) of block 0
    c = blk0[3, 3, :]
    if bc == BC_OUTFLOW:
        assert np.array_equal(c, glob[0, 0, :])
    elif bc == BC_PERIODIC:
        assert np.array_equal(c, glob[31, 31, :])
    else:
        ref = glob[0, 0, :].copy()
        ref[VELX] *= -1
        ref[VELY] *= -1
        assert np.array_equal(c, ref)


def test_driver_dt_control(oracle):
    # Driver_computeDt.F90:452,460
    assert oracle.driver_dt(1.0, 0.1) == pytest.approx(0.2)
    assert oracle.driver_dt(0.15, 0.1) == 0.15
    assert oracle.driver_dt(1e-20, 0.1) == 1e-10
    from flashx_b200.hydro import driver_dt, initial_dt
    hp = HydroParams()
    for a, b in [(1.0, 0.1), (0.15, 0.1), (1e-20, 0.1)]:
        assert driver_dt(a, b, hp) == oracle.driver_dt(a, b)
    assert initial_dt(1.0, hp) == 1e-10 and initial_dt(1e-12, hp) == pytest.approx(1e-13)


def test_weno_and_hll_paths_run_and_conserve(oracle):
    geom = Geometry(2, 16, 16, 1, 2, 2, 1, bc=(BC_PERIODIC,) * 6)
    for hp in (HydroParams(order=5), HydroParams(order=5, wenoMethod="WENOZ"),
               HydroParams(RiemannSolver="HLL", slopeLimiter="minmod"),
               HydroParams(slopeLimiter="vanLeer", charLimiting=False)):
        unk = S.kelvin_helmholtz(geom, hp)
        p = oracle.make_params(geom.as_dict(), hp)
        I0 = oracle.integrals(p, unk)
        run_oracle(oracle, geom, hp, unk, nsteps=5)
        I1 = oracle.integrals(p, unk)
        assert np.all(np.isfinite(unk))
        assert abs(I1[0] - I0[0]) / I0[0] < 1e-13
        assert abs(I1[4] - I0[4]) / I0[4] < 1e-13


def test_3d_oracle_sod_and_conservation(oracle):
    """3-D PPM with full CTU corner coupling: Sod along x stays planar, and a
    periodic noisy gas conserves mass and energy."""
    geom = Geometry(3, 16, 16, 16, 2, 1, 1, bc=(BC_OUTFLOW,) * 6)
    hp = HydroParams()
    unk = S.sod(geom, hp, xangle=0.0, yangle=90.0, posn=0.5)
    run_oracle(oracle, geom, hp, unk, nsteps=10)
    g = S.gather_global(geom, unk)
    assert np.allclose(g[:, :, :, DENS], g[0:1, 0:1, :, DENS], rtol=0, atol=1e-14)
    geom = Geometry(3, 16, 16, 16, 1, 1, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams(gamma=5.0 / 3.0)
    unk = S.noisy_gas(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    I0 = oracle.integrals(p, unk)
    run_oracle(oracle, geom, hp, unk, nsteps=3)
    I1 = oracle.integrals(p, unk)
    assert abs(I1[0] - I0[0]) / I0[0] < 1e-13
    assert abs(I1[4] - I0[4]) / I0[4] < 1e-13


@pytest.mark.parametrize("name", ["sod2d_1step", "kh2d_3step"])
def test_golden_fixtures(oracle, name):
    """Committed oracle outputs (tests/golden/gen_golden.py) reproduce bit for bit."""
    path = os.path.join(GOLDEN, name + ".npz")
    z = np.load(path)
    sys.path.insert(0, GOLDEN)
    from gen_golden import CASES
    geom, hp, init, nsteps = CASES[name]()
    unk = init(geom, hp)
    run_oracle(oracle, geom, hp, unk, nsteps=nsteps)
    g = S.gather_global(geom, unk)
    assert np.array_equal(g, z["state"])


def test_flattening_acts_only_at_strong_shocks(oracle):
    """use_flattening (hy_getRiemannState.F90:367-465): FlatTilde vanishes where
    the pressure jump is below a third of the local pressure, so a smooth flow
    evolves bit-identically with and without it; at the Sod shock it switches
    on, adds diffusion, and the solution stays close to the exact one."""
    geom = Geometry(2, 16, 16, 1, 4, 4, 1, bc=(BC_PERIODIC,) * 6)
    outs = []
    for flat in (False, True):
        hp = HydroParams(use_flattening=flat, gamma=5.0 / 3.0)
        unk = S.noisy_gas(geom, hp)
        run_oracle(oracle, geom, hp, unk, nsteps=5)
        outs.append(unk)
    np.testing.assert_array_equal(outs[0], outs[1])

    geom = Geometry(2, 16, 16, 1, 8, 8, 1, bc=(BC_OUTFLOW,) * 6)
    res = []
    for flat in (False, True):
        hp = HydroParams(use_flattening=flat)
        unk = S.sod(geom, hp)
        run_oracle(oracle, geom, hp, unk, tmax=0.2)
        g = S.gather_global(geom, unk)[0]
        N = g.shape[0]
        idx = np.arange(N)
        xi = (2 * (idx + 0.5) / N - 1.0) / math.sqrt(2.0) + 0.5
        rho_ex, _, _ = sod_exact(xi, 0.2)
        keep = (xi > 0.05) & (xi < 0.95)
        res.append((g, np.mean(np.abs(g[idx, idx, DENS][keep] - rho_ex[keep]))))
    assert not np.array_equal(res[0][0], res[1][0])
    assert res[1][1] < 5e-3


def test_artificial_viscosity_conserves_and_acts(oracle):
    """use_avisc (hy_getFaceFlux.F90:397-438): the viscous fluxes are
    conservative (periodic KH keeps mass, momentum and energy to roundoff)
    and change the solution where the flow converges (Sod)."""
    geom = Geometry(2, 16, 16, 1, 4, 4, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams(use_avisc=True, cvisc=0.3)
    unk = S.kelvin_helmholtz(geom, hp)
    p = oracle.make_params(geom.as_dict(), hp)
    I0 = oracle.integrals(p, unk)
    run_oracle(oracle, geom, hp, unk, nsteps=20)
    I1 = oracle.integrals(p, unk)
    assert abs(I1[0] - I0[0]) / I0[0] < 1e-13
    assert abs(I1[1] - I0[1]) < 1e-13 * I0[0]
    assert abs(I1[4] - I0[4]) / I0[4] < 1e-13
    g2 = Geometry(2, 16, 16, 1, 4, 4, 1, bc=(BC_OUTFLOW,) * 6)
    outs = []
    for av in (False, True):
        h = HydroParams(use_avisc=av)
        u = S.sod(g2, h)
        run_oracle(oracle, g2, h, u, nsteps=10)
        outs.append(S.gather_global(g2, u)[..., DENS])
    assert not np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("order", [2, 3, 5])
def test_gravity_2d_free_fall_and_axis_symmetry(oracle, order):
    """Constant gravity in 2-D (hy_getRiemannState.F90:843-885,
    hy_unsplitUpdate.F90:1234-1245, hy_gravityStepBlk.F90:54-78).
    A uniform periodic gas falls freely: every cell's velocity grows by g dt
    per step (the two half steps) while density and pressure stay put.  And
    the 2-D Rayleigh-Taylor problem with gravity along y, transposed so that
    gravity acts along x, gives the transposed result."""
    g = (0.03, -0.1, 0.0)
    geom = Geometry(2, 16, 16, 1, 2, 2, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams(order=order, useGravity=True, gravity=g)
    shape = (1, 32, 32)
    one = np.ones(shape)
    unk = S.scatter_global(geom, S._finish(hp, one, 0.0 * one, 0.0 * one, 0.0 * one, one))
    p = oracle.make_params(geom.as_dict(), hp)
    dt = 0.5 * oracle.compute_dt(p, unk)
    for _ in range(4):
        oracle.hydro_step(p, unk, dt, dt)
    f = S.gather_global(geom, unk)
    assert np.allclose(f[..., VELX], 4 * dt * g[0], rtol=1e-12, atol=0)
    assert np.allclose(f[..., VELY], 4 * dt * g[1], rtol=1e-12, atol=0)
    assert np.allclose(f[..., DENS], 1.0, rtol=1e-13, atol=0)
    assert np.allclose(f[..., PRES], 1.0, rtol=1e-12, atol=0)

    # Rayleigh-Taylor along y, and the same problem with x as the vertical axis
    geom_y = Geometry(2, 16, 16, 1, 2, 3, 1, bbox=((0.0, 1.0), (0.0, 1.5), (0.0, 1.0)),
                      bc=(BC_PERIODIC, BC_PERIODIC, BC_REFLECTING, BC_REFLECTING, BC_OUTFLOW, BC_OUTFLOW))
    geom_x = Geometry(2, 16, 16, 1, 3, 2, 1, bbox=((0.0, 1.5), (0.0, 1.0), (0.0, 1.0)),
                      bc=(BC_REFLECTING, BC_REFLECTING, BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW))
    hp_y = HydroParams(order=order, useGravity=True, gravity=(0.0, -0.1, 0.0))
    hp_x = HydroParams(order=order, useGravity=True, gravity=(-0.1, 0.0, 0.0))
    uy = S.rayleigh_taylor(geom_y, hp_y)
    fy = S.gather_global(geom_y, uy)
    fx = fy.transpose(0, 2, 1, 3).copy()
    fx[..., [VELX, VELY]] = fx[..., [VELY, VELX]]
    ux = S.scatter_global(geom_x, fx)
    py, px = oracle.make_params(geom_y.as_dict(), hp_y), oracle.make_params(geom_x.as_dict(), hp_x)
    dt = 0.5 * oracle.compute_dt(py, uy)
    for _ in range(3):
        oracle.hydro_step(py, uy, dt, dt)
        oracle.hydro_step(px, ux, dt, dt)
    ry = S.gather_global(geom_y, uy)
    rx = S.gather_global(geom_x, ux).transpose(0, 2, 1, 3).copy()
    rx[..., [VELX, VELY]] = rx[..., [VELY, VELX]]
    sel = [DENS, VELX, VELY, PRES, ENER, EINT]
    assert np.max(np.abs(ry[..., VELY])) > 1e-4          # the interface moves
    scale = np.maximum(np.abs(ry[..., sel]), 1e-3)
    assert np.max(np.abs(rx[..., sel] - ry[..., sel]) / scale) < 1e-11


# ---- species and mass scalars (hy_fullSpecMsFluxHandling) ----------------------
def _uniform_flow(geom, hp, v=(0.5, 0.3, 0.2)):
    xc, yc, zc, _, _ = S.cell_coords(geom)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    one = np.ones_like(X)
    return S.scatter_global(geom, S._finish(hp, one, v[0] * one, v[1] * one, (v[2] if geom.ndim == 3 else 0.) * one, one))


@pytest.mark.parametrize("ndim,order", [(2, 3), (2, 5), (2, 2), (3, 3), (3, 5)])
def test_species_oracle_conservation_and_hydro_unchanged(oracle, ndim, order):
    """Advected mass fractions on a periodic KH-like flow: the hydro state is
    the same with and without them, the mass of every mass scalar is conserved
    to round-off, the species stay normalised, and the mass of each species
    stays conserved up to the renormalisation's round-off."""
    geom = (Geometry(2, 16, 16, 1, 2, 2, 1, bc=(BC_PERIODIC,) * 6) if ndim == 2 else
            Geometry(3, 8, 8, 8, 2, 2, 2, bc=(BC_PERIODIC,) * 6))
    hp = HydroParams(order=order)
    unk = S.kelvin_helmholtz(geom, hp)
    spec = S.species_blob(geom, ns=3, nspecies=2)
    p = oracle.make_params(geom.as_dict(), hp)
    ref = unk.copy()
    u, sp = unk.copy(), spec.copy()
    dv = np.prod(geom.deltas()[:ndim])
    mass0 = [np.sum(S.gather_global(geom, u)[..., DENS] * S.gather_global(geom, sp)[..., q]) * dv for q in range(3)]
    dt = 0.4 * oracle.compute_dt(p, u)
    for _ in range(6):
        oracle.hydro_step(p, ref, dt, dt)
        oracle.hydro_step(p, u, dt, dt, spec=sp, nspecies=2)
    assert np.array_equal(u, ref)
    g, gs = S.gather_global(geom, u), S.gather_global(geom, sp)
    mass1 = [np.sum(g[..., DENS] * gs[..., q]) * dv for q in range(3)]
    assert abs(mass1[2] - mass0[2]) / mass0[2] < 1e-13
    for q in range(2):
        assert abs(mass1[q] - mass0[q]) / (mass0[0] + mass0[1]) < 1e-12
    assert np.max(np.abs(gs[..., 0] + gs[..., 1] - 1.0)) < 1e-14
    # PPM and MUSCL-Hancock stay within [0, 1]; WENO5 with 3-D CTU terms may dip slightly
    assert np.all(gs[..., 0] > -1e-3) and np.all(gs[..., 0] < 1 + 1e-3)


def test_species_oracle_uniform_and_translated(oracle):
    """A single species that is one everywhere stays one exactly; a smooth
    blob carried by a uniform periodic flow (rho = p = 1, v = (0.5, 0.3))
    arrives translated by v t (L1 error of the profile small), and a
    constant mass scalar stays constant to round-off."""
    geom = Geometry(2, 16, 16, 1, 4, 4, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams()
    unk = _uniform_flow(geom, hp)
    spec = S.species_blob(geom, ns=3, nspecies=1, radius=0.15, width=0.05)
    spec[..., 1] = 1.0            # a second "species" slot used as the constant mass scalar
    spec[..., 2] = 0.25
    one = np.ones(spec.shape[:-1] + (1,))
    p = oracle.make_params(geom.as_dict(), hp)
    dt = 0.5 * oracle.compute_dt(p, unk)
    t = 0.0
    u1, s1 = unk.copy(), one.copy()
    while t < 0.2 - 1e-12:
        step = min(dt, 0.2 - t)
        oracle.hydro_step(p, unk, step, step, spec=spec, nspecies=0)
        oracle.hydro_step(p, u1, step, step, spec=s1, nspecies=1)
        t += step
    assert np.all(S.gather_global(geom, s1) == 1.0)
    gs = S.gather_global(geom, spec)[0]
    assert np.max(np.abs(gs[..., 1] - 1.0)) < 1e-13 and np.max(np.abs(gs[..., 2] - 0.25)) < 1e-13
    xc, yc, _, _, _ = S.cell_coords(geom)
    Y, X = np.meshgrid(yc, xc, indexing="ij")
    dxp = (X - 0.5 - 0.5 * 0.2 + 0.5) % 1.0 - 0.5
    dyp = (Y - 0.5 - 0.3 * 0.2 + 0.5) % 1.0 - 0.5
    exact = 0.5 * (1.0 - np.tanh((np.sqrt(dxp ** 2 + dyp ** 2) - 0.15) / 0.05))
    assert np.mean(np.abs(gs[..., 0] - exact)) < 0.01


def test_species_oracle_transpose_symmetry(oracle):
    """Swapping x and y of the flow and of the blob swaps the result."""
    geom = Geometry(2, 16, 16, 1, 2, 2, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams()
    unk = S.kelvin_helmholtz(geom, hp)
    spec = S.species_blob(geom, ns=1, nspecies=0, center=(0.4, 0.6, 0.5))
    g, gs = S.gather_global(geom, unk), S.gather_global(geom, spec)
    gt = g.transpose(0, 2, 1, 3).copy()
    gt[..., [VELX, VELY]] = gt[..., [VELY, VELX]]
    ut, st = S.scatter_global(geom, gt), S.scatter_global(geom, gs.transpose(0, 2, 1, 3).copy())
    p = oracle.make_params(geom.as_dict(), hp)
    dt = 0.4 * oracle.compute_dt(p, unk)
    for _ in range(4):
        oracle.hydro_step(p, unk, dt, dt, spec=spec, nspecies=0)
        oracle.hydro_step(p, ut, dt, dt, spec=st, nspecies=0)
    a = S.gather_global(geom, spec)
    b = S.gather_global(geom, st).transpose(0, 2, 1, 3)
    assert np.max(np.abs(a - b)) < 1e-13


def _cons_eigenvectors(V, d):
    """hy_eigenVector.F90 (OnlyHydro, cons = .true.) in numpy, stored as the
    reference stores them: L[variable, wave], R[variable, wave]."""
    rho, vel, p, ge = V[0], np.array(V[1:4]), V[4], V[6]
    c = math.sqrt(V[5] * p / rho)
    v1, v2, v3 = 1 + d, 1 + (d + 1) % 3, 1 + (d + 2) % 3
    V1, V2, V3 = vel[d], vel[(d + 1) % 3], vel[(d + 2) % 3]
    k = 1 - ge
    na = 0.5 / c ** 2
    u2 = 0.5 * np.dot(vel, vel)
    H = (rho * u2 - p / k + p) / rho
    L = np.zeros((5, 5))
    Rm = np.zeros((5, 5))
    L[[0, v1, v2, v3, 4], 0] = [na * (-k * u2 + V1 * c), -na * (-k * V1 + c), na * k * V2, na * k * V3, -na * k]
    L[[0, v2], 1] = [-V2, 1]
    L[[0, v1, v2, v3, 4], 2] = [1 + 2 * na * k * u2, -k * V1 / c ** 2, -k * V2 / c ** 2, -k * V3 / c ** 2, k / c ** 2]
    L[[0, v3], 3] = [-V3, 1]
    L[[0, v1, v2, v3, 4], 4] = [na * (-k * u2 - V1 * c), -na * (-k * V1 - c), na * k * V2, na * k * V3, -na * k]
    Rm[[0, v1, v2, v3, 4], 0] = [1, V1 - c, V2, V3, H - V1 * c]
    Rm[[v2, 4], 1] = [1, V2]
    Rm[[0, v1, v2, v3, 4], 2] = [1, V1, V2, V3, u2]
    Rm[[v3, 4], 3] = [1, V3]
    Rm[[0, v1, v2, v3, 4], 4] = [1, V1 + c, V2, V3, H + V1 * c]
    lam = np.array([vel[d] - c, vel[d], vel[d], vel[d], vel[d] + c])
    return lam, L, Rm


def _marquina_numpy(VL, VR, d, modified):
    """hy_Marquina.F90:120-227 / hy_MarquinaModified.F90:120-195 line by line
    in numpy, Fortran indices kept: leigL(k, 1:5) is L[k, :] (the row of
    variable k across the waves, as the reference writes it)."""
    lamL, LL, RL = _cons_eigenvectors(VL, d)
    lamR, LR, RR = _cons_eigenvectors(VR, d)
    UL, UR = _cons(VL)[:5], _cons(VR)[:5]
    FL, FR = _phys_flux(VL, d), _phys_flux(VR, d)
    F = np.zeros(6)
    if modified:
        sig = np.zeros(5)
        for k in range(5):
            sig += 0.5 * (abs(lamL[k]) + abs(lamR[k])) * (RR[:, k] * (LR[:, k] @ UR) - RL[:, k] * (LL[:, k] @ UL))
        F[:5] = 0.5 * (FR[:5] + FL[:5] - sig)
        F[5] = 0.5 * (FR[5] + FL[5])
        return F
    amax = max(np.max(np.abs(lamL)), np.max(np.abs(lamR)))
    vL, vR = np.zeros(5), np.zeros(5)
    for k in range(5):
        if lamL[k] * lamR[k] > 0:
            if lamL[k] > 0:
                vL[k] = LL[k, :] @ FL[:5] + LL[k, 1 + d] * FL[5]
            else:
                vR[k] = LR[k, :] @ FR[:5] + LR[k, 1 + d] * FR[5]
        else:
            vL[k] = 0.5 * (LL[k, :] @ FL[:5] + amax * (LL[k, :] @ UL) + LL[k, 1 + d] * FL[5])
            vR[k] = 0.5 * (LR[k, :] @ FR[:5] - amax * (LR[k, :] @ UR) + LR[k, 1 + d] * FR[5])
    F[:5] = RL @ vL + RR @ vR
    return F


@pytest.mark.parametrize("solver", ["Marquina", "MarquinaModified"])
def test_marquina_fluxes_follow_the_reference_lines(oracle, solver):
    """The oracle's Marquina fluxes equal an independent numpy restatement of
    the reference routines (both directions, subsonic and supersonic pairs,
    waves of both signs) to rounding; MarquinaModified gives the physical
    flux of identical states, Marquina as written does not (its transposed
    left-eigenvector read and doubled face pressure make it inconsistent)."""
    geom = Geometry(2, 16, 16, 1, 1, 1, 1)
    p = oracle.make_params(geom.as_dict(), HydroParams(RiemannSolver=solver))
    rng = np.random.default_rng(7)
    for _ in range(40):
        VL = _state(rng.uniform(0.2, 2), *rng.uniform(-3, 3, 3), rng.uniform(0.1, 3))
        VR = _state(rng.uniform(0.2, 2), *rng.uniform(-3, 3, 3), rng.uniform(0.1, 3))
        for d in range(3):
            F = oracle.riemann(p, d, VL, VR)
            want = _marquina_numpy(VL, VR, d, solver == "MarquinaModified")
            assert np.allclose(F[:6], want, rtol=1e-11, atol=1e-11 * np.max(np.abs(want)))
    V = _state(1.3, 0.2, -0.1, 0.05, 0.9)
    F = oracle.riemann(p, 0, V, V)
    if solver == "MarquinaModified":
        assert np.array_equal(F[:6], _phys_flux(V, 0))
    else:
        assert not np.allclose(F[:5], _phys_flux(V, 0)[:5])
        assert F[5] == 0.0
    # vacuum guard and imaginary sound speed as the other solvers
    assert np.all(oracle.riemann(p, 0, _state(1e-40, 0, 0, 0, 1.0), V)[:6] == 0.0)
    bad = _state(1.0, 0, 0, 0, 1.0)
    bad[5] = -1.4
    with pytest.raises(RuntimeError):
        oracle.riemann(p, 0, bad, V)


def test_sod_2d_marquina_modified_matches_exact_solution(oracle):
    """MarquinaModified with PPM on the 45-degree Sod problem, 128^2, t = 0.2:
    the bounds of the HLLC test against the exact solution."""
    geom = Geometry(2, 16, 16, 1, 8, 8, 1, bc=(BC_OUTFLOW,) * 6)
    hp = HydroParams(RiemannSolver="MarquinaModified")
    unk = S.sod(geom, hp)
    t, n = run_oracle(oracle, geom, hp, unk, tmax=0.2)
    assert abs(t - 0.2) < 1e-12 and n > 50
    g = S.gather_global(geom, unk)[0]
    N = g.shape[0]
    idx = np.arange(N)
    x = (idx + 0.5) / N
    xi = (2 * x - 1.0) / math.sqrt(2.0) + 0.5
    rho_ex, u_ex, p_ex = sod_exact(xi, 0.2)
    keep = (xi > 0.05) & (xi < 0.95)
    l1 = lambda a, b: np.mean(np.abs(a[keep] - b[keep]))
    assert l1(g[idx, idx, DENS], rho_ex) < 0.01
    assert l1(g[idx, idx, PRES], p_ex) < 0.01
    assert l1((g[idx, idx, VELX] + g[idx, idx, VELY]) / math.sqrt(2.0), u_ex) < 0.02


def _shock_flags_numpy(unk, g):
    """hy_shockDetectBlk.F90 in numpy on a filled 2-D UNK: 1 where the sum of
    |central pressure difference| / 2 reaches 0.5 min p over the cell's 3x3
    box and the velocity divergence is at most -0.1 min c_s over the box."""
    out = np.zeros(unk.shape[:1] + (unk.shape[2] - 2 * g, unk.shape[3] - 2 * g))
    for b in range(unk.shape[0]):
        B = unk[b, 0]
        P = B[..., PRES]
        cs = np.sqrt(B[..., GAMC] * P / B[..., DENS])
        for j in range(g, B.shape[0] - g):
            for i in range(g, B.shape[1] - g):
                minP, minC = P[j - 1:j + 2, i - 1:i + 2].min(), cs[j - 1:j + 2, i - 1:i + 2].min()
                divv = 0.5 * ((B[j, i + 1, VELX] - B[j, i - 1, VELX]) + B[j + 1, i, VELY] - B[j - 1, i, VELY])
                gp = abs(0.5 * (P[j, i + 1] - P[j, i - 1])) + abs(0.5 * (P[j + 1, i] - P[j - 1, i]))
                out[b, j - g, i - g] = 1.0 if (gp >= 0.5 * minP and -0.1 * minC >= divv) else 0.0
    return out


def test_shock_detector_and_hybrid_solver(oracle):
    """shockDetect marks the cells the two switches of hy_shockDetectBlk pick
    (against numpy on the filled state before the step) and leaves them in
    UNK's SHOK slot; the hybrid Riemann solver (HLL next to a marked cell,
    HLLC elsewhere) stays within the exact Sod bounds at t = 0.2 and differs
    from plain HLLC."""
    geom = Geometry(2, 16, 16, 1, 8, 8, 1, bc=(BC_OUTFLOW,) * 6)
    hp = HydroParams(RiemannSolver="hybrid")
    assert hp.shock_detect
    p = oracle.make_params(geom.as_dict(), hp)
    u = S.sod(geom, hp)
    run_oracle(oracle, geom, hp, u, tmax=0.05)          # the shock has formed
    pre = u.copy()
    oracle.fill_guardcells(p, pre)
    dt = 0.5 * oracle.compute_dt(p, u)
    oracle.hydro_step(p, u, dt, dt)
    g = geom.nguard
    shok = u[:, 0, g:-g, g:-g, SHOK]
    assert np.array_equal(shok, _shock_flags_numpy(pre, g))
    assert 20 < shok.sum() < 0.2 * shok.size
    unk = S.sod(geom, hp)
    run_oracle(oracle, geom, hp, unk, tmax=0.2)
    gl = S.gather_global(geom, unk)[0]
    N = gl.shape[0]
    idx = np.arange(N)
    xi = (2 * (idx + 0.5) / N - 1.0) / math.sqrt(2.0) + 0.5
    rho_ex, u_ex, p_ex = sod_exact(xi, 0.2)
    keep = (xi > 0.05) & (xi < 0.95)
    assert np.mean(np.abs(gl[idx, idx, DENS][keep] - rho_ex[keep])) < 0.01
    assert np.mean(np.abs(gl[idx, idx, PRES][keep] - p_ex[keep])) < 0.01
    ref = S.sod(geom, HydroParams())
    run_oracle(oracle, geom, HydroParams(), ref, tmax=0.2)
    assert not np.array_equal(S.gather_global(geom, ref)[..., DENS], S.gather_global(geom, unk)[..., DENS])
