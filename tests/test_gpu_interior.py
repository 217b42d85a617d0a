"""GPU tests of the interior transfers (fxb_put_interior, fxb_get_interior):
the cells and variables they move, that guard cells stay as they were and
the other slots of interior cells get the values last read from the host,
and that a host loop which round-trips interiors every step steps exactly
like the device-resident loop (FP64, bit for bit)."""
import numpy as np
import pytest

from flashx_b200 import simulations as S
from flashx_b200.hydro import FlashXError, HydroDevice
from flashx_b200.parallel import SlabDecomposition
from flashx_b200.params import (BC_OUTFLOW, BC_PERIODIC, DENS, EINT, ENER, GAMC, GAME, NUNK, PRES, SHOK, TEMP,
                                VELX, VELY, VELZ, Geometry, HydroParams)

pytestmark = pytest.mark.gpu

DEV_VARS = [DENS, EINT, ENER, GAMC, GAME, PRES, TEMP, VELX, VELY, VELZ]


def _interior(geom, a):
    g = geom.nguard
    ks = slice(g, -g) if geom.ndim == 3 else slice(None)
    return a[:, ks, g:-g, g:-g, :]


def _guard_mask(geom, shape):
    m = np.ones(shape[:4], dtype=bool)
    g = geom.nguard
    ks = slice(g, -g) if geom.ndim == 3 else slice(None)
    m[:, ks, g:-g, g:-g] = False
    return m


def _cases():
    kh = Geometry(2, 16, 16, 1, 4, 3, 1, bc=(BC_PERIODIC,) * 6)
    rt = Geometry(3, 16, 16, 16, 2, 2, 2,
                  bc=(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW))
    return {
        "kh2d": (kh, HydroParams(), S.kelvin_helmholtz),
        "rt3d": (rt, HydroParams(order=5, useGravity=True, gravity=(0.0, 0.0, -0.1)), S.rayleigh_taylor),
        "sod_shock": (Geometry(2, 16, 16, 1, 4, 2, 1, bc=(BC_OUTFLOW,) * 6), HydroParams(shockDetect=True), S.sod),
    }


@pytest.mark.parametrize("name", ["kh2d", "rt3d", "sod_shock"])
def test_get_interior_writes_interiors_only(name, need_gpu):
    geom, hp, init = _cases()[name]
    unk = init(geom, hp)
    dev = HydroDevice(geom, hp, "fp64")
    dev.attach_unk(unk.copy())
    dt = 0.5 * dev.Hydro_computeDt()
    for _ in range(2):
        dev.Hydro(0.0, dt, dt)
    full = np.zeros(geom.unk_shape)
    dev.sync_to_host(full)
    sentinel = -7.25
    got = np.full(geom.unk_shape, sentinel)
    dev.get_interior(got)
    moved = DEV_VARS + ([SHOK] if hp.shockDetect else [])
    others = [v for v in range(NUNK) if v not in moved]
    gi, fi = _interior(geom, got), _interior(geom, full)
    assert np.array_equal(gi[..., moved], fi[..., moved])
    # the other slots of the rows carry the values last read from the host
    assert np.array_equal(gi[..., others], _interior(geom, unk)[..., others])
    assert np.all(got[_guard_mask(geom, geom.unk_shape)] == sentinel)
    if hp.shockDetect:
        assert gi[..., SHOK].sum() > 0
    dev.close()


def _one_step(geom, hp, put=None, attach=None):
    """A fresh device (the library holds one grid at a time): attach, then
    optionally put_interior, then one step; returns (dt, UNK after sync)."""
    dev = HydroDevice(geom, hp, "fp64")
    dev.attach_unk(np.ascontiguousarray(attach))
    if put is not None:
        dev.put_interior(put)
    dt = 0.5 * dev.Hydro_computeDt()
    dev.Hydro(0.0, dt, dt)
    out = np.zeros(geom.unk_shape)
    dev.sync_to_host(out)
    dev.close()
    return dt, out


@pytest.mark.parametrize("name", ["kh2d", "rt3d"])
def test_put_interior_equals_attach(name, need_gpu):
    """The device state after put_interior(h) is the state attach_unk(h)
    gives: interiors from h (its guard cells are not read), guard cells
    filled from them."""
    geom, hp, init = _cases()[name]
    unk = init(geom, hp)
    mod = unk.copy()
    rng = np.random.default_rng(7)
    inner = _interior(geom, mod)
    inner[..., DENS] *= 1.0 + 0.01 * rng.random(inner.shape[:4])
    inner[..., PRES] *= 1.0 + 0.01 * rng.random(inner.shape[:4])
    dta, oa = _one_step(geom, hp, attach=mod)
    mod[_guard_mask(geom, mod.shape)] = np.nan
    dtb, ob = _one_step(geom, hp, attach=unk, put=mod)
    assert dta == dtb
    assert np.array_equal(oa[..., DEV_VARS], ob[..., DEV_VARS])
    # and the put really replaced the attached state
    _, oc = _one_step(geom, hp, attach=unk)
    assert not np.array_equal(oa[..., DENS], oc[..., DENS])


@pytest.mark.parametrize("name", ["kh2d", "rt3d"])
def test_host_round_trip_loop_matches_resident_loop(name, need_gpu):
    """A driver whose host units touch UNK every step (put, step, get) steps
    bit for bit like the device-resident loop, dt sequence included."""
    geom, hp, init = _cases()[name]
    unk = init(geom, hp)
    runs = {}
    for mode in ("resident", "round_trip"):
        host = unk.copy()
        dev = HydroDevice(geom, hp, "fp64")
        dev.attach_unk(host)
        dt = 0.5 * dev.Hydro_computeDt()
        dts = []
        for _ in range(3):
            if mode == "round_trip":
                dev.put_interior(host)
            dev.Hydro(0.0, dt, dt)
            if mode == "round_trip":
                dev.get_interior(host)
            dt = min(dt, dev.Hydro_computeDt())
            dts.append(dt)
        if mode == "resident":
            dev.sync_to_host(host)
        runs[mode] = (dts, _interior(geom, host)[..., DEV_VARS].copy())
        dev.close()
    assert runs["resident"][0] == runs["round_trip"][0]
    assert np.array_equal(runs["resident"][1], runs["round_trip"][1])


def test_interior_transfers_with_species_and_slab(need_gpu):
    """Mass fractions ride along; a slab (self-exchanging on its periodic
    axis) maps its stored planes with the halo offset."""
    geom = Geometry(2, 16, 16, 1, 2, 4, 1, bc=(BC_PERIODIC,) * 6)
    hp = HydroParams()
    unk = S.kelvin_helmholtz(geom, hp)
    spec = S.species_blob(geom, ns=2, nspecies=2)
    full0 = np.ascontiguousarray(np.concatenate([unk, spec], axis=-1))
    dec = SlabDecomposition(geom, 1, 0, self_halo=True)
    for kw in ({"species": (2, 2)}, {"slab": dec}):
        u0 = full0 if "species" in kw else unk
        dev = HydroDevice(geom, hp, "fp64", **kw)
        dev.attach_unk(u0.copy())
        dt = 0.5 * dev.Hydro_computeDt()
        dev.Hydro(0.0, dt, dt)
        full = np.zeros(u0.shape)
        dev.sync_to_host(full)
        got = np.zeros(u0.shape)
        dev.get_interior(got)
        vars_ = DEV_VARS + ([NUNK, NUNK + 1] if "species" in kw else [])
        assert np.array_equal(_interior(geom, got)[..., vars_], _interior(geom, full)[..., vars_])
        # put back a changed state and read it again
        _interior(geom, got)[..., DENS] *= 1.5
        dev.put_interior(got)
        back = np.zeros(u0.shape)
        dev.get_interior(back)
        assert np.array_equal(_interior(geom, back)[..., vars_], _interior(geom, got)[..., vars_])
        dev.close()


def test_put_interior_needs_an_attached_unk(need_gpu):
    geom, hp, init = _cases()["kh2d"]
    dev = HydroDevice(geom, hp, "fp64")
    with pytest.raises(FlashXError):
        dev.put_interior(init(geom, hp))
    dev.close()


def test_a_replaced_device_refuses_calls(need_gpu):
    """The library holds one grid: a second HydroDevice replaces the first,
    whose calls then raise instead of acting on the newer grid, and whose
    close leaves the newer grid alone."""
    geom, hp, init = _cases()["kh2d"]
    unk = init(geom, hp)
    a = HydroDevice(geom, hp, "fp64")
    a.attach_unk(unk.copy())
    b = HydroDevice(geom, hp, "fp64")
    b.attach_unk(unk.copy())
    with pytest.raises(FlashXError):
        a.Hydro_computeDt()
    a.close()
    dt = 0.5 * b.Hydro_computeDt()
    b.Hydro(0.0, dt, dt)
    b.close()
    with pytest.raises(FlashXError):
        b.Hydro_computeDt()
