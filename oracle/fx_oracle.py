"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, and only as the checker.  The oracle restates the Flash-X
unsplit-hydro solver in plain C (oracle/fx_oracle.c); its header lists the
reference files it follows.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfx_oracle.so")

NUNK = 11
DENS, EINT, ENER, GAMC, GAME, PRES, SHOK, TEMP, VELX, VELY, VELZ = range(11)
BC_PERIODIC, BC_OUTFLOW, BC_REFLECTING = 0, 1, 2
ROE, LLF, HLL, HLLC, MARQ, MARM, HYBR = 1, 2, 3, 4, 5, 7, 8
LIMITERS = {"minmod": 1, "mc": 2, "vanleer": 3, "hybrid": 4, "limited": 5}


class FxoParams(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int),
        ("nxb", ctypes.c_int), ("nyb", ctypes.c_int), ("nzb", ctypes.c_int),
        ("nblockx", ctypes.c_int), ("nblocky", ctypes.c_int), ("nblockz", ctypes.c_int),
        ("nguard", ctypes.c_int),
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
        ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
        ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
        ("bc", ctypes.c_int * 6),
        ("order", ctypes.c_int), ("weno_method", ctypes.c_int),
        ("riemann", ctypes.c_int), ("limiter", ctypes.c_int),
        ("char_limiting", ctypes.c_int), ("use_3d_full_ctu", ctypes.c_int),
        ("use_aux_eint", ctypes.c_int), ("use_gravity", ctypes.c_int),
        ("grav", ctypes.c_double * 3),
        ("cfl", ctypes.c_double), ("gamma", ctypes.c_double),
        ("eint_switch", ctypes.c_double), ("small_dens", ctypes.c_double),
        ("small_e", ctypes.c_double), ("small_p", ctypes.c_double),
        ("tiny", ctypes.c_double), ("fpres", ctypes.c_double),
        ("limited_beta", ctypes.c_double),
        ("gas_constant", ctypes.c_double), ("abar", ctypes.c_double),
        ("flattening", ctypes.c_int), ("entropy_fix", ctypes.c_int), ("steepening", ctypes.c_int),
        ("use_avisc", ctypes.c_int), ("cvisc", ctypes.c_double),
        ("use_hybrid", ctypes.c_int), ("hybrid_kappa", ctypes.c_double),
        ("shock_detect", ctypes.c_int),
    ]


_lib = None


def build():
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(FxoParams)
        D = ctypes.POINTER(ctypes.c_double)
        L.fxo_unk_size.argtypes = [P]; L.fxo_unk_size.restype = ctypes.c_long
        L.fxo_fill_guardcells.argtypes = [P, D]
        L.fxo_eos_interior.argtypes = [P, D]
        L.fxo_hydro_step.argtypes = [P, D, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.fxo_hydro_step_spec.argtypes = [P, D, D, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int]
        L.fxo_fill_guardcells_spec.argtypes = [P, D, ctypes.c_int]
        L.fxo_compute_dt.argtypes = [P, D, D]
        L.fxo_driver_dt.argtypes = [ctypes.c_double] * 5
        L.fxo_driver_dt.restype = ctypes.c_double
        L.fxo_integrals.argtypes = [P, D, D]
        L.fxo_riemann.argtypes = [P, ctypes.c_int, D, D, D]
        I = ctypes.POINTER(ctypes.c_int)
        L.fxo_amr_create.argtypes = [P, ctypes.c_int, I, I, I]
        L.fxo_amr_create.restype = ctypes.c_void_p
        L.fxo_amr_free.argtypes = [ctypes.c_void_p]
        L.fxo_amr_info.argtypes = [ctypes.c_void_p, I, I]
        L.fxo_amr_leaf_flags.argtypes = [ctypes.c_void_p, ctypes.c_int, I, I]
        L.fxo_amr_fill_guardcells.argtypes = [ctypes.c_void_p, D]
        L.fxo_amr_hydro_step.argtypes = [ctypes.c_void_p, D, ctypes.c_double, ctypes.c_int]
        L.fxo_amr_compute_dt.argtypes = [ctypes.c_void_p, D, D]
        L.fxo_amr_integrals.argtypes = [ctypes.c_void_p, D, D]
        U8 = ctypes.POINTER(ctypes.c_ubyte)
        L.fxo_amr_hydro_step_roles.argtypes = [ctypes.c_void_p, D, ctypes.c_double, U8, ctypes.c_int]
        L.fxo_amr_compute_dt_roles.argtypes = [ctypes.c_void_p, D, U8, D]
        L.fxo_amr_integrals_roles.argtypes = [ctypes.c_void_p, D, U8, D]
        L.fxo_amr_mark_refine.argtypes = [ctypes.c_void_p, D, ctypes.c_int, I, D, D, D, ctypes.c_int, I, D]
        L.fxo_amr_regrid.argtypes = [ctypes.c_void_p, D, ctypes.c_void_p, D]
        _lib = L
    return _lib


def make_params(geom, hp):
    """Build the C parameter struct from a geometry dict and a hydro-parameter
    object exposing the Flash-X runtime-parameter names (see
    flashx_b200.params.HydroParams)."""
    p = FxoParams()
    p.ndim = geom["ndim"]
    p.nxb, p.nyb, p.nzb = geom["nxb"], geom["nyb"], geom["nzb"]
    p.nblockx, p.nblocky, p.nblockz = geom["nblockx"], geom["nblocky"], geom["nblockz"]
    p.nguard = geom.get("nguard", 4)
    (p.xmin, p.xmax), (p.ymin, p.ymax), (p.zmin, p.zmax) = geom["bbox"]
    for i, b in enumerate(geom["bc"]):
        p.bc[i] = b
    p.order = hp.order
    p.weno_method = 2 if hp.wenoMethod.upper() == "WENOZ" else 1
    p.riemann = {"HLLC": HLLC, "HLL": HLL, "LLF": LLF, "ROE": ROE, "MARQUINA": MARQ,
                 "MARQUINAMODIFIED": MARM, "HYBRID": HYBR}[hp.RiemannSolver.upper()]
    p.limiter = LIMITERS[hp.slopeLimiter.lower()]
    p.char_limiting = int(hp.charLimiting)
    p.use_3d_full_ctu = int(hp.use_3dFullCTU)
    p.use_aux_eint = int(hp.use_auxEintEqn)
    p.use_gravity = int(hp.useGravity)
    for i in range(3):
        p.grav[i] = hp.gravity[i]
    p.cfl, p.gamma = hp.cfl, hp.gamma
    p.eint_switch, p.small_dens, p.small_e, p.small_p = hp.eintSwitch, hp.smlrho, hp.smalle, hp.smallp
    p.tiny, p.fpres, p.limited_beta = hp.tiny, hp.hy_fPresInMomFlux, hp.LimitedSlopeBeta
    p.gas_constant, p.abar = hp.gasConstant, hp.eos_singleSpeciesA
    p.flattening = int(hp.use_flattening)
    p.entropy_fix = 0 if not hp.entropy else (1 if hp.entropyFixMethod.upper() == "HARTENHYMAN" else 2)
    p.steepening = int(hp.use_steepening)
    p.use_avisc = int(hp.use_avisc)
    p.cvisc = hp.cvisc
    p.use_hybrid = int(hp.use_hybridOrder)
    p.hybrid_kappa = hp.hybridOrderKappa
    p.shock_detect = int(getattr(hp, "shock_detect", False))
    return p


def _dp(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fill_guardcells(p, unk):
    lib().fxo_fill_guardcells(ctypes.byref(p), _dp(unk))


def eos_interior(p, unk):
    lib().fxo_eos_interior(ctypes.byref(p), _dp(unk))


def hydro_step(p, unk, dt, dt_old, nthreads=0, spec=None, nspecies=None):
    """One unsplit step; `spec` (blk, k, j, i, ns) advects ns mass fractions
    with it, the first `nspecies` (default all) renormalised as species."""
    if spec is None:
        rc = lib().fxo_hydro_step(ctypes.byref(p), _dp(unk), dt, dt_old, nthreads)
    else:
        ns = spec.shape[-1]
        nsp = ns if nspecies is None else nspecies
        rc = lib().fxo_hydro_step_spec(ctypes.byref(p), _dp(unk), _dp(spec), ns, nsp, dt, dt_old, nthreads)
    if rc:
        raise RuntimeError(f"oracle hydro step failed with code {rc}")


def fill_guardcells_spec(p, spec):
    lib().fxo_fill_guardcells_spec(ctypes.byref(p), _dp(spec), spec.shape[-1])


def compute_dt(p, unk):
    out = ctypes.c_double()
    rc = lib().fxo_compute_dt(ctypes.byref(p), _dp(unk), ctypes.byref(out))
    if rc:
        raise RuntimeError("oracle: computed dt is not positive")
    return out.value


def driver_dt(dt_cfl, dt_old, factor=2.0, dtmin=1e-10, dtmax=1e5):
    return lib().fxo_driver_dt(dt_cfl, dt_old, factor, dtmin, dtmax)


def integrals(p, unk):
    out = np.zeros(7)
    lib().fxo_integrals(ctypes.byref(p), _dp(unk), _dp(out))
    return out


def riemann(p, direction, VL, VR):
    """Flux of one Riemann problem; VL/VR = dens velx vely velz pres gamc game eint."""
    vl = np.ascontiguousarray(VL, dtype=np.float64)
    vr = np.ascontiguousarray(VR, dtype=np.float64)
    F = np.zeros(8)
    rc = lib().fxo_riemann(ctypes.byref(p), direction, _dp(vl), _dp(vr), _dp(F))
    if rc:
        raise RuntimeError("Riemann solver ierr")
    return F


class Amr:
    """Oracle of the block-structured AMR step (fx_oracle_amr.inc).  `levels`
    and `bcoords` list the leaves (level from 1, block coordinates at that
    level); leaf UNK arrays are (nleaf, k, j, i, var) with guard cells."""

    ERRORS = {1: "bad geometry", 2: "level or coordinate out of range", 3: "overlapping leaves",
              4: "incomplete tree", 5: "not 2:1 balanced"}

    def __init__(self, p, levels, bcoords):
        self.p = p
        lv = np.ascontiguousarray(levels, dtype=np.int32)
        bc = np.ascontiguousarray(bcoords, dtype=np.int32).reshape(-1, 3)
        err = ctypes.c_int()
        I = ctypes.POINTER(ctypes.c_int)
        self.h = lib().fxo_amr_create(ctypes.byref(p), len(lv), lv.ctypes.data_as(I),
                                      bc.ctypes.data_as(I), ctypes.byref(err))
        if not self.h:
            raise ValueError(f"oracle AMR tree rejected: {self.ERRORS.get(err.value, err.value)}")
        self.nleaf = len(lv)

    def close(self):
        if self.h:
            lib().fxo_amr_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        nb, ml = ctypes.c_int(), ctypes.c_int()
        lib().fxo_amr_info(self.h, ctypes.byref(nb), ctypes.byref(ml))
        return nb.value, ml.value

    def leaf_flags(self, leaf):
        fin = (ctypes.c_int * 6)()
        eos = (ctypes.c_int * 27)()
        lib().fxo_amr_leaf_flags(self.h, leaf, fin, eos)
        return list(fin), list(eos)

    def fill_guardcells(self, unk):
        rc = lib().fxo_amr_fill_guardcells(self.h, _dp(unk))
        if rc:
            raise RuntimeError(f"oracle AMR guard fill failed with code {rc}")

    @staticmethod
    def _roles(roles):
        if roles is None:
            return None
        r = np.ascontiguousarray(roles, dtype=np.uint8)
        return r, r.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))

    def hydro_step(self, unk, dt, nthreads=0, roles=None):
        """The AMR step; with `roles` (per leaf: 1 owned, 2 flux ghost, 0
        not stepped) one rank's share of a mesh split over ranks."""
        if roles is None:
            rc = lib().fxo_amr_hydro_step(self.h, _dp(unk), dt, nthreads)
        else:
            keep, rp = self._roles(roles)
            rc = lib().fxo_amr_hydro_step_roles(self.h, _dp(unk), dt, rp, nthreads)
        if rc:
            raise RuntimeError(f"oracle AMR hydro step failed with code {rc}")

    def compute_dt(self, unk, roles=None):
        out = ctypes.c_double()
        if roles is None:
            rc = lib().fxo_amr_compute_dt(self.h, _dp(unk), ctypes.byref(out))
        else:
            keep, rp = self._roles(roles)
            rc = lib().fxo_amr_compute_dt_roles(self.h, _dp(unk), rp, ctypes.byref(out))
        if rc:
            raise RuntimeError("oracle: computed dt is not positive")
        return out.value

    def mark_refine_derefine(self, unk, refine_vars, max_refine):
        """Grid_markRefineDerefine on the leaves.  refine_vars: (UNK index,
        refine_cutoff, derefine_cutoff, refine_filter) per refinement variable.
        Returns (flags, errors): 1 refine, -1 derefine, 0 neither; the error
        estimate of the last variable per leaf."""
        nv = len(refine_vars)
        iv = (ctypes.c_int * nv)(*[int(r[0]) for r in refine_vars])
        rc_ = (ctypes.c_double * nv)(*[float(r[1]) for r in refine_vars])
        dc = (ctypes.c_double * nv)(*[float(r[2]) for r in refine_vars])
        fl = (ctypes.c_double * nv)(*[float(r[3]) for r in refine_vars])
        flags = np.zeros(self.nleaf, dtype=np.int32)
        err = np.zeros(self.nleaf)
        I = ctypes.POINTER(ctypes.c_int)
        rc = lib().fxo_amr_mark_refine(self.h, _dp(unk), nv, iv, rc_, dc, fl, int(max_refine),
                                       flags.ctypes.data_as(I), _dp(err))
        if rc:
            raise RuntimeError(f"oracle AMR refinement marking failed with code {rc}")
        return flags, err

    def integrals(self, unk, roles=None):
        out = np.zeros(7)
        if roles is None:
            lib().fxo_amr_integrals(self.h, _dp(unk), _dp(out))
        else:
            keep, rp = self._roles(roles)
            lib().fxo_amr_integrals_roles(self.h, _dp(unk), rp, _dp(out))
        return out

    def regrid(self, unk, new):
        """Data of the leaves of `new` (an Amr of the updated tree) from this
        tree's leaf UNK: Grid_updateRefinement's restriction, copies,
        prolongation of new children and Eos.  Returns the new leaf UNK."""
        out = np.zeros((new.nleaf,) + unk.shape[1:])
        rc = lib().fxo_amr_regrid(self.h, _dp(np.ascontiguousarray(unk)), new.h, _dp(out))
        if rc:
            raise RuntimeError({6: "oracle regrid: stencil cell without a block",
                                7: "oracle regrid: a new block's parent was not a leaf"}.get(rc, f"oracle regrid {rc}"))
        return out
