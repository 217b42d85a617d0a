"""Host-side mirror of the Flash-X hydro interface over libflashx_b200.so.

The reference's Fortran driver calls Hydro(simTime, dt, dtOld) once per step
(FX/physics/Hydro/Hydro_interface.F90, impl unsplit/levelFlux/Hydro.F90:20),
Hydro_computeDt per leaf block from Driver_computeDt (unsplit/
Hydro_computeDt.F90:28-34, reduced by MPI_AllReduce MIN in
Driver/DriverMain/Driver_computeDt.F90:373,383) and Grid_fillGuardCells before
any stencil use (Grid/Grid_fillGuardCells.F90:283).  `HydroDevice` exposes the
same three operations with the same argument meaning; the work runs in the
CUDA library (ctypes, plain C ABI).  There is no CPU fallback: if the library
or a GPU is missing every call raises.
"""
import ctypes
import functools
import os

import numpy as np

from .params import Geometry, HydroParams, NUNK, UNK_VARS

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(HERE, "..", "libflashx_b200.so"))
BUILD_DIR = os.path.normpath(os.path.join(HERE, ".."))

FXB_OK, FXB_EARG, FXB_ECUDA, FXB_ESOUND, FXB_ERIEMANN, FXB_EDT, FXB_EUNSUPPORTED, FXB_ETIMEOUT = range(8)
FXB_FP64, FXB_MIXED = 0, 1
# enum fxb_var order of include/flashx_b200.h
FXB_VARS = ("dens", "eint", "ener", "gamc", "game", "pres", "temp", "velx", "vely", "velz")

# variable order of an AMR leaf message (fxb_amr_pack_leaves / fxb_amr_unpack_leaves)
LEAF_MSG_VARS = ("dens", "velx", "vely", "velz", "pres", "gamc", "game", "eint", "ener", "temp")

# entry points declared in include/flashx_b200.h
ABI_SYMBOLS = ("fxb_init", "fxb_register_blocks", "fxb_attach_unk", "fxb_fill_guardcells",
               "fxb_hydro_step", "fxb_compute_dt", "fxb_advance", "fxb_eos", "fxb_sync_to_host",
               "fxb_sync_from_host", "fxb_put_interior", "fxb_get_interior", "fxb_integrals", "fxb_integrals_noalloc", "fxb_mark_refine_derefine",
               "fxb_last_timing", "fxb_stream", "fxb_tuning", "fxb_last_error", "fxb_finalize",
               "fxb_init_slab", "fxb_halo_doubles", "fxb_halo_pack", "fxb_halo_unpack", "fxb_regrid",
               "fxb_refine_derefine", "fxb_counters", "fxb_init_species", "fxb_amr_set_roles",
               "fxb_amr_leaf_doubles", "fxb_amr_pack_leaves", "fxb_amr_unpack_leaves")
# fxb_counters slots
COUNT_STEPS, COUNT_DT_DEVICE, COUNT_DT_CACHED, COUNT_GC_FILLS, COUNT_GC_DOUBLES = range(5)


class FxbParams(ctypes.Structure):
    _fields_ = [
        ("order", ctypes.c_int), ("weno_method", ctypes.c_int), ("riemann", ctypes.c_int),
        ("limiter", ctypes.c_int), ("char_limiting", ctypes.c_int), ("use_3d_full_ctu", ctypes.c_int),
        ("use_aux_eint", ctypes.c_int), ("use_gravity", ctypes.c_int),
        ("grav", ctypes.c_double * 3),
        ("cfl", ctypes.c_double), ("gamma", ctypes.c_double), ("eint_switch", ctypes.c_double),
        ("small_dens", ctypes.c_double), ("small_e", ctypes.c_double), ("small_p", ctypes.c_double),
        ("tiny", ctypes.c_double), ("fpres", ctypes.c_double), ("limited_beta", ctypes.c_double),
        ("gas_constant", ctypes.c_double), ("abar", ctypes.c_double),
        ("precision", ctypes.c_int), ("flattening", ctypes.c_int), ("entropy_fix", ctypes.c_int),
        ("steepening", ctypes.c_int), ("use_avisc", ctypes.c_int), ("cvisc", ctypes.c_double),
        ("upwind_tvd", ctypes.c_int), ("hybrid_order", ctypes.c_int), ("hybrid_kappa", ctypes.c_double),
        ("shock_detect", ctypes.c_int), ("shock_slot", ctypes.c_int),
    ]


class FxbDomain(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int), ("nxb", ctypes.c_int), ("nyb", ctypes.c_int), ("nzb", ctypes.c_int),
        ("nguard", ctypes.c_int), ("nblockx", ctypes.c_int), ("nblocky", ctypes.c_int),
        ("nblockz", ctypes.c_int), ("bbox", (ctypes.c_double * 2) * 3), ("bc", ctypes.c_int * 6),
    ]


class FxbBlockDesc(ctypes.Structure):
    _fields_ = [("level", ctypes.c_int), ("bcoord", ctypes.c_int * 3)]


class FxbSlab(ctypes.Structure):
    _fields_ = [("layer_lo", ctypes.c_int), ("layer_hi", ctypes.c_int),
                ("halo_lo", ctypes.c_int), ("halo_hi", ctypes.c_int)]


class FxbError(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int), ("message", ctypes.c_char * 256)]


class FlashXError(RuntimeError):
    """Raised where the reference would call Driver_abort."""

    def __init__(self, code, message):
        super().__init__(f"[flashx_b200 error {code}] {message}")
        self.code = code


_lib = None


def load_library(path=LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FlashXError(FXB_ECUDA, f"{path} not found: build it with `make -C {BUILD_DIR}`")
    L = ctypes.CDLL(path)
    D = ctypes.POINTER(ctypes.c_double)
    I32 = ctypes.POINTER(ctypes.c_int32)
    L.fxb_init.argtypes = [ctypes.POINTER(FxbParams), ctypes.POINTER(FxbDomain), I32, ctypes.c_int]
    L.fxb_register_blocks.argtypes = [ctypes.POINTER(FxbBlockDesc), ctypes.c_int]
    L.fxb_attach_unk.argtypes = [D]
    L.fxb_fill_guardcells.argtypes = [ctypes.c_int, ctypes.c_int, D]
    L.fxb_counters.argtypes = [ctypes.POINTER(ctypes.c_longlong)]
    L.fxb_init_species.argtypes = [ctypes.c_int, ctypes.c_int, I32]
    L.fxb_amr_set_roles.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.fxb_amr_leaf_doubles.argtypes = []
    L.fxb_amr_leaf_doubles.restype = ctypes.c_long
    L.fxb_amr_pack_leaves.argtypes = [I32, ctypes.c_int, ctypes.c_void_p]
    L.fxb_amr_unpack_leaves.argtypes = [I32, ctypes.c_int, ctypes.c_void_p]
    L.fxb_hydro_step.argtypes = [ctypes.c_double] * 3
    L.fxb_compute_dt.argtypes = [D, I32]
    L.fxb_advance.argtypes = [ctypes.c_int, D, D, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.fxb_eos.argtypes = []
    L.fxb_sync_to_host.argtypes = [D]
    L.fxb_sync_from_host.argtypes = [D]
    L.fxb_put_interior.argtypes = [D]
    L.fxb_get_interior.argtypes = [D]
    L.fxb_integrals.argtypes = [D]
    L.fxb_integrals_noalloc.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_long, ctypes.c_double,
                                                                 ctypes.c_void_p, ctypes.c_void_p]
    L.fxb_last_timing.argtypes = [D, ctypes.POINTER(ctypes.c_int)]
    L.fxb_tuning.argtypes = [ctypes.c_char_p, ctypes.c_int]
    L.fxb_stream.restype = ctypes.c_void_p
    L.fxb_last_error.argtypes = [ctypes.POINTER(FxbError)]
    L.fxb_finalize.restype = None
    L.fxb_init_slab.argtypes = L.fxb_init.argtypes + [ctypes.POINTER(FxbSlab)]
    L.fxb_halo_doubles.argtypes = [ctypes.c_int]
    L.fxb_halo_doubles.restype = ctypes.c_long
    L.fxb_halo_pack.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    L.fxb_halo_unpack.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.fxb_regrid.argtypes = [ctypes.POINTER(FxbBlockDesc), ctypes.c_int]
    L.fxb_refine_derefine.argtypes = [ctypes.POINTER(FxbDomain), ctypes.POINTER(FxbBlockDesc), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(FxbBlockDesc), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    for name in ABI_SYMBOLS:
        if name not in ("fxb_stream", "fxb_finalize", "fxb_halo_doubles", "fxb_amr_leaf_doubles"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def _check(rc):
    if rc != FXB_OK:
        err = FxbError()
        _lib.fxb_last_error(ctypes.byref(err))
        raise FlashXError(rc, err.message.decode(errors="replace"))


def _dp(a):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("UNK must be a C-contiguous float64 array (Fortran unk(var,i,j,k,blk))")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_fxb_params(hp: HydroParams, precision="fp64"):
    hp.validate()
    p = FxbParams()
    p.order = hp.order
    p.weno_method = 2 if hp.wenoMethod.upper() == "WENOZ" else 1
    p.riemann = {"HLLC": 4, "HLL": 3, "LLF": 2, "ROE": 1, "MARQUINA": 5,
                 "MARQUINAMODIFIED": 7, "HYBRID": 8}[hp.RiemannSolver.upper()]
    p.limiter = {"minmod": 1, "mc": 2, "vanleer": 3, "hybrid": 4, "limited": 5}[hp.slopeLimiter.lower()]
    p.char_limiting = int(hp.charLimiting)
    p.use_3d_full_ctu = int(hp.use_3dFullCTU)
    p.use_aux_eint = int(hp.use_auxEintEqn)
    p.use_gravity = int(hp.useGravity)
    for i in range(3):
        p.grav[i] = hp.gravity[i]
    p.cfl, p.gamma, p.eint_switch = hp.cfl, hp.gamma, hp.eintSwitch
    p.small_dens, p.small_e, p.small_p, p.tiny = hp.smlrho, hp.smalle, hp.smallp, hp.tiny
    p.fpres, p.limited_beta = hp.hy_fPresInMomFlux, hp.LimitedSlopeBeta
    p.gas_constant, p.abar = hp.gasConstant, hp.eos_singleSpeciesA
    p.precision = {"fp64": FXB_FP64, "mixed": FXB_MIXED}[precision]
    p.flattening = int(hp.use_flattening)
    p.entropy_fix = 0 if not hp.entropy else (1 if hp.entropyFixMethod.upper() == "HARTENHYMAN" else 2)
    p.steepening = int(hp.use_steepening)
    p.use_avisc = int(hp.use_avisc)
    p.cvisc = hp.cvisc
    p.upwind_tvd = int(hp.use_upwindTVD)
    p.hybrid_order = int(hp.use_hybridOrder)
    p.hybrid_kappa = hp.hybridOrderKappa
    p.shock_detect = int(hp.shock_detect)
    p.shock_slot = UNK_VARS.index("shok") if hp.shock_detect else -1
    return p


def make_fxb_domain(geom: Geometry):
    d = FxbDomain()
    d.ndim, d.nxb, d.nyb, d.nzb, d.nguard = geom.ndim, geom.nxb, geom.nyb, geom.nzb, geom.nguard
    d.nblockx, d.nblocky, d.nblockz = geom.nblockx, geom.nblocky, geom.nblockz
    for a in range(3):
        d.bbox[a][0], d.bbox[a][1] = geom.bbox[a]
    for i in range(6):
        d.bc[i] = geom.bc[i]
    return d


def default_var_map():
    """0-based UNK slots (Simulation.h *_VAR - 1) of the UHD + Gamma setup."""
    vm = (ctypes.c_int32 * len(FXB_VARS))()
    for i, name in enumerate(FXB_VARS):
        vm[i] = UNK_VARS.index(name)
    return vm


def leaf_blocks(geom: Geometry, layers=None):
    """Leaf-block list of a uniform block grid in Flash-X block order; with
    `layers` = (lo, hi) only the blocks of those layers of the slowest axis."""
    ny = geom.nblocky if geom.ndim >= 2 else 1
    nz = geom.nblockz if geom.ndim == 3 else 1
    ys, zs = range(ny), range(nz)
    if layers is not None:
        if geom.ndim == 2:
            ys = range(*layers)
        else:
            zs = range(*layers)
    n = geom.nblockx * len(ys) * len(zs)
    arr = (FxbBlockDesc * n)()
    b = 0
    for bz in zs:
        for by in ys:
            for bx in range(geom.nblockx):
                arr[b].level = 1
                arr[b].bcoord[0], arr[b].bcoord[1], arr[b].bcoord[2] = bx, by, bz
                b += 1
    return arr


def amr_leaf_message(geom: Geometry, unk, leaves):
    """The message fxb_amr_pack_leaves makes of `leaves` of a host UNK (an
    AmrMesh UNK, default variable map): per leaf the interior cells of the
    variables LEAF_MSG_VARS, [leaf][var][k][j][i]."""
    g = geom.nguard
    sl = [slice(g, g + n) if n > 1 else slice(0, 1) for n in (geom.nzb, geom.nyb, geom.nxb)]
    slots = [UNK_VARS.index(v) for v in LEAF_MSG_VARS]
    sub = unk[np.asarray(leaves, dtype=np.int64)][:, sl[0], sl[1], sl[2]][..., slots]
    return np.ascontiguousarray(np.moveaxis(sub, -1, 1)).reshape(-1)


def mesh_blocks(levels, bcoords):
    """Leaf-block list of an AMR mesh (levels from 1, block coordinates at
    each leaf's level), in UNK slot order."""
    n = len(levels)
    arr = (FxbBlockDesc * n)()
    for b in range(n):
        arr[b].level = int(levels[b])
        arr[b].bcoord[0], arr[b].bcoord[1], arr[b].bcoord[2] = (int(v) for v in bcoords[b])
    return arr


def refine_derefine(mesh, flags, lrefine_min=1, lrefine_max=None):
    """PARAMESH's tree update in the library (fxb_refine_derefine, host
    code): the new AmrMesh of `mesh` for leaf marks `flags` (mesh order)."""
    from .amr import AmrMesh
    lib = load_library()
    lmax = lrefine_max if lrefine_max is not None else mesh.maxlev + 1
    blocks = mesh_blocks(mesh.levels, mesh.bcoords)
    fl = (ctypes.c_int * mesh.nleaf)(*[int(f) for f in flags])
    cap = mesh.nleaf * (8 if mesh.geom.ndim == 3 else 4)
    out = (FxbBlockDesc * cap)()
    n = ctypes.c_int()
    d = make_fxb_domain(mesh.geom)
    _check(lib.fxb_refine_derefine(ctypes.byref(d), blocks, mesh.nleaf, fl, int(lrefine_min), int(lmax), out, cap,
                                   ctypes.byref(n)))
    return AmrMesh(mesh.geom, [(out[i].level, (out[i].bcoord[0], out[i].bcoord[1], out[i].bcoord[2]))
                               for i in range(n.value)])


class HydroDevice:
    """The unsplit hydro solver on one B200, behind the reference interface.

    `mesh` (a flashx_b200.amr.AmrMesh over `geom`'s root blocks) selects a
    block-structured AMR mesh; without it the blocks form the uniform grid.
    `slab` (a flashx_b200.parallel.SlabDecomposition of `geom`) makes this
    device one rank's slab of the uniform grid: it holds that rank's blocks
    (UNK slots in the grid's block order) and exchanges halos with the
    neighbouring ranks before each step and before guard cells go to the
    host; Hydro_computeDt and integrals cover the rank's own cells, for the
    caller to reduce over ranks.
    `amr_split` (a flashx_b200.parallel.AmrDecomposition of `mesh`) makes it
    one rank's share of an AMR mesh: the device holds the whole mesh, the
    host UNK the rank's own leaves (unk_shape); it steps its own leaves (and
    computes the fluxes of its flux ghosts) and receives the other ranks'
    leaves its guard fills read before each step and before guard cells go
    to the host; Hydro_computeDt and integrals cover its own leaves."""

    def __init__(self, geom: Geometry, hp: HydroParams, precision="fp64", mesh=None, slab=None, species=None,
                 amr_split=None):
        """species = (nspec, nspecies): that many advected mass fractions in
        UNK slots NUNK .. NUNK + nspec - 1 after the hydro variables (the
        first nspecies renormalised as species, the rest mass scalars)."""
        global _active
        self.lib = load_library()
        # the library holds one grid: this device replaces any earlier one
        self._token = _active = object()
        self.geom, self.hp, self.precision, self.mesh, self.slab = geom, hp, precision, mesh, slab
        nspec = species[0] if species else 0
        self.nunk = NUNK + nspec
        self._p = make_fxb_params(hp, precision)
        self._d = make_fxb_domain(geom)
        self._vm = default_var_map()
        self.exchange = None
        if slab is not None:
            if mesh is not None:
                raise ValueError("a slab splits a uniform grid, not an AMR mesh")
            self._s = FxbSlab(slab.layer_lo, slab.layer_hi, slab.halo_lo, slab.halo_hi)
            _check(self.lib.fxb_init_slab(ctypes.byref(self._p), ctypes.byref(self._d), self._vm, self.nunk,
                                          ctypes.byref(self._s)))
        else:
            _check(self.lib.fxb_init(ctypes.byref(self._p), ctypes.byref(self._d), self._vm, self.nunk))
        if nspec:
            slots = (ctypes.c_int32 * nspec)(*range(NUNK, NUNK + nspec))
            _check(self.lib.fxb_init_species(nspec, int(species[1]), slots))
        if slab is not None:
            b0, b1 = slab.block_range()
            blocks, n = leaf_blocks(geom, (slab.layer_lo, slab.layer_hi)), b1 - b0
            self.unk_shape = (n,) + geom.block_shape[:-1] + (self.nunk,)
            if slab.halo_lo or slab.halo_hi:
                self.exchange = self._make_exchange(slab)
        elif mesh is None:
            blocks, n = leaf_blocks(geom), geom.nblocks
            self.unk_shape = geom.unk_shape[:-1] + (self.nunk,)
        else:
            blocks, n = mesh_blocks(mesh.levels, mesh.bcoords), mesh.nleaf
            self.unk_shape = mesh.unk_shape
        _check(self.lib.fxb_register_blocks(blocks, n))
        self.unk = None
        self.split = None
        if amr_split is not None:
            if mesh is None or amr_split.mesh is not mesh:
                raise ValueError("amr_split must decompose the mesh given")
            self._set_split(amr_split)

    def _set_split(self, dec):
        roles = np.ascontiguousarray(dec.roles, dtype=np.uint8)
        _check(self.lib.fxb_amr_set_roles(roles.ctypes.data, len(roles)))
        self.split = dec
        self.unk_shape = (len(dec.owned()),) + dec.mesh.unk_shape[1:]
        self.exchange = self._make_amr_exchange(dec) if dec.world > 1 else None

    def _make_amr_exchange(self, dec):
        import torch
        from .parallel import AmrExchange
        lib = self.lib
        lists = {}

        def i32(leaves):
            key = id(leaves)
            if key not in lists:
                lists[key] = (leaves, np.ascontiguousarray(leaves, dtype=np.int32))
            a = lists[key][1]
            return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(a)

        def pack(leaves, buf):
            p, n = i32(leaves)
            _check(lib.fxb_amr_pack_leaves(p, n, ctypes.c_void_p(buf.data_ptr())))

        def unpack(leaves, buf):
            p, n = i32(leaves)
            _check(lib.fxb_amr_unpack_leaves(p, n, ctypes.c_void_p(buf.data_ptr())))

        import torch.distributed as dist
        dev = torch.device("cuda", torch.cuda.current_device())
        stream = torch.cuda.ExternalStream(lib.fxb_stream(), device=dev)
        host = dist.is_initialized() and dist.get_backend() != "nccl"     # e.g. gloo: messages via pinned host copies
        return AmrExchange(dec, lib.fxb_amr_leaf_doubles(), pack, unpack, device=dev, stream=stream, host_stage=host)

    def unpack_leaves(self, leaves, buf):
        """fxb_amr_unpack_leaves: store the interiors in the message `buf` (a
        float64 CUDA tensor laid out as amr_leaf_message) into `leaves`."""
        a = np.ascontiguousarray(leaves, dtype=np.int32)
        _check(self.lib.fxb_amr_unpack_leaves(a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(a),
                                              ctypes.c_void_p(buf.data_ptr())))

    def pack_leaves(self, leaves, buf):
        """fxb_amr_pack_leaves: the interiors of `leaves` into the message `buf`."""
        a = np.ascontiguousarray(leaves, dtype=np.int32)
        _check(self.lib.fxb_amr_pack_leaves(a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(a),
                                            ctypes.c_void_p(buf.data_ptr())))

    def _make_exchange(self, slab):
        import torch
        from .parallel import HaloExchange
        lib = self.lib
        ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())

        def pack(send_lo, n_lo, send_hi, n_hi):
            _check(lib.fxb_halo_pack(ptr(send_lo), n_lo, ptr(send_hi), n_hi))

        def unpack(recv_lo, recv_hi):
            _check(lib.fxb_halo_unpack(ptr(recv_lo), ptr(recv_hi)))

        import torch.distributed as dist
        dev = torch.device("cuda", torch.cuda.current_device())
        stream = torch.cuda.ExternalStream(lib.fxb_stream(), device=dev)
        host = dist.is_initialized() and dist.get_backend() != "nccl"     # e.g. gloo: planes via pinned host copies
        return HaloExchange(slab, lib.fxb_halo_doubles(1), pack, unpack, device=dev, stream=stream, host_stage=host)

    def fill_halos(self):
        """Grid_fillGuardCells between ranks: the halo planes from the
        neighbouring slabs, or the other ranks' leaves this rank's guard
        fills read (every rank calls it at the same point)."""
        if self.exchange is not None:
            self.exchange()

    # ---- data movement
    def attach_unk(self, unk):
        """Take the host UNK (Fortran unk(var,i,j,k,blk) as a C-order array)."""
        if unk.shape != self.unk_shape:
            raise ValueError(f"UNK shape {unk.shape} != {self.unk_shape}")
        self.unk = unk
        _check(self.lib.fxb_attach_unk(_dp(unk)))

    def sync_to_host(self, unk=None):
        unk = self.unk if unk is None else unk
        if unk is None or unk.shape != self.unk_shape:
            raise ValueError(f"sync_to_host needs a UNK of shape {self.unk_shape}")
        self.fill_halos()
        _check(self.lib.fxb_sync_to_host(_dp(unk)))
        return unk

    def put_interior(self, unk=None):
        """Replace the device state's block interiors with the host UNK's
        (fxb_put_interior: the hydro variables and mass fractions only)."""
        unk = self.unk if unk is None else unk
        if unk is None or unk.shape != self.unk_shape:
            raise ValueError(f"put_interior needs a UNK of shape {self.unk_shape}")
        self._mapped = unk          # the library maps this array's pages: keep it alive
        _check(self.lib.fxb_put_interior(_dp(unk)))

    def get_interior(self, unk=None):
        """Write the device state's block interiors into the host UNK
        (fxb_get_interior); its guard cells keep their values, the other
        slots of interior cells get the values last read from the host.
        AMR meshes copy whole blocks (sync_to_host)."""
        unk = self.unk if unk is None else unk
        if unk is None or unk.shape != self.unk_shape:
            raise ValueError(f"get_interior needs a UNK of shape {self.unk_shape}")
        if self.mesh is not None:
            return self.sync_to_host(unk)
        self._mapped = unk
        _check(self.lib.fxb_get_interior(_dp(unk)))
        return unk

    # ---- the reference interface
    def Grid_fillGuardCells(self, unk=None, mask=None, doEos=True):
        """Fill the guard cells (and interiors) of the host UNK from the device.
        mask: names of the variables to fill (Grid_fillGuardCells' mask;
        None = all); only those cross PCIe and are written.  doEos: Eos on
        the guard regions next to other refinement levels (AMR meshes; the
        uniform grid ignores it, as UG's Grid_fillGuardCells does)."""
        unk = self.unk if unk is None else unk
        if unk is None or unk.shape != self.unk_shape:
            raise ValueError(f"Grid_fillGuardCells needs a UNK of shape {self.unk_shape}")
        bits = 0
        for name in (mask or ()):
            bits |= 1 << FXB_VARS.index(name)
        self.fill_halos()
        _check(self.lib.fxb_fill_guardcells(bits, int(bool(doEos)), _dp(unk)))
        return unk

    def Hydro(self, simTime, dt, dtOld):
        self.fill_halos()
        _check(self.lib.fxb_hydro_step(float(simTime), float(dt), float(dtOld)))

    def Hydro_computeDt(self, location=False):
        """Global CFL time step of the current state (min over blocks).  With
        location=True also the limiting cell as Flash-X's dtMinLoc: i, j, k
        (1-based, guard cells counted), refinement level, 1-based block."""
        out = ctypes.c_double()
        loc = (ctypes.c_int32 * 5)() if location else None
        _check(self.lib.fxb_compute_dt(ctypes.byref(out), loc))
        return (out.value, list(loc)) if location else out.value

    def Eos_wrapped(self):
        _check(self.lib.fxb_eos())

    # ---- driver helpers
    def advance(self, nsteps, dt, dt_old):
        """nsteps of Hydro + Driver_computeDt on the device (CUDA graph); a
        slab with halos or a split AMR mesh steps from the host instead,
        exchanging halos or leaves and reducing dt over the ranks every step."""
        hp = self.hp
        if self.exchange is not None:
            from .parallel import allreduce_min
            for _ in range(nsteps):
                self.Hydro(0.0, dt, dt_old)
                dt_old, dt = dt, driver_dt(allreduce_min(self.Hydro_computeDt()), dt, hp)
            return dt, dt_old
        a, b = ctypes.c_double(dt), ctypes.c_double(dt_old)
        _check(self.lib.fxb_advance(int(nsteps), ctypes.byref(a), ctypes.byref(b),
                                    hp.tstep_change_factor, hp.dtmin, hp.dtmax))
        return a.value, b.value

    def integrals(self):
        out = np.zeros(7)
        _check(self.lib.fxb_integrals(_dp(out)))
        return out

    def Grid_markRefineDerefine(self, refine_vars, max_refine):
        """Grid_markRefineDerefine on the registered AMR mesh.  refine_vars:
        (variable name, refine_cutoff, derefine_cutoff, refine_filter) per
        refinement variable, names as in UNK ("dens", "pres", ...).
        Returns (flags, errors) per leaf: 1 refine, -1 derefine, 0 neither;
        the error estimate of the last variable.  On a split mesh every rank
        first receives every leaf, so that all ranks mark the same leaves."""
        if self.split is not None and self.exchange is not None:
            self._full_exchange()
        nv = len(refine_vars)
        ids = [FXB_VARS.index(r[0]) for r in refine_vars]
        iv = (ctypes.c_int * nv)(*ids)
        rc_ = (ctypes.c_double * nv)(*[float(r[1]) for r in refine_vars])
        dc = (ctypes.c_double * nv)(*[float(r[2]) for r in refine_vars])
        fl = (ctypes.c_double * nv)(*[float(r[3]) for r in refine_vars])
        n = self.mesh.nleaf if self.mesh is not None else self.unk_shape[0]   # every leaf, split mesh or not
        flags = np.zeros(n, dtype=np.int32)
        err = np.zeros(n)
        _check(self.lib.fxb_mark_refine_derefine(nv, iv, rc_, dc, fl, int(max_refine),
                                                 flags.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(err)))
        return flags, err

    def Grid_updateRefinement(self, flags, lrefine_min=1, lrefine_max=None):
        """Grid_updateRefinement after Grid_markRefineDerefine: the tree update
        (PARAMESH's amr_refine_derefine, fxb_refine_derefine on the host),
        then the data movement on the device (fxb_regrid).  Returns the new
        AmrMesh; the host UNK must then have its shape (`unk_shape`) for
        sync_to_host."""
        if self.mesh is None:
            raise ValueError("Grid_updateRefinement needs an AMR mesh")
        new = refine_derefine(self.mesh, flags, lrefine_min, lrefine_max)
        if self.split is not None:
            # every leaf's data on every rank for the data movement, then the
            # new mesh's Morton split
            from .parallel import AmrDecomposition
            if self.exchange is not None:
                self._full_exchange()
        _check(self.lib.fxb_regrid(mesh_blocks(new.levels, new.bcoords), new.nleaf))
        self.mesh = new
        self.unk_shape = new.unk_shape
        self.unk = None
        if self.split is not None:
            self._set_split(AmrDecomposition(new, self.split.world, self.split.rank, self.split.hops))
        return new

    def _full_exchange(self):
        """Every rank's own leaves to every other rank (before a regrid, whose
        prolongation and restriction read leaves anywhere in the mesh)."""
        import torch
        import torch.distributed as dist
        dec, n = self.split, self.lib.fxb_amr_leaf_doubles()
        dev = torch.device("cuda", torch.cuda.current_device())
        stream = torch.cuda.ExternalStream(self.lib.fxb_stream(), device=dev)
        most = max(dec.bounds[r + 1] - dec.bounds[r] for r in range(dec.world))
        host = dist.get_backend() != "nccl"      # e.g. gloo: through pinned host copies
        with torch.cuda.stream(stream):
            mine = torch.empty(most * n, dtype=torch.float64, device=dev)
            self.pack_leaves(dec.owned(), mine)
            if host:
                mine_h = torch.empty(most * n, dtype=torch.float64, pin_memory=True)
                mine_h.copy_(mine, non_blocking=True)
                stream.synchronize()
                parts_h = [torch.empty(most * n, dtype=torch.float64) for _ in range(dec.world)]
                dist.all_gather(parts_h, mine_h)
                parts = [p.to(dev, non_blocking=False) for p in parts_h]
            else:
                parts = [torch.empty(most * n, dtype=torch.float64, device=dev) for _ in range(dec.world)]
                dist.all_gather(parts, mine)
            for r in range(dec.world):
                if r != dec.rank:
                    self.unpack_leaves(dec.owned(r), parts[r])

    def tuning(self):
        """The launch shape in use (the batched-block path tunes it at attach)."""
        buf = ctypes.create_string_buffer(1024)
        _check(self.lib.fxb_tuning(buf, 1024))
        return buf.value.decode()

    def counters(self):
        """fxb_counters: hydro steps, device and cached Hydro_computeDt calls,
        guard fills to the host and the doubles they moved."""
        c = (ctypes.c_longlong * 5)()
        _check(self.lib.fxb_counters(c))
        return list(c)

    def last_timing(self):
        ms = ctypes.c_double()
        n = ctypes.c_int()
        _check(self.lib.fxb_last_timing(ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def close(self):
        """Release the library's grid (fxb_finalize), unless a newer device
        has replaced this one already."""
        global _active
        if _active is self._token:
            self.lib.fxb_finalize()
            _active = None
        self._mapped = None


_active = None   # token of the HydroDevice whose grid the library holds


def _guarded(fn):
    @functools.wraps(fn)
    def call(self, *args, **kwargs):
        if _active is not self._token:
            raise FlashXError(FXB_EARG, "this HydroDevice was replaced by a newer one or closed "
                                        "(the library holds one grid at a time)")
        return fn(self, *args, **kwargs)
    return call


for _name in ("attach_unk", "sync_to_host", "put_interior", "get_interior", "Grid_fillGuardCells", "Hydro",
              "Hydro_computeDt", "Eos_wrapped", "advance", "integrals", "Grid_markRefineDerefine",
              "Grid_updateRefinement", "unpack_leaves", "pack_leaves", "fill_halos", "tuning", "counters",
              "last_timing"):
    setattr(HydroDevice, _name, _guarded(getattr(HydroDevice, _name)))


def driver_dt(dt_cfl, dt_old, hp: HydroParams):
    """Driver_computeDt.F90:452,460: growth limit, then clamp."""
    dt_new = dt_cfl if dt_cfl < dt_old * hp.tstep_change_factor else dt_old * hp.tstep_change_factor
    dt_new = dt_new if dt_new > hp.dtmin else hp.dtmin
    return dt_new if dt_new < hp.dtmax else hp.dtmax


def initial_dt(dt_cfl, hp: HydroParams):
    """Driver_verifyInitDt.F90:234-250."""
    slow = 0.1
    return slow * dt_cfl if hp.dtinit > slow * dt_cfl else hp.dtinit
