"""Runtime parameters of the unsplit hydro solver, under their Flash-X names.

Defaults are the values the benchmark configurations use: the Config
defaults of FX/physics/Hydro/HydroMain/unsplit/Config:44-50,127-181 and
FX/physics/Hydro/HydroMain/Config:26 (cfl 0.8), overridden where
FX/Simulation/SimulationMain/Sod/flash.par sets them (slopeLimiter "mc",
charLimiting .true., eintSwitch 1e-4), with order 3 (PPM) and HLLC.
"""
from dataclasses import dataclass, field, asdict

# Slot order of Flash-X UNK for UHD + Gamma (alphabetical, bin/unitCfg.py).
UNK_VARS = ("dens", "eint", "ener", "gamc", "game", "pres", "shok", "temp",
            "velx", "vely", "velz")
NUNK = len(UNK_VARS)
DENS, EINT, ENER, GAMC, GAME, PRES, SHOK, TEMP, VELX, VELY, VELZ = range(NUNK)

BC_PERIODIC, BC_OUTFLOW, BC_REFLECTING = 0, 1, 2
BC_NAMES = {"periodic": BC_PERIODIC, "outflow": BC_OUTFLOW, "reflect": BC_REFLECTING,
            "reflecting": BC_REFLECTING}


@dataclass
class HydroParams:
    order: int = 3                      # 2 = MUSCL-Hancock, 3 = PPM, 5 = WENO
    wenoMethod: str = "WENO5"           # WENO5 | WENOZ
    RiemannSolver: str = "HLLC"         # HLLC | HLL | LLF | Roe | Marquina | MarquinaModified | hybrid
    slopeLimiter: str = "mc"            # minmod | mc | vanLeer | hybrid | limited
    LimitedSlopeBeta: float = 1.0
    charLimiting: bool = True
    use_3dFullCTU: bool = True
    use_auxEintEqn: bool = True
    transOrder: int = 1
    use_flattening: bool = False
    entropy: bool = False               # Roe's entropy fix (hy_entropyFix.F90)
    entropyFixMethod: str = "HartenHyman"   # HartenHyman | Harten
    use_steepening: bool = False
    use_upwindTVD: bool = False         # off with NGUARD <= 4 (unsplit/Hydro_init.F90:137)
    use_avisc: bool = False             # artificial viscosity
    cvisc: float = 0.1
    use_hybridOrder: bool = False       # first-order states at shocks
    hybridOrderKappa: float = 0.0
    shockDetect: bool = False           # the strong-shock flag SHOK (hy_shockDetectBlk); on with RiemannSolver hybrid
    shockLowerCFL: bool = False
    hydroComputeDtOption: int = -1
    cfl: float = 0.8
    gamma: float = 1.4
    eintSwitch: float = 1.0e-4
    smlrho: float = 1.0e-10
    smallp: float = 1.0e-10
    smalle: float = 1.0e-10
    tiny: float = 1.0e-16
    hy_fPresInMomFlux: float = 1.0
    gasConstant: float = 8.3144598e7    # PhysicalConstants "ideal gas constant"
    eos_singleSpeciesA: float = 1.0
    useGravity: bool = False
    gravity: tuple = (0.0, 0.0, 0.0)
    # Driver dt control (FX/Driver/DriverMain/Config:76-121)
    dtinit: float = 1.0e-10
    dtmin: float = 1.0e-10
    dtmax: float = 1.0e5
    tstep_change_factor: float = 2.0

    @property
    def shock_detect(self):
        """Hydro_init.F90:117-122, 391-394: the shock detector runs when asked
        for, and always with the hybrid Riemann solver."""
        return bool(self.shockDetect) or self.RiemannSolver.upper() == "HYBRID"

    def validate(self):
        """Reject option combinations this path does not implement, the way
        Hydro_init aborts on unknown choices."""
        if self.order not in (2, 3, 5):
            raise ValueError("order must be 2 (MUSCL-Hancock), 3 (PPM) or 5 (WENO)")
        if self.RiemannSolver.upper() not in ("HLLC", "HLL", "LLF", "ROE", "MARQUINA", "MARQUINAMODIFIED", "HYBRID"):
            raise ValueError("RiemannSolver must be HLLC, HLL, LLF, Roe, Marquina, MarquinaModified or hybrid")
        if self.shockLowerCFL:
            raise ValueError("shockLowerCFL is not implemented")
        if self.slopeLimiter.lower() not in ("minmod", "mc", "vanleer", "hybrid", "limited"):
            raise ValueError("unknown slopeLimiter " + self.slopeLimiter)
        if self.wenoMethod.upper() not in ("WENO5", "WENOZ"):
            raise ValueError("wenoMethod must be WENO5 or WENOZ")
        if self.transOrder != 1:
            raise ValueError("[hy_upwindTransverseFlux]: No high-order transFlux support! Please set transOrder=1.")
        if self.entropyFixMethod.upper() not in ("HARTENHYMAN", "HARTEN"):
            raise ValueError("entropyFixMethod must be HartenHyman or Harten")
        if self.use_flattening and self.useGravity:
            raise ValueError("use_flattening with gravity is not supported by this path")
        if self.hydroComputeDtOption != -1:
            raise ValueError("hydroComputeDtOption must be -1")
        return self

    def as_dict(self):
        return asdict(self)


@dataclass
class Geometry:
    """A uniform grid of equal blocks (Flash-X UG, or PARAMESH at one level)."""
    ndim: int
    nxb: int
    nyb: int
    nzb: int
    nblockx: int
    nblocky: int
    nblockz: int
    bbox: tuple = ((0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    bc: tuple = (BC_OUTFLOW,) * 6
    nguard: int = 4

    @property
    def nblocks(self):
        return self.nblockx * self.nblocky * self.nblockz

    @property
    def ncells(self):
        return self.nblocks * self.nxb * self.nyb * self.nzb

    @property
    def block_shape(self):
        """UNK block shape in C order: (k, j, i, var) with guard cells."""
        g = self.nguard
        nk = self.nzb + 2 * g if self.ndim == 3 else 1
        nj = self.nyb + 2 * g if self.ndim >= 2 else 1
        return (nk, nj, self.nxb + 2 * g, NUNK)

    @property
    def unk_shape(self):
        return (self.nblocks,) + self.block_shape

    def deltas(self):
        (x0, x1), (y0, y1), (z0, z1) = self.bbox
        dx = (x1 - x0) / (self.nxb * self.nblockx)
        dy = (y1 - y0) / (self.nyb * self.nblocky) if self.ndim >= 2 else 1.0
        dz = (z1 - z0) / (self.nzb * self.nblockz) if self.ndim == 3 else 1.0
        return dx, dy, dz

    def as_dict(self):
        return {"ndim": self.ndim, "nxb": self.nxb, "nyb": self.nyb, "nzb": self.nzb,
                "nblockx": self.nblockx, "nblocky": self.nblocky, "nblockz": self.nblockz,
                "bbox": self.bbox, "bc": self.bc, "nguard": self.nguard}
