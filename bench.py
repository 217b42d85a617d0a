#!/usr/bin/env python
"""Benchmark: zone-updates/s of the unsplit hydro step on B200.

Workload (N=1 per GPU): 2-D Kelvin-Helmholtz, 2048^2 cells as 128x128 blocks
of 16^2, periodic, PPM + HLLC, CFL 0.8 (the benchmark's second configuration;
seeded synthetic initial state from flashx_b200.simulations).  A step is one
Hydro() call over the whole grid plus Driver_computeDt: guard resolution,
reconstruction, Riemann solve, conserved update, energyFix, Eos and the CFL
reduction.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is the plain FP64 path (bit-identical
to the oracle); the FP32-reconstruction/FP64-update path is reported under
`mixed` with its L1 density error against the FP64 result.  State arrays
(2 x 10 x 4.2M FP64 = 671 MB) exceed the 126 MB L2, so no flush is needed.
"""
import argparse
import json
import os
import statistics
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "flash-x_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "zone-updates/s FP64 vs FP32+FP64-update at stated L1 err; % HBM roofline"
UNIT = "zone-updates/s"
BYTES_PER_ZONE = 152   # 9 FP64 reads + 10 FP64 writes per zone-update (algorithmic)
FLOPS_FILES = {"kh2d": os.path.join(ROOT, "profiles", "hydro2d_kh2048_flops.json")}
TRAFFIC_FILES = {"kh2d": os.path.join(ROOT, "profiles", "hydro2d_kh2048_traffic.json"),
                 "rt3d": os.path.join(ROOT, "profiles", "hydro3d_rt256_traffic.json"),
                 "amr3d": os.path.join(ROOT, "profiles", "amr_step_amr3d5230_traffic.json")}
WORKLOADS = {
    "kh2d": "kh2d: 2-D Kelvin-Helmholtz 2048^2 (128x128 blocks of 16^2), periodic, PPM+HLLC, "
            "mc/char limiting, CFL 0.8, gamma 1.4",
    "sod2d": "sod2d: 2-D Sod at 45 deg, 256^2 (16x16 blocks of 16^2), outflow, PPM+HLLC, CFL 0.8",
    "rt3d": "rt3d: 3-D Rayleigh-Taylor 256^3 (4096 blocks of 16^3), WENO5+HLLC, g_z=-0.1, periodic x/y, "
            "reflecting z, full CTU",
    "sweep3d": "sweep3d: 3-D noisy gas 64^3 (64 blocks of 16^3), periodic, PPM+HLLC, gamma 5/3",
    "amr3d": "amr3d: 3-D block-structured AMR, 16^3 blocks on 4^3 roots, levels 1-4 refined where "
             "|grad rho|/rho > 0.1 around a seeded level-set interface (rho 1 vs 10), periodic, PPM+HLLC, "
             "PARAMESH guard fill + flux correction every step",
}


def make_problem(name, scale=1.0):
    """(geom, hp, leaf UNK, mesh or None, zones) of a benchmark problem."""
    from flashx_b200 import simulations as S
    if name == "amr3d":
        from flashx_b200 import amr as A
        from flashx_b200.params import BC_PERIODIC, Geometry, HydroParams
        nroot = max(1, int(round(4 * scale)))
        geom = Geometry(3, 16, 16, 16, nroot, nroot, nroot, bc=(BC_PERIODIC,) * 6)
        hp = HydroParams()
        mesh, unk = A.levelset_problem(geom, hp, maxlev=4)
        return geom, hp, unk, mesh, mesh.ncells()
    geom, hp, init = S.config(name, scale=scale)
    return geom, hp, init(geom, hp), None, geom.ncells


def slab_split(geom, world, rank):
    """N > 1 on a uniform grid: the whole grid is `world` copies of the
    per-GPU grid stacked along its slowest axis (y in 2-D, z in 3-D), split
    into one slab per rank with halos exchanged every step (weak scaling:
    each GPU keeps the per-GPU grid's cells).  Returns (whole grid, slab)."""
    import dataclasses
    from flashx_b200.parallel import SlabDecomposition
    ax = geom.ndim - 1
    bbox = list(geom.bbox)
    lo, hi = bbox[ax]
    bbox[ax] = (lo, lo + world * (hi - lo))
    key = "nblocky" if geom.ndim == 2 else "nblockz"
    whole = dataclasses.replace(geom, bbox=tuple(bbox), **{key: getattr(geom, key) * world})
    return whole, SlabDecomposition(whole, world, rank)


def interiors(geom, unk, mesh):
    """Cell values of all (leaf) block interiors, (cells, var)."""
    from flashx_b200 import simulations as S
    if mesh is None:
        return S.gather_global(geom, unk).reshape(-1, unk.shape[-1])
    g = geom.nguard
    return unk[:, g:-g, g:-g, g:-g, :].reshape(-1, unk.shape[-1])


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="kh2d", choices=["kh2d", "sod2d", "rt3d", "sweep3d", "amr3d"],
                    help="kh2d (default, the headline workload) or another benchmark problem")
    ap.add_argument("--scale", type=float, default=1.0, help="block count per axis relative to the config")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=500,
                    help="steps of the mixed-vs-FP64 L1 and conservation-drift leg (0: skip)")
    ap.add_argument("--sweep", action="store_true",
                    help="throughput sweep of the batched-block path: one JSON line per (block size, count, "
                         "reconstruction, precision)")
    ap.add_argument("--sweep-blocks", type=int, nargs="+", default=[8, 16, 32],
                    help="block sizes (cells per side) the sweep covers")
    ap.add_argument("--sweep-min-blocks", type=int, default=0,
                    help="skip sweep points with fewer blocks")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return m.get("hbm_gbs", 6650.0), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Polls SM clocks and clock-event (throttle) reasons through NVML every
    10 ms while the timed region runs (read-only queries)."""

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.samples = []
        self._stop = None
        self._thr = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.cuda_index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def start(self):
        import threading
        try:
            import pynvml
            h = self._handle()
        except Exception:
            self._thr = None
            return
        self.smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        self._stop = threading.Event()
        bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap,
                "hw_power_brake": pynvml.nvmlClocksEventReasonHwPowerBrakeSlowdown}

        def run():
            while not self._stop.is_set():
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, [k for k, b in bits.items() if r & b]))
                except Exception:
                    pass
                self._stop.wait(0.01)
        self._thr = threading.Thread(target=run, daemon=True)
        self._thr.start()

    def stop(self):
        if self._thr is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        self._stop.set()
        self._thr.join()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(s for s, _ in self.samples), "sm_max_mhz": self.smax,
                "reasons": sorted({r for _, rs in self.samples for r in rs}), "samples": len(self.samples)}


def dist_setup(args, backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
        return dist, world, rank, local
    return None, 1, 0, local


def cpu_baseline_amr(seconds=10.0):
    """The oracle's AMR step (OpenMP over leaves, all host cores) on the full
    AMR workload, as many steps as fit in `seconds` (at least one)."""
    from oracle import fx_oracle as O
    geom, hp, unk, mesh, ncell = make_problem("amr3d")
    am = O.Amr(O.make_params(geom.as_dict(), hp), mesh.levels, mesh.bcoords)
    dt = 0.5 * am.compute_dt(unk)
    n, t0 = 0, time.perf_counter()
    while n == 0 or time.perf_counter() - t0 < seconds:
        am.hydro_step(unk, dt)
        dt = O.driver_dt(am.compute_dt(unk), dt)
        n += 1
    el = time.perf_counter() - t0
    cores = os.cpu_count()
    return {"value": ncell * n / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"amr3d {mesh.nleaf} leaves ({ncell} zones), {n} steps in {el:.1f} s, "
                      f"OpenMP over leaves on {cores} threads"}


def cpu_baseline_run(name, seconds=10.0, scale=1 / 4):
    """The oracle (OpenMP over blocks, all host cores) on a bounded sample of
    the workload: the same problem at `scale` blocks per axis (the stated
    size for the 2-D workloads, 1/4 per axis for the 3-D ones), as many steps
    as fit in `seconds`."""
    if name == "amr3d":
        return cpu_baseline_amr(seconds)
    from flashx_b200 import simulations as S
    from oracle import fx_oracle as O
    geom, hp, init = S.config(name, scale=scale)
    unk = init(geom, hp)
    p = O.make_params(geom.as_dict(), hp)
    dt = 0.5 * O.compute_dt(p, unk)
    O.hydro_step(p, unk, dt, dt)          # warm-up (thread pool, page-in)
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        O.hydro_step(p, unk, dt, dt)
        dt = O.driver_dt(O.compute_dt(p, unk), dt)
        n += 1
    el = time.perf_counter() - t0
    cores = os.cpu_count()
    nx = geom.nxb * geom.nblockx
    return {"value": geom.ncells * n / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{name} {nx}^{geom.ndim} ({geom.ncells} zones), {n} steps in {el:.1f} s, "
                      f"OpenMP over blocks on {cores} threads"}


def run_reference(args):
    dist, world, rank, _ = dist_setup(args, "gloo")
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    from oracle import fx_oracle as O
    if args.config == "amr3d":
        geom, hp, unk, mesh, ncell = make_problem("amr3d")
        am = O.Amr(O.make_params(geom.as_dict(), hp), mesh.levels, mesh.bcoords)
        step = lambda dt: am.hydro_step(unk, dt)
        cfl_dt = lambda: am.compute_dt(unk)
        steps, warm = max(1, min(args.steps, 3)), min(args.warmup, 1)
        sample = f"amr3d {mesh.nleaf} leaves ({ncell} zones) per step"
    else:
        # 2-D workloads at their stated size; 3-D ones (seconds per oracle
        # step at 256^3) at 1/4 of the blocks per axis
        scale = 1.0 if args.config in ("kh2d", "sod2d") else 1 / 4
        geom, hp, unk, mesh, ncell = make_problem(args.config, scale=scale)
        p = O.make_params(geom.as_dict(), hp)
        step = lambda dt: O.hydro_step(p, unk, dt, dt)
        cfl_dt = lambda: O.compute_dt(p, unk)
        steps, warm = args.steps, args.warmup
        if scale == 1.0 and args.config == "kh2d":
            steps, warm = min(args.steps, 20), min(args.warmup, 3)
        sample = f"{args.config} {geom.nxb * geom.nblockx}^{geom.ndim} per step" + (
            " (the stated configuration)" if scale == 1.0 else " (1/4 of the blocks per axis)")
    dt = 0.5 * cfl_dt()
    for _ in range(warm):
        step(dt)
        dt = O.driver_dt(cfl_dt(), dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        step(dt)
        dt = O.driver_dt(cfl_dt(), dt)
    el = time.perf_counter() - t0
    v = ncell * steps / el
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": warm, "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOADS[args.config] + f"; sampled as {sample}"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": f"oracle restatement of the Flash-X unsplit solver (the Fortran reference "
                                       f"cannot be built here), {sample}, {steps} timed steps, "
                                       f"OpenMP on {os.cpu_count()} threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def host_unk_round_trip(dev, hp, unk0, steps, barrier, max_over_ranks, global_min, zones, interior=True):
    """A caller whose host units read and write UNK every step.  interior:
    each step puts the block interiors of the hydro variables on the device
    (fxb_put_interior), runs Hydro and Driver_computeDt and gets the updated
    interiors back (fxb_get_interior); Hydro refills guard cells itself.
    Otherwise the whole pinned UNK crosses both ways (fxb_sync_from_host, then
    fxb_fill_guardcells with guard cells filled)."""
    import torch
    from flashx_b200.hydro import driver_dt
    interior = interior and dev.mesh is None       # AMR meshes move whole blocks either way
    host = torch.empty(unk0.shape, dtype=torch.float64, pin_memory=not interior).numpy()
    host[...] = unk0
    dev.attach_unk(host)
    if interior:                # page-lock and map the UNK once, outside the timed loop
        dev.put_interior(host)
    dt = dt_old = 0.5 * dev.Hydro_computeDt()
    barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        if interior:
            dev.put_interior(host)
        else:
            dev.attach_unk(host)
        dev.Hydro(0.0, dt, dt_old)
        dt_old, dt = dt, driver_dt(global_min(dev.Hydro_computeDt()), dt, hp)
        if interior:
            dev.get_interior(host)
        else:
            dev.Grid_fillGuardCells(host)
    barrier()
    el = max_over_ranks(time.perf_counter() - t0)
    if interior:
        g = dev.geom
        ncell = int(np.prod(unk0.shape[:1])) * g.nxb * g.nyb * (g.nzb if g.ndim == 3 else 1)
        nbytes = ncell * 10 * 8
        note = ("block interiors of the ten hydro variables from host UNK to the device and back every "
                "step (fxb_put_interior / fxb_get_interior: the UNK is page-locked once, its interior rows cross "
                "PCIe as strided copies on the copy engine), for callers whose host units touch UNK every step; "
                "Hydro fills the guard cells on the device")
    else:
        nbytes = int(host.nbytes)
        note = ("whole pinned UNK (guard cells included) to the device (fxb_sync_from_host) and back with its "
                "guard cells filled (fxb_fill_guardcells) every step")
    return {"value": zones * steps / el, "unit": UNIT, "h2d_bytes_per_step": nbytes + 24,
            "d2h_bytes_per_step": nbytes + 8, "steps": steps, "note": note}


def accuracy_leg(geom, hp, unk0, mesh, steps, global_min):
    """Mixed precision against plain FP64 on the workload over `steps` steps of
    one dt sequence (the FP64 run's Driver_computeDt sequence, replayed by the
    mixed run through Hydro(dt)): relative L1 of density, pressure and speed
    |v| over all (leaf) interior cells, and for both precisions the mass and
    total-energy drift |I(t) - I(0)| / |I(0)| from the volume integrals."""
    from flashx_b200.hydro import HydroDevice, driver_dt
    res = {"steps": steps}
    states, drift, dts = {}, {}, []
    for prec in ("fp64", "mixed"):
        dev = HydroDevice(geom, hp, prec, mesh=mesh)
        dev.attach_unk(unk0.copy())
        I0 = dev.integrals()
        if prec == "fp64":
            dt = dt_old = 0.5 * dev.Hydro_computeDt()
            for _ in range(steps):
                dts.append(dt)
                dev.Hydro(0.0, dt, dt_old)
                dt_old, dt = dt, driver_dt(global_min(dev.Hydro_computeDt()), dt, hp)
        else:
            for i, dt in enumerate(dts):
                dev.Hydro(0.0, dt, dts[i - 1] if i else dt)
        I1 = dev.integrals()
        st = np.zeros(unk0.shape)
        dev.sync_to_host(st)
        dev.close()
        states[prec] = interiors(geom, st, mesh)
        drift[prec] = {"mass": float(abs(I1[0] - I0[0]) / abs(I0[0])),
                       "total_energy": float(abs(I1[4] - I0[4]) / abs(I0[4]))}
    a, b = states["mixed"], states["fp64"]
    rel = lambda x, y: float(np.mean(np.abs(x - y)) / max(np.mean(np.abs(y)), 1e-300))
    speed = lambda u: np.sqrt(u[:, 8] ** 2 + u[:, 9] ** 2 + u[:, 10] ** 2)
    res["l1_rel_mixed_vs_fp64"] = {"dens": rel(a[:, 0], b[:, 0]), "pres": rel(a[:, 5], b[:, 5]),
                                   "speed": rel(speed(a), speed(b))}
    res["drift"] = drift
    res["simulated_time"] = float(sum(dts))
    res["note"] = ("same dt sequence for both precisions (FP64 Driver_computeDt); drift is the relative change "
                   "of the volume integrals of mass and total energy (conserved on periodic domains; "
                   "gravity and open boundaries exchange energy)")
    return res


def per_block_driver(dev, geom, mesh, hp, steps, global_min):
    """The Fortran driver's calling pattern: per step one Hydro() and one
    Hydro_computeDt per leaf block (Driver_computeDt.F90:306), each returning
    dtCheck and dtMinLoc, reduced on the host; through the C ABI with host
    buffers.  The library reduces on the device at the first call of a step
    and answers the others from its cache (counted by fxb_counters)."""
    import ctypes
    from flashx_b200.hydro import COUNT_DT_CACHED, COUNT_DT_DEVICE, _check, driver_dt
    lib = dev.lib
    f = lib.fxb_compute_dt
    nblk = dev.unk_shape[0]       # this rank's blocks
    out = ctypes.c_double()
    loc = (ctypes.c_int32 * 5)()
    pout = ctypes.byref(out)
    dt = dt_old = 0.5 * dev.Hydro_computeDt()
    c0 = dev.counters()
    t0 = time.perf_counter()
    for _ in range(steps):
        dev.fill_halos()          # halos or leaves from the other ranks (no-op on one GPU)
        _check(lib.fxb_hydro_step(0.0, dt, dt_old))
        dtcheck = 1e300
        for _b in range(nblk):
            _check(f(pout, loc))
            if out.value < dtcheck:
                dtcheck = out.value
        dt_old, dt = dt, driver_dt(global_min(dtcheck), dt, hp)
    el = time.perf_counter() - t0
    c1 = dev.counters()
    return {"value": geom_zones(geom, mesh) * steps / el, "unit": UNIT, "steps": steps,
            "h2d_bytes_per_step": 24, "d2h_bytes_per_step": 16,
            "hydro_computeDt_calls_per_step": nblk,
            "device_dt_reductions_per_step": (c1[COUNT_DT_DEVICE] - c0[COUNT_DT_DEVICE]) / steps,
            "cached_dt_calls_per_step": (c1[COUNT_DT_CACHED] - c0[COUNT_DT_CACHED]) / steps,
            "note": "per step: fxb_hydro_step, then fxb_compute_dt(dt, dtMinLoc) once per leaf block from a Python "
                    "loop (ctypes call overhead included); one device reduction per step, the other calls "
                    "return the cached result"}


def geom_zones(geom, mesh):
    return mesh.ncells() if mesh is not None else geom.ncells


def fp_roofline(config, precision, zones_per_s):
    """Floating-point roofline of the hot kernel from the FP operations per
    zone-update counted by ncu (profiles/*_flops.json: DADD + DMUL + 2 DFMA,
    FADD + FMUL + 2 FFMA; divisions and square roots count as the FMA
    sequences they execute) times the measured zone-update rate, against the
    nominal FP64 / FP32 peaks (no measured figure exists for them)."""
    try:
        with open(FLOPS_FILES[config]) as f:
            fj = json.load(f)
    except Exception:
        return None
    c, pk = fj[precision], fj["peaks_nominal_tflops"]
    f64 = c["fp64_flops_per_zone"] * zones_per_s / 1e12
    f32 = c["fp32_flops_per_zone"] * zones_per_s / 1e12
    return {"bound": "fp64 pipe" if precision == "fp64" else "fp32 + fp64 pipes",
            "achieved_fp64": f64, "achieved_fp32": f32, "peak_fp64": pk["fp64"], "peak_fp32": pk["fp32"],
            "unit": "TFLOP/s", "frac_fp64": f64 / pk["fp64"], "frac_fp32": f32 / pk["fp32"],
            "fp64_flops_per_zone": c["fp64_flops_per_zone"], "fp32_flops_per_zone": c["fp32_flops_per_zone"],
            "peak_kind": "nominal"}


def regrid_cycle(dev, hp, mesh):
    """One Grid_updateRefinement on the AMR workload after the timed steps
    (not part of the zone-update rate): refinement marks on the device
    (density criterion of the workload, Paramesh4 defaults refine_cutoff 0.8,
    derefine_cutoff 0.2, refine_filter 0.01), the tree update on the host
    (fxb_refine_derefine),
    the data movement on the device (fxb_regrid), then two steps on the new
    mesh.  Host wall time of each part, with the device synchronised."""
    import torch
    maxlev = int(max(mesh.levels))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    flags, _ = dev.Grid_markRefineDerefine([("dens", 0.8, 0.2, 0.01)], maxlev)
    t1 = time.perf_counter()
    from flashx_b200.hydro import refine_derefine
    new = refine_derefine(dev.mesh, flags, 1, maxlev)
    t2 = time.perf_counter()
    from flashx_b200.hydro import _check, mesh_blocks
    _check(dev.lib.fxb_regrid(mesh_blocks(new.levels, new.bcoords), new.nleaf))
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    dev.mesh, dev.unk_shape = new, new.unk_shape
    dt = 0.5 * dev.Hydro_computeDt()
    for _ in range(2):
        dev.Hydro(0.0, dt, dt)
    step_ms = dev.last_timing()[0]
    return {"leaves_before": int(mesh.nleaf), "leaves_after": int(new.nleaf),
            "marked_refine": int(np.sum(np.asarray(flags) == 1)), "marked_derefine": int(np.sum(np.asarray(flags) == -1)),
            "mark_ms": 1e3 * (t1 - t0), "tree_update_ms": 1e3 * (t2 - t1),
            "regrid_ms": 1e3 * (t3 - t2), "step_ms_after": step_ms,
            "note": "regrid_ms covers fxb_regrid: restriction, copies, prolongation, Eos and the new mesh's "
                    "tree, neighbour tables and guard-fill plan (the tuned launch shapes are kept)"}


def run_ours(args):
    import torch
    dist, world, rank, local = dist_setup(args, "nccl")
    torch.cuda.set_device(local)
    from flashx_b200 import simulations as S
    from flashx_b200.hydro import HydroDevice, driver_dt

    geom, hp, unk0, mesh, ncell = make_problem(args.config, scale=args.scale)
    K, W = args.steps, args.warmup

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from flashx_b200.parallel import allreduce_min as global_min   # Driver_computeDt's AllReduce(MIN)

    # uniform grids split into slabs over the ranks, AMR meshes into Morton
    # ranges of `world` stacked copies (each rank owns one copy's leaves)
    slab = split = None
    if world > 1 and mesh is None:
        whole, slab = slab_split(geom, world, rank)
    elif world > 1:
        from flashx_b200 import amr as A
        from flashx_b200.parallel import AmrDecomposition
        whole, wmesh = A.stack_copies(mesh, world)
        split = AmrDecomposition(wmesh, world, rank)
        assert split.bounds[rank] == rank * mesh.nleaf and len(split.owned()) == mesh.nleaf

    def timed_run(precision):
        if slab is not None:
            dev = HydroDevice(whole, hp, precision, slab=slab)   # this rank's slab: the per-GPU grid's blocks
        elif split is not None:
            dev = HydroDevice(whole, hp, precision, mesh=wmesh, amr_split=split)   # host UNK: the own copy
        else:
            dev = HydroDevice(geom, hp, precision, mesh=mesh)
        dev.attach_unk(unk0.copy())
        dt = global_min(0.5 * dev.Hydro_computeDt())
        ext = torch.cuda.ExternalStream(dev.lib.fxb_stream())
        if world == 1:
            dt, dt_old = dev.advance(W, dt, dt)
            barrier()
            clk = Clocks(local); clk.start()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            dt, dt_old = dev.advance(K, dt, dt_old)
            e1.record(ext)
            barrier()
            clocks = clk.stop()
            ms = e0.elapsed_time(e1)
            launches = dev.last_timing()[1]
        else:
            dt_old = dt
            for _ in range(W):
                dev.Hydro(0.0, dt, dt_old)
                dt_old, dt = dt, driver_dt(global_min(dev.Hydro_computeDt()), dt, hp)
            barrier()
            clk = Clocks(local); clk.start()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            for _ in range(K):
                dev.Hydro(0.0, dt, dt_old)
                dt_old, dt = dt, driver_dt(global_min(dev.Hydro_computeDt()), dt, hp)
            e1.record(ext)
            barrier()
            clocks = clk.stop()
            ms = e0.elapsed_time(e1)
            launches = dev.last_timing()[1] * K
        ms = max_over_ranks(ms)
        return dev, ms, launches, clocks

    # ---- FP64 (headline)
    dev, ms, launches, clocks = timed_run("fp64")
    value = world * ncell * K / (ms / 1e3)
    # kernel-only timing of the fused hydro kernel for the roofline
    kms = []
    dt = 0.5 * dev.Hydro_computeDt()
    for _ in range(min(K, 10)):
        dev.Hydro(0.0, dt, dt)
        kms.append(dev.last_timing()[0])
    dev.Hydro_computeDt()
    kernel_ms = statistics.mean(kms)
    fp64_state = np.zeros(unk0.shape)
    # e2e: host-driven loop through the C ABI, dt crossing PCIe every step
    dev.attach_unk(unk0.copy())
    dt = dt_old = 0.5 * dev.Hydro_computeDt()
    barrier()
    t0 = time.perf_counter()
    t_sim = 0.0
    for _ in range(K):
        dev.Hydro(t_sim + dt, dt, dt_old)
        t_sim += dt
        dt_old, dt = dt, driver_dt(global_min(dev.Hydro_computeDt()), dt, hp)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = world * ncell * K / e2e_s
    dev.sync_to_host(fp64_state)
    ref_after = interiors(geom, fp64_state, mesh)
    e2e_host = host_unk_round_trip(dev, hp, unk0, min(K, 20), barrier, max_over_ranks, global_min, world * ncell)
    e2e_host_full = host_unk_round_trip(dev, hp, unk0, min(K, 10), barrier, max_over_ranks, global_min,
                                        world * ncell, interior=False)
    dev.attach_unk(unk0.copy())
    e2e_driver = per_block_driver(dev, geom, mesh, hp, min(K, 5), global_min)

    peak, peak_kind = measured_peaks()
    achieved = BYTES_PER_ZONE * ncell / (kernel_ms / 1e3) / 1e9
    traffic = None
    try:
        with open(TRAFFIC_FILES[args.config]) as f:
            tj = json.load(f)
        if tj.get("zones") == ncell:
            traffic = tj.get("bytes_per_launch")
    except Exception:
        pass

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded initial state of the workload, Philox4x32-10 where random)",
            "config": {"workload": WORKLOADS[args.config] + ("" if args.scale == 1.0 else f" at scale {args.scale}"),
                       "zones_per_gpu": ncell,
                       "parallelism": ("single" if world == 1 else
                                       f"AMR mesh of {world} copies of the per-GPU mesh stacked along z, split in "
                                       f"Morton ranges (one copy per GPU); per step each rank receives the "
                                       f"{len(split.ghosts[rank]) if split else 0} leaves its guard fills read "
                                       f"(NCCL send/recv) and computes the fluxes of "
                                       f"{int((split.roles == 2).sum()) if split else 0} finer face neighbours; "
                                       f"common dt (all-reduce)" if slab is None else
                                       f"slabs: {world} copies of the grid stacked along its slowest axis, one "
                                       f"slab per GPU, halos of {slab.halos[0]} planes exchanged every step "
                                       f"(NCCL send/recv), common dt (all-reduce)"),
                       "l2": "inputs larger than L2 (state %.0f MB vs 126 MB L2)" % (2 * 10 * 8 * ncell / 1e6),
                       "timing": "CUDA events on the library stream, device dt loop (CUDA graph)"},
            "clocks": clocks,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "hydro2d_kernel<double>" if geom.ndim == 2 else
                                   ("AMR step (restriction, guard fill, 3-D pipeline, flux correction, update)<double>"
                                    if mesh is not None else
                                    "3-D pipeline (sig3d, states3d x3, flux3d x3, update3d)<double>"),
                         "kernel_ms": kernel_ms,
                         "algorithmic_bytes_per_zone": BYTES_PER_ZONE},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 24, "d2h_bytes_per_step": 8,
                    "note": "host loop via fxb_hydro_step/fxb_compute_dt: (t, dt, dtOld) in, dt out per step; "
                            "UNK stays resident on the device"},
            "e2e_host_unk": e2e_host,
            "e2e_host_unk_full": e2e_host_full,
            "e2e_driver": e2e_driver}
    flops = fp_roofline(args.config, "fp64", ncell / (kernel_ms / 1e3))
    if flops:
        line["roofline_fp"] = flops
    line["config"]["tuning"] = dev.tuning()
    if mesh is not None:
        line["config"]["leaves_per_level"] = mesh.level_counts()
        if world == 1:
            line["regrid"] = regrid_cycle(dev, hp, mesh)
    dev.close()

    # ---- mixed precision
    if not args.no_mixed:
        mdev, mms, mlaunch, mclk = timed_run("mixed")
        mstate = np.zeros(unk0.shape)
        # same steps as the FP64 e2e run for the error estimate
        mdev.attach_unk(unk0.copy())
        dt = dt_old = 0.5 * mdev.Hydro_computeDt()
        for _ in range(K):
            mdev.Hydro(0.0, dt, dt_old)
            dt_old, dt = dt, driver_dt(global_min(mdev.Hydro_computeDt()), dt, hp)
        mdev.sync_to_host(mstate)
        m_after = interiors(geom, mstate, mesh)
        mdev.close()
        l1 = {v: float(np.mean(np.abs(m_after[..., i] - ref_after[..., i])) / max(np.mean(np.abs(ref_after[..., i])), 1e-300))
              for v, i in (("dens", 0), ("pres", 5), ("velx", 8), ("vely", 9))}
        mflops = fp_roofline(args.config, "mixed", ncell * K / (mms / 1e3))
        line["mixed"] = {"value": world * ncell * K / (mms / 1e3), "ms_per_step": mms / K,
                         "speedup_vs_fp64": ms / mms, "l1_rel_vs_fp64_after_steps": l1,
                         "dtype": "f32 reconstruction/Riemann + f64 update", "clocks": mclk}
        if mflops:
            line["mixed"]["roofline_fp"] = mflops

    if not args.no_mixed and world == 1 and args.accuracy_steps > 0:
        line["accuracy"] = accuracy_leg(geom, hp, unk0, mesh, args.accuracy_steps, global_min)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_run(args.config, scale=args.scale if geom.ndim == 2 else args.scale / 4)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def host_available():
    """Bytes of host memory available now (MemAvailable), 12 GB if unknown."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 12e9


def sweep_points(hbm_bytes, host_limit=None, blocks=(8, 16, 32)):
    """(n, nb) pairs: blocks of n^3 interior cells, (2 nb)^3 leaves at level 2,
    capped by the host UNK (guard cells included; at most 45 % of the host
    memory available) and by device memory."""
    host_limit = 0.45 * host_available() if host_limit is None else host_limit
    pts = []
    for n in blocks:
        for nb in (2, 4, 8, 16, 29):
            count = (2 * nb) ** 3
            unk_bytes = count * (n + 8) ** 3 * 11 * 8
            store_bytes = 2 * (count + nb ** 3) * n ** 3 * 10 * 8
            if unk_bytes <= host_limit and store_bytes <= 0.4 * hbm_bytes:
                pts.append((n, nb))
    return pts


def run_sweep(args):
    """Configuration 5: 3-D noisy gas (gamma 5/3) in blocks of 8^3, 16^3 and 32^3,
    64 to 195,112 blocks (capped by memory), PPM and WENO5, FP64 and mixed, run
    through the batched-block path (every block a leaf at level 2, guard cells
    filled by the AMR kernels) with its tuned launch shape."""
    import torch
    from flashx_b200 import amr as A
    from flashx_b200 import simulations as S
    from flashx_b200.hydro import HydroDevice
    from flashx_b200.params import BC_PERIODIC, Geometry, HydroParams
    torch.cuda.set_device(0)
    peak, peak_kind = measured_peaks()
    hbm = torch.cuda.get_device_properties(0).total_memory
    for n, nb in sweep_points(hbm, blocks=args.sweep_blocks):
        if (2 * nb) ** 3 < args.sweep_min_blocks:
            continue
        root = Geometry(3, n, n, n, nb, nb, nb, bc=(BC_PERIODIC,) * 6)
        fine = Geometry(3, n, n, n, 2 * nb, 2 * nb, 2 * nb, bc=(BC_PERIODIC,) * 6)
        # every block a leaf at level 2, Morton order; the state filled in place
        # (the values of the uniform grid's noisy gas at the same cells)
        mesh = A.AmrMesh(root, [(2, (i, j, k)) for k in range(2 * nb) for j in range(2 * nb) for i in range(2 * nb)])
        hp0 = HydroParams(gamma=5.0 / 3.0)
        unk = np.zeros(mesh.unk_shape)
        S.noisy_gas_blocks(fine, hp0, mesh.bcoords, unk, chunk=256, threads=os.cpu_count() or 1)
        zones = mesh.ncells()
        K = max(3, min(50, int(4e8 / zones)))
        for order in (3, 5):
            for prec in ("fp64", "mixed"):
                hp = HydroParams(gamma=5.0 / 3.0, order=order)
                dev = HydroDevice(root, hp, prec, mesh=mesh)
                dev.attach_unk(unk)
                dt = 0.5 * dev.Hydro_computeDt()
                dt, dto = dev.advance(3, dt, dt)
                dt, dto = dev.advance(K, dt, dto)
                ms, launches = dev.last_timing()
                value = zones * K / (ms / 1e3)
                achieved = BYTES_PER_ZONE * value / 1e9
                line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": 3,
                        "ms_per_step": ms / K, "higher_is_better": True, "dtype": "f64" if prec == "fp64" else
                        "f32 reconstruction/Riemann + f64 update", "data": "synthetic (Philox noise, Box-Muller)",
                        "config": {"workload": f"sweep3d blocks of {n}^3, {mesh.nleaf} blocks, "
                                               f"{'PPM' if order == 3 else 'WENO5'}+HLLC, batched-block path",
                                   "block": n, "blocks": mesh.nleaf, "zones": zones, "order": order,
                                   "precision": prec, "tuning": dev.tuning()},
                        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                     "frac": achieved / peak, "peak_kind": peak_kind},
                        "gpu_launches": launches}
                print(json.dumps(line), flush=True)
                dev.close()


def main():
    args = parse()
    if args.sweep:
        run_sweep(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
