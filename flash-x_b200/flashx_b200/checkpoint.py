"""Checkpoint, restart and comparison of the hydro state.

A checkpoint holds the datasets of a Flash-X HDF5 checkpoint for the
variables and tree of this path (IO/IOMain/hdf5/io_createDatasets.F90:88-130,
io_h5write_header.c:269-330, io_h5write_lists.c:380-430): "unknown names",
one dataset per variable named by its four-letter name with shape
(blocks, nzb, nyb, nxb), "refine level", "node type", "which child",
"coordinates", "block size", "bounding box", "integer scalars" and
"real scalars" (nstep, time, dt, dtold), the runtime parameters split by
type, and "sim info".  This image has no HDF5 library, so the container is
a NumPy .npz archive with those dataset names as keys; the arrays keep the
shapes and meanings of the HDF5 datasets.  Only leaf blocks are stored (node
type 1): parents are rebuilt from the leaves at restart, as the device does
on every step.

`compare` restates what sfocu (tools/sfocu) reports for two checkpoints:
blocks are matched by refinement level and position, and for every
variable the largest absolute and relative differences and the L1 norm of
the difference relative to the L1 norm of the first file.
"""
import dataclasses
import json

import numpy as np

from .params import Geometry, HydroParams, NUNK, UNK_VARS


def _leaf_geometry(geom: Geometry, levels, bcoords):
    """Block centres, sizes and bounding boxes of leaves (level, coords)."""
    ndim = geom.ndim
    nb0 = (geom.nblockx, geom.nblocky, geom.nblockz)
    lo = np.array([geom.bbox[a][0] for a in range(3)])
    ext = np.array([geom.bbox[a][1] - geom.bbox[a][0] for a in range(3)])
    n = len(levels)
    size = np.zeros((n, ndim))
    coord = np.zeros((n, ndim))
    box = np.zeros((n, ndim, 2))
    for b in range(n):
        for a in range(ndim):
            bs = ext[a] / (nb0[a] * 2.0 ** (int(levels[b]) - 1))
            size[b, a] = bs
            box[b, a, 0] = lo[a] + bcoords[b][a] * bs
            box[b, a, 1] = box[b, a, 0] + bs
            coord[b, a] = box[b, a, 0] + 0.5 * bs
    return coord, size, box


def write_checkpoint(path, geom: Geometry, hp: HydroParams, unk, mesh=None, time=0.0, dt=0.0, dtold=0.0,
                     nstep=0):
    """IO_writeCheckpoint for the host UNK (leaves, guard cells ignored).
    `mesh`: the AmrMesh of an AMR run, None for the uniform grid."""
    g = geom.nguard
    nk = geom.nzb if geom.ndim == 3 else 1
    gk = g if geom.ndim == 3 else 0
    gj = g if geom.ndim >= 2 else 0
    nj = geom.nyb if geom.ndim >= 2 else 1
    inner = unk[:, gk:gk + nk, gj:gj + nj, g:g + geom.nxb, :]
    if mesh is None:
        nbz = geom.nblockz if geom.ndim == 3 else 1
        nby = geom.nblocky if geom.ndim >= 2 else 1
        levels = np.ones(geom.nblocks, dtype=np.int32)
        bcoords = np.array([(i, j, k) for k in range(nbz) for j in range(nby) for i in range(geom.nblockx)],
                           dtype=np.int32)
    else:
        levels, bcoords = np.asarray(mesh.levels, dtype=np.int32), np.asarray(mesh.bcoords, dtype=np.int32)
    if inner.shape[0] != len(levels):
        raise ValueError("UNK and block list differ in length")
    coord, size, box = _leaf_geometry(geom, levels, bcoords)
    which = np.array([1 + (c[0] & 1) + 2 * (c[1] & 1) + 4 * (c[2] & 1) if l > 1 else -1
                      for l, c in zip(levels, bcoords)], dtype=np.int32)
    data = {"unknown names": np.array([v.ljust(4)[:4] for v in UNK_VARS]),
            "refine level": levels, "node type": np.ones(len(levels), dtype=np.int32), "which child": which,
            "coordinates": coord, "block size": size, "bounding box": box,
            "block coordinates": bcoords,   # PARAMESH position of each leaf at its level (not in HDF5 files)
            "integer scalars": np.array([("nstep", nstep), ("nxb", geom.nxb), ("nyb", geom.nyb),
                                         ("nzb", geom.nzb), ("dimensionality", geom.ndim),
                                         ("globalnumblocks", len(levels))],
                                        dtype=[("name", "U80"), ("value", np.int64)]),
            "real scalars": np.array([("time", time), ("dt", dt), ("dtold", dtold)],
                                     dtype=[("name", "U80"), ("value", np.float64)]),
            "sim info": np.array(json.dumps({"setup": "flashx_b200 unsplit hydro", "geometry": geom.as_dict()}))}
    rp = hp.as_dict()
    for kind, pytype, dtype in (("integer", int, np.int64), ("real", float, np.float64),
                                ("logical", bool, np.int64), ("string", str, "U80")):
        items = [(k, v) for k, v in rp.items() if type(v) is pytype]
        data[f"{kind} runtime parameters"] = np.array(items, dtype=[("name", "U80"), ("value", dtype)])
    data["gravity"] = np.array(rp["gravity"], dtype=np.float64)
    for v, name in enumerate(UNK_VARS):
        data[name.ljust(4)[:4]] = np.ascontiguousarray(inner[..., v])
    with open(path, "wb") as f:
        np.savez(f, **data)


def read_checkpoint(path):
    """IO_readCheckpoint: a dict with geom, hp, levels, bcoords, unk (guard
    cells zero; leaf order of the file), time, dt, dtold, nstep."""
    z = np.load(path, allow_pickle=False)
    info = json.loads(str(z["sim info"]))
    gd = info["geometry"]
    geom = Geometry(gd["ndim"], gd["nxb"], gd["nyb"], gd["nzb"], gd["nblockx"], gd["nblocky"], gd["nblockz"],
                    bbox=tuple(tuple(b) for b in gd["bbox"]), bc=tuple(gd["bc"]), nguard=gd["nguard"])
    kw = {}
    names = {f.name for f in dataclasses.fields(HydroParams)}
    for kind in ("integer", "real", "logical", "string"):
        for name, value in z[f"{kind} runtime parameters"]:
            name = str(name)
            if name in names:
                kw[name] = bool(value) if kind == "logical" else (int(value) if kind == "integer" else
                                                                   (float(value) if kind == "real" else str(value)))
    kw["gravity"] = tuple(float(x) for x in z["gravity"])
    hp = HydroParams(**kw)
    levels, bcoords = z["refine level"], z["block coordinates"]
    n = len(levels)
    unk = np.zeros((n,) + geom.block_shape)
    g = geom.nguard
    nk = geom.nzb if geom.ndim == 3 else 1
    gk = g if geom.ndim == 3 else 0
    gj = g if geom.ndim >= 2 else 0
    nj = geom.nyb if geom.ndim >= 2 else 1
    for v, name in enumerate(UNK_VARS):
        unk[:, gk:gk + nk, gj:gj + nj, g:g + geom.nxb, v] = z[name.ljust(4)[:4]]
    ints = {str(k): int(v) for k, v in z["integer scalars"]}
    reals = {str(k): float(v) for k, v in z["real scalars"]}
    return {"geom": geom, "hp": hp, "levels": levels, "bcoords": bcoords, "unk": unk, "nstep": ints["nstep"],
            "time": reals["time"], "dt": reals["dt"], "dtold": reals["dtold"]}


def restart_mesh(ck):
    """The AmrMesh of a checkpoint (None for a uniform grid)."""
    if np.all(ck["levels"] == 1) and len(ck["levels"]) == ck["geom"].nblocks:
        return None
    from .amr import AmrMesh
    return AmrMesh(ck["geom"], [(int(l), tuple(int(v) for v in c)) for l, c in zip(ck["levels"], ck["bcoords"])])


def compare(path_a, path_b, variables=None):
    """sfocu-style comparison: per variable the largest absolute difference,
    the largest relative difference |a - b| / max(|a|, |b|) and the L1 norm of
    a - b over the L1 norm of a, over blocks matched by level and position.
    Raises if the two files hold different block sets."""
    za, zb = np.load(path_a), np.load(path_b)
    ka = {(int(l), tuple(int(v) for v in c)): i for i, (l, c) in enumerate(zip(za["refine level"],
                                                                            za["block coordinates"]))}
    kb = {(int(l), tuple(int(v) for v in c)): i for i, (l, c) in enumerate(zip(zb["refine level"],
                                                                            zb["block coordinates"]))}
    if set(ka) != set(kb):
        raise ValueError("the checkpoints hold different block sets")
    order = sorted(ka)
    ia, ib = [ka[k] for k in order], [kb[k] for k in order]
    out = {}
    for name in (variables or [str(n).strip() for n in za["unknown names"]]):
        key = name.ljust(4)[:4]
        a, b = za[key][ia], zb[key][ib]
        d = np.abs(a - b)
        den = np.maximum(np.abs(a), np.abs(b))
        rel = np.where(den > 0, d / np.where(den > 0, den, 1.0), 0.0)
        l1a = np.sum(np.abs(a))
        out[name] = {"max_abs": float(d.max()), "max_rel": float(rel.max()),
                     "l1_rel": float(d.sum() / l1a) if l1a > 0 else float(d.sum())}
    return out
