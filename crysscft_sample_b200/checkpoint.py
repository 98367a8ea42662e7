"""Checkpoint and resume of an SCFT run (the reference only writes its final fields as
text, src/crysSCFT_sample.cpp:271-282, 511; this is the binary dump it lacks).

A checkpoint is one ``.npz`` file: the physical-grid fields wA, wB (what the iteration
depends on), phiA, phiB of the last iteration, and a JSON header with the solver (kind,
logical grid, 3m translations, anisotropic PMMM), the cell, fA, ds, chiN, the simple-mixing
acceptance, the mixing mode, the precision and the number of iterations done.  Resuming
restores the fields; an Anderson history restarts empty.
"""
from __future__ import annotations

import json

import numpy as np

FORMAT = "crysscft-b200-checkpoint/1"
_KEYS = ("kind", "grid_log", "cell", "fA", "ds", "xN", "acceptance", "iterations")


def write(path, meta: dict, fields: dict) -> None:
    """Write `fields` (wA, wB, phiA, phiB: 1-D float64 arrays of equal size) with `meta`."""
    missing = [k for k in _KEYS if k not in meta]
    if missing:
        raise ValueError(f"checkpoint header lacks {missing}")
    arrays = {k: np.ascontiguousarray(fields[k], dtype=np.float64).ravel() for k in ("wA", "wB", "phiA", "phiB")}
    sizes = {a.size for a in arrays.values()}
    if len(sizes) != 1:
        raise ValueError("checkpoint fields differ in size")
    header = dict(meta, format=FORMAT)
    with open(path, "wb") as f:
        np.savez(f, header=np.frombuffer(json.dumps(header, sort_keys=True).encode(), dtype=np.uint8), **arrays)


def read(path):
    """(meta, fields) of a checkpoint written by `write`."""
    with np.load(path, allow_pickle=False) as z:
        header = json.loads(bytes(z["header"]).decode())
        if header.get("format") != FORMAT:
            raise ValueError(f"not a checkpoint of this library: {header.get('format')!r}")
        fields = {k: np.array(z[k]) for k in ("wA", "wB", "phiA", "phiB")}
    header.pop("format")
    return header, fields


def save(run, path) -> None:
    """Checkpoint a DiblockSCFT `run` (crysscft_sample_b200.scft)."""
    s = run.solver
    g = getattr(s, "_g", None)
    meta = {
        "kind": s._kind, "grid_log": list(s.get_grid_size_log()), "cell": [float(v) for v in s.get_cell_para()],
        "fA": float(run.fA), "ds": float(run.ds), "xN": float(run.xN), "acceptance": float(run.acceptance),
        "iterations": int(run.iterations_done), "precision": run.get_precision(), "mixing": list(run.mixing),
        "translational_part": None if g is None else [float(v) for v in g],
        "anisotropic": bool(getattr(s, "anisotropic", False)),
    }
    write(path, meta, run.get_fields())


def resume(path, device: int = -1):
    """A new DiblockSCFT (and its solver) in the state a checkpoint recorded."""
    from . import scft, solvers

    meta, f = read(path)
    kind = meta["kind"]
    if kind == "3M":
        g = meta.get("translational_part") or (0.0,) * 9
        solver = solvers.CrysPSSolver3m(meta["grid_log"], translational_part=g, device=device)
    elif kind == "PMMM":
        solver = solvers.CrysPSSolverPmmm(meta["grid_log"], device=device, anisotropic=meta.get("anisotropic", False))
    else:
        solver = solvers.make_solver(kind, meta["grid_log"], device=device)
    solver.set_cell_para(tuple(meta["cell"]))
    run = scft.DiblockSCFT(solver, meta["fA"], meta["ds"], meta["xN"], meta["acceptance"])
    run.set_fields(f["wA"], f["wB"])
    run.iterations_done = int(meta["iterations"])
    if meta.get("precision", "fp64") != "fp64":
        run.set_precision(meta["precision"])
    mixing = meta.get("mixing") or ["simple"]
    if mixing[0] == "anderson":
        run.set_mixing("anderson", history=int(mixing[1]), beta=float(mixing[2]))
    return run
