"""Autotuner for batched solves of voxel pieces.

Pieces are put in size classes (their grid cells rounded up to a power of two). For
each class it times one representative piece's full solve (setup + PCG to the
requested tolerance) under every candidate setting -- block-Jacobi sweeps before and
after each coarse correction (the reference does one, statics/src/bodies.rs:386,
396-401) and the stencil tile (the window of parts grouped by axis) -- and keeps the
fastest. Choices are cached in a JSON file keyed by class, precision and tolerance, so
a later batch of the same classes is not tuned again.
"""
from __future__ import annotations

import json
import os
import time

from . import FP64, MIXED, Solver, options

SWEEPS = (1, 2, 3)
TILES = (256, 1024, 4096)
DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_cache.json")


def size_class(state) -> int:
    cells = int(state.size)
    c = 1
    while c < cells:
        c <<= 1
    return c


def _key(cls: int, precision: int, tol: float) -> str:
    return f"{cls}:{'mixed' if precision == MIXED else 'fp64'}:{tol:g}"


def load(path: str = DEFAULT_CACHE) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save(cache: dict, path: str = DEFAULT_CACHE) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune_class(solver: Solver, piece, precision: int = MIXED, tol: float = 1e-8, repeats: int = 2) -> dict:
    """Times every (sweeps, tile) on one piece; returns the fastest with its timings."""
    state, k = piece
    trials = []
    for sweeps in SWEEPS:
        for tile in TILES:
            opt = options(tol=tol, precision=precision, sweeps=sweeps, tile=tile, max_iter=20000)
            best = None
            for _ in range(repeats):
                t = time.perf_counter()
                _, info = solver.solve_grid(state, k, opt)
                dt = time.perf_counter() - t
                if info["status"] != 0:
                    dt = float("inf")
                best = dt if best is None else min(best, dt)
            trials.append({"sweeps": sweeps, "tile": tile, "seconds": best, "iterations": info["iterations"]})
    win = min(trials, key=lambda t: t["seconds"])
    return {"sweeps": win["sweeps"], "tile": win["tile"], "seconds": win["seconds"], "trials": trials}


def choose(solver: Solver, pieces, precision: int = MIXED, tol: float = 1e-8, path: str = DEFAULT_CACHE) -> dict:
    """The setting for each size class present in `pieces` (tuning the classes the cache
    lacks). Returns {class: {"sweeps": s, "tile": t, ...}}."""
    cache = load(path)
    out, changed = {}, False
    for piece in pieces:
        cls = size_class(piece[0])
        if cls in out:
            continue
        key = _key(cls, precision, tol)
        if key not in cache:
            cache[key] = tune_class(solver, piece, precision, tol)
            changed = True
        out[cls] = cache[key]
    if changed:
        save(cache, path)
    return out


def solve_batch(solver: Solver, pieces, precision: int = MIXED, tol: float = 1e-8, path: str = DEFAULT_CACHE,
                settings: dict | None = None):
    """Solves `pieces` grouped by size class, each group one batched solve with its
    tuned setting. Returns (motions, infos) in the order of `pieces`."""
    settings = settings or choose(solver, pieces, precision, tol, path)
    groups: dict[int, list[int]] = {}
    for i, p in enumerate(pieces):
        groups.setdefault(size_class(p[0]), []).append(i)
    motions, infos = [None] * len(pieces), [None] * len(pieces)
    for cls, idx in groups.items():
        s = settings[cls]
        opt = options(tol=tol, precision=precision, sweeps=s["sweeps"], tile=s["tile"], max_iter=20000)
        outs, inf = solver.solve_grid_batch([pieces[i] for i in idx], opt)
        for j, i in enumerate(idx):
            motions[i], infos[i] = outs[j], inf[j]
    return motions, infos
