"""Autotuner for batched solves of voxel pieces.

Pieces are put in size classes (their grid cells rounded up to a power of two). For
each class it times a batched solve (setup + PCG to the requested tolerance, as the
batch will run) of up to SAMPLES of its pieces under every candidate setting --
block-Jacobi sweeps before and after each coarse correction (the reference does one,
statics/src/bodies.rs:386, 396-401) and the stencil tile (the window of parts grouped
by axis) -- and keeps the fastest setting that solved every sample. A batch iterates
until its slowest piece converges, so timing single pieces misjudges a setting: two
sweeps per level cut the mean iteration count but can leave a straggler (the damped-
Jacobi step 4/(3 lambda_max) is the reference's choice for one sweep; on some pieces
two sweeps lose definiteness and CG stalls), so a setting counts only if all its
samples converge within TRIAL_MAX_ITER iterations. Choices are
cached in a JSON file keyed by class, precision and tolerance, so a later batch of the
same classes is not tuned again. A piece that still fails in the batched solve is
solved again alone with the reference's one sweep (its info then says retried).
"""
from __future__ import annotations

import json
import os
import time

from . import FP64, MIXED, Solver, options

SWEEPS = (1, 2)
TILES = (256, 1024, 4096)
SAMPLES = 8
TRIAL_MAX_ITER = 2000
MAX_ITER = 20000
FALLBACK = {"sweeps": 1, "tile": 0}
DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_cache.json")


def converged(info: dict, tol: float) -> bool:
    """The solve met its criterion (the recursively updated residual at tol) and its true
    residual, recomputed in FP64, is within rounding of the recurrence of it (2 tol)."""
    return info["status"] == 0 and info["residual"] <= 2.0 * tol


def size_class(state) -> int:
    cells = int(state.size)
    c = 1
    while c < cells:
        c <<= 1
    return c


def _key(cls: int, precision: int, tol: float) -> str:
    return f"batch:{cls}:{precision}:{tol:g}"


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


def tune_class(solver: Solver, samples, precision: int = MIXED, tol: float = 1e-8, repeats: int = 2) -> dict:
    """Times a batched solve of the sample pieces under every (sweeps, tile); returns the
    fastest setting that solved all of them, with the timings (the reference's setting if
    none did)."""
    trials = []
    for sweeps in SWEEPS:
        for tile in TILES:
            opt = options(tol=tol, precision=precision, sweeps=sweeps, tile=tile, max_iter=TRIAL_MAX_ITER)
            best, iters = float("inf"), []
            for _ in range(repeats):
                t = time.perf_counter()
                _, infos = solver.solve_grid_batch(samples, opt)
                dt = time.perf_counter() - t
                iters = [i["iterations"] for i in infos]
                if any(not converged(i, tol) for i in infos):
                    dt = float("inf")
                    best = dt
                    break
                best = min(best, dt)
            trials.append({"sweeps": sweeps, "tile": tile, "seconds": best, "iterations": iters})
    ok = [t for t in trials if t["seconds"] < float("inf")]
    if not ok:
        return dict(FALLBACK, seconds=None, trials=trials)
    win = min(ok, key=lambda t: t["seconds"])
    return {"sweeps": win["sweeps"], "tile": win["tile"], "seconds": win["seconds"], "trials": trials}


def choose(solver: Solver, pieces, precision: int = MIXED, tol: float = 1e-8, path: str = DEFAULT_CACHE) -> dict:
    """The setting for each size class present in `pieces` (tuning the classes the cache
    lacks on up to SAMPLES of their pieces). Returns {class: {"sweeps": s, "tile": t, ...}}."""
    cache = load(path)
    classes: dict[int, list] = {}
    for piece in pieces:
        classes.setdefault(size_class(piece[0]), []).append(piece)
    out, changed = {}, False
    for cls, members in classes.items():
        key = _key(cls, precision, tol)
        if key not in cache:
            cache[key] = tune_class(solver, members[:SAMPLES], precision, tol)
            changed = True
        out[cls] = cache[key]
    if changed:
        save(cache, path)
    return out


def solve_batch(solver: Solver, pieces, precision: int = MIXED, tol: float = 1e-8, path: str = DEFAULT_CACHE,
                settings: dict | None = None):
    """Solves `pieces` with their size classes' tuned settings: the pieces that share a
    setting form one batched solve (fewer, larger batches than one per class); a piece
    that did not converge is solved again alone with the reference's setting. Returns
    (motions, infos) in the order of `pieces`."""
    settings = settings or choose(solver, pieces, precision, tol, path)
    groups: dict[tuple, list[int]] = {}
    for i, p in enumerate(pieces):
        s = settings.get(size_class(p[0]), FALLBACK)
        groups.setdefault((s["sweeps"], s["tile"]), []).append(i)
    motions, infos = [None] * len(pieces), [None] * len(pieces)
    for (sweeps, tile), idx in groups.items():
        opt = options(tol=tol, precision=precision, sweeps=sweeps, tile=tile, max_iter=MAX_ITER)
        outs, inf = solver.solve_grid_batch([pieces[i] for i in idx], opt)
        for j, i in enumerate(idx):
            motions[i], infos[i] = outs[j], inf[j]
    fallback = options(tol=tol, precision=precision, sweeps=FALLBACK["sweeps"], tile=FALLBACK["tile"],
                       max_iter=MAX_ITER)
    for i, info in enumerate(infos):
        if not converged(info, tol):
            motions[i], infos[i] = solver.solve_grid(*pieces[i], fallback)
            infos[i]["retried"] = True
    return motions, infos
