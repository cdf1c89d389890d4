"""Autotuner for batched solves of voxel pieces.

A batch iterates until its slowest piece converges (converged pieces skip their work but
ride along), so the setting that matters is the one for the batch as a whole, and one
batch beats several: per-size-class settings would split the batch into one solve per
setting, each as slow as its worst member. So the tuner times a batched solve (setup +
PCG to the requested tolerance, as the batch will run) of a sample of the batch -- up to
SAMPLES pieces spread evenly over its size range -- under every candidate setting:
block-Jacobi sweeps before and after each coarse correction (the reference does one,
statics/src/bodies.rs:386, 396-401) and the level-0 stencil (sc_options.tile: 0 the
brick stencil, whose iterations run in brick order, or the per-part stencil in the
reference's part order with a window of 1024 parts grouped by axis). It keeps the fastest setting that solved every sample: two sweeps per level cut
the mean iteration count but can leave a straggler (the damped-Jacobi step 4/(3
lambda_max) is the reference's choice for one sweep; on some pieces two sweeps lose
definiteness and CG stalls), so a setting counts only if all its samples converge within
TRIAL_MAX_ITER iterations. Choices are cached in a JSON file keyed by the batch's size
classes, precision and tolerance, so a later batch of the same classes is not tuned
again. A piece that fails in the batched solve under a setting other than the
reference's is solved again alone with the reference's one sweep (its info then says
retried).
"""
from __future__ import annotations

import json
import os
import time

from . import FP64, MIXED, Solver, options

SWEEPS = (1, 2)
TILES = (0, 1024)  # the brick stencil (brick order), the per-part stencil (the reference's order)
SAMPLES = 32
TRIAL_MAX_ITER = 2000
MAX_ITER = 20000
FALLBACK = {"sweeps": 1, "tile": 0}
DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_cache.json")


def converged(info: dict, tol: float) -> bool:
    """The solve met its criterion: status OK and its true residual |b - K x| / |b|,
    recomputed in FP64, at most tol (up to the rounding of that ratio), or at most the
    piece's FP64 floor (info["residual_floor"]: the residual rounding x to FP64 leaves,
    which no FP64 vector of motions gets under). The solver holds every piece to this,
    replacing a drifted recursive residual by the true one."""
    return info["status"] == 0 and info["residual"] <= max(tol, info.get("residual_floor", 0.0)) * (1.0 + 1e-9)


def above_tol_at_floor(info: dict, tol: float) -> bool:
    """Converged at its FP64 floor, which lies above tol."""
    return converged(info, tol) and info["residual"] > tol * (1.0 + 1e-9)


def size_class(state) -> int:
    cells = int(state.size)
    c = 1
    while c < cells:
        c <<= 1
    return c


def _key(classes, precision: int, tol: float) -> str:
    return "batch:" + "-".join(str(c) for c in sorted(set(classes))) + f":{precision}:{tol:g}"


def sample(pieces, count: int = SAMPLES) -> list:
    """Up to `count` of `pieces`, spread evenly over them in order of size."""
    order = sorted(range(len(pieces)), key=lambda i: int(pieces[i][0].size))
    if len(order) <= count:
        return [pieces[i] for i in order]
    step = (len(order) - 1) / (count - 1)
    return [pieces[order[round(j * step)]] for j in range(count)]


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


def tune(solver: Solver, samples, precision: int = MIXED, tol: float = 1e-8, repeats: int = 2) -> dict:
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
                if any(i["status"] != 0 for i in infos):
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
    """The setting for a batch of `pieces` (tuned on a sample of them unless the cache has
    one for the same size classes). Returns {"sweeps": s, "tile": t, ...}."""
    cache = load(path)
    key = _key([size_class(p[0]) for p in pieces], precision, tol)
    if key not in cache:
        cache[key] = tune(solver, sample(pieces), precision, tol)
        save(cache, path)
    return cache[key]


def solve_batch(solver: Solver, pieces, precision: int = MIXED, tol: float = 1e-8, path: str = DEFAULT_CACHE,
                setting: dict | None = None):
    """Solves `pieces` in one batched solve with the batch's tuned setting; a piece that
    failed (a status other than OK) under a setting other than the reference's is solved
    again alone with the reference's setting. Returns (motions, infos) in the order of
    `pieces`."""
    setting = setting or choose(solver, pieces, precision, tol, path)
    opt = options(tol=tol, precision=precision, sweeps=setting["sweeps"], tile=setting["tile"], max_iter=MAX_ITER)
    motions, infos = solver.solve_grid_batch(pieces, opt)
    motions, infos = list(motions), list(infos)
    if (setting["sweeps"], setting["tile"]) != (FALLBACK["sweeps"], FALLBACK["tile"]):
        fallback = options(tol=tol, precision=precision, sweeps=FALLBACK["sweeps"], tile=FALLBACK["tile"],
                           max_iter=MAX_ITER)
        for i, info in enumerate(infos):
            if info["status"] != 0:
                motions[i], infos[i] = solver.solve_grid(*pieces[i], fallback)
                infos[i]["retried"] = True
    return motions, infos
