"""ORACLE — test infrastructure only.

ctypes front end of the CPU restatement of the reference's `statics` solve
(statics/src/{model,lattice,bodies}.rs) and its coarse-level gather
(statics/src/gather.rs), built from oracle/*.cpp into
oracle/_build/liboracle.so by oracle/Makefile). Only tests/, the smoke check and
bench.py's CPU legs (the CPU baseline and reference arm; the probes' CPU timings, and the
reference's scenes the gather probe measures) import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

STONE, WOOD, MASONRY, SOIL, STEEL, LEAVES = range(6)

_lib = None


def build() -> str:
    """Compile the restatement (a no-op when the library is up to date)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, D, I64, I32, U8 = C.c_void_p, C.c_double, C.c_int64, C.c_int32, C.c_uint8
        pd, pi64, pi32, pu8, pf = (C.POINTER(D), C.POINTER(I64), C.POINTER(I32), C.POINTER(U8),
                                   C.POINTER(C.c_float))
        L.or_scene.restype = P
        L.or_scene.argtypes = [C.c_int, C.c_int, D, D, D, C.c_int]
        L.or_grid.restype = P
        L.or_grid.argtypes = [C.c_int, C.c_int, C.c_int, pu8, pf, D, D]
        L.or_free.argtypes = [P]
        L.or_sizes.argtypes = [P, pi64, pi64]
        L.or_export.argtypes = [P, pd, pd, pu8, pi64, pi64, pi64, pd, pd, pd, pd, pd, pd, pi64]
        L.or_motions.restype = C.c_int
        L.or_motions.argtypes = [P, pu8, pu8, pd, D, I64, I64, pd, pd, pi64, pd, pi64, pi64, pd, I64, pi64,
                                 pi32, I64]
        L.or_moved.argtypes = [P, pd, pd]
        L.or_cell_energy.argtypes = [P, pd, I64, pd]
        L.or_used_standing.argtypes = [P, pd]
        L.or_settle.argtypes = [P, pd, pi64, pu8]
        L.or_strengths.argtypes = [P, pd, pd, pd]
        L.or_as_generated.argtypes = [P, P]
        L.or_clone.restype = P
        L.or_clone.argtypes = [P]
        L.or_level0_apply.argtypes = [P, I64, pd, pd]
        L.or_invert.argtypes = [pd, pd]
        L.or_coarse_site.argtypes = [pi64, C.c_uint32, pi64]
        L.or_coarse_site.restype = I64
        L.or_block.restype = P
        L.or_block.argtypes = [C.c_int, pd, pd, pd, C.c_int]
        L.or_gather.restype = P
        L.or_gather.argtypes = [P, C.c_int]
        L.or_full.argtypes = [C.c_int, pd]
        L.or_materials.argtypes = [P, pi32, pi32, pd]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_threads.restype = C.c_int
        L.or_generate_piece.restype = C.c_int
        L.or_generate_piece.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, pu8, pf]
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def threads() -> int:
    return int(lib().or_threads())


K_UNIFORM, K_LOGNORMAL = 0, 1
CELL_EMPTY, CELL_FREE, CELL_HELD = 0, 1, 2


def generate_piece(nx: int, ny: int, nz: int, seed: int, k_dist: int = K_UNIFORM):
    """The benchmark's seeded synthetic piece (generate_oracle.cpp): state (nx, ny, nz)
    uint8 of CELL_* and k float32, made without the product library."""
    state = np.zeros((nx, ny, nz), np.uint8)
    k = np.zeros((nx, ny, nz), np.float32)
    rc = lib().or_generate_piece(nx, ny, nz, seed, k_dist, _p(state, C.c_uint8), _p(k, C.c_float))
    if rc != 0:
        raise ValueError(f"bad piece dimensions {nx} x {ny} x {nz}")
    return state, k


class Lattice:
    """A level's nodes and bonds, held by the restatement (lattice.rs:61-71)."""

    def __init__(self, handle):
        if not handle:
            raise ValueError("oracle returned no lattice")
        self.h = handle
        n, b = C.c_int64(), C.c_int64()
        lib().or_sizes(self.h, C.byref(n), C.byref(b))
        self.n_nodes, self.n_bonds = n.value, b.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_free(self.h)
            self.h = None

    @classmethod
    def scene(cls, kind: str, mat: int = STONE, a: float = 0, b: float = 0, c: float = 0, level: int = 0):
        kinds = {"cantilever": 0, "tree": 1, "portico": 2, "rock": 3, "tower": 4, "pendant": 5}
        return cls(lib().or_scene(kinds[kind], mat, a, b, c, level))

    @classmethod
    def block(cls, mat: int, lo, hi, half, level: int = 0):
        """Every site of solids(level, lo, hi) whose centre lies strictly inside the box
        |x_k| < half[k], of material `mat`, free (lattice.rs:87-163)."""
        lo, hi, half = (np.ascontiguousarray(v, dtype=np.float64) for v in (lo, hi, half))
        lat = cls(lib().or_block(int(mat), _p(lo, C.c_double), _p(hi, C.c_double), _p(half, C.c_double), level))
        lat.level = level
        return lat

    @classmethod
    def grid(cls, state: np.ndarray, k: np.ndarray, g_over_e: float = 0.4, rho: float = 512.0):
        state = np.ascontiguousarray(state, dtype=np.uint8)
        k = np.ascontiguousarray(k, dtype=np.float32)
        nx, ny, nz = state.shape
        lat = cls(lib().or_grid(nx, ny, nz, _p(state, C.c_uint8), _p(k, C.c_float), g_over_e, rho))
        lat.grid_shape = (nx, ny, nz)
        return lat

    def export(self) -> dict:
        n, b = self.n_nodes, self.n_bonds
        out = dict(x=np.zeros((n, 3)), m=np.zeros(n), held=np.zeros(n, np.uint8), around=np.zeros((n, 2, 3), np.int64),
                   bi=np.zeros(b, np.int64), bj=np.zeros(b, np.int64), p=np.zeros((b, 3)), n=np.zeros((b, 3)),
                   a=np.zeros(b), d=np.zeros(b), e=np.zeros(b), g=np.zeros(b), cell=np.zeros(b, np.int64))
        lib().or_export(self.h, _p(out["x"], C.c_double), _p(out["m"], C.c_double), _p(out["held"], C.c_uint8),
                        _p(out["around"], C.c_int64), _p(out["bi"], C.c_int64), _p(out["bj"], C.c_int64),
                        _p(out["p"], C.c_double), _p(out["n"], C.c_double), _p(out["a"], C.c_double),
                        _p(out["d"], C.c_double), _p(out["e"], C.c_double), _p(out["g"], C.c_double),
                        _p(out["cell"], C.c_int64))
        return out

    def motions(self, loads: np.ndarray, alive=None, gone=None, tol=1e-6, few=64, max_iter=100000,
                hierarchy=False, max_levels=64):
        """bodies.rs:429-468: each node's motion under `loads` (n_nodes x 6)."""
        loads = np.ascontiguousarray(loads, dtype=np.float64).reshape(self.n_nodes, 6)
        out = np.zeros((self.n_nodes, 6))
        work = C.c_double()
        iters = C.c_int64()
        secs = np.zeros(3)
        counts = np.zeros(max_levels, np.int64)
        pairs = np.zeros(max_levels, np.int64)
        steps = np.zeros(max_levels)
        nlev = C.c_int64()
        up_cap = 2 * self.n_nodes + 16 if hierarchy else 0
        up = np.zeros(up_cap, np.int32) if hierarchy else None
        al = None if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        gn = None if gone is None else np.ascontiguousarray(gone, dtype=np.uint8)
        lib().or_motions(self.h, _p(al, C.c_uint8), _p(gn, C.c_uint8), _p(loads, C.c_double), tol, few, max_iter,
                         _p(out, C.c_double), C.byref(work), C.byref(iters), _p(secs, C.c_double),
                         _p(counts, C.c_int64), _p(pairs, C.c_int64), _p(steps, C.c_double), max_levels,
                         C.byref(nlev), _p(up, C.c_int32), up_cap)
        info = dict(work=work.value, iterations=iters.value, seconds=secs[0], setup_seconds=secs[1],
                    solve_seconds=secs[2])
        nl = nlev.value
        info["counts"] = counts[:nl].tolist()
        info["pairs"] = pairs[:nl].tolist()
        info["steps"] = steps[:nl].tolist()
        if hierarchy:
            ups, pos = [], 0
            for l in range(nl - 1):
                c = info["counts"][l]
                ups.append(up[pos:pos + c].copy())
                pos += c
            info["up"] = ups
        return out, info

    def moved(self, x: np.ndarray) -> np.ndarray:
        f = np.zeros((self.n_bonds, 3))
        x = np.ascontiguousarray(x, dtype=np.float64)
        lib().or_moved(self.h, _p(x, C.c_double), _p(f, C.c_double))
        return f

    def cell_energy(self, x: np.ndarray, n_cells: int) -> np.ndarray:
        e = np.zeros(n_cells)
        x = np.ascontiguousarray(x, dtype=np.float64)
        lib().or_cell_energy(self.h, _p(x, C.c_double), n_cells, _p(e, C.c_double))
        return e

    def strengths(self) -> dict:
        """Each bond's tensile, compressive and shear strength (its material's)."""
        b = self.n_bonds
        out = dict(ft=np.zeros(b), fc=np.zeros(b), fs=np.zeros(b))
        lib().or_strengths(self.h, _p(out["ft"], C.c_double), _p(out["fc"], C.c_double), _p(out["fs"], C.c_double))
        return out

    def used_standing(self) -> np.ndarray:
        u = np.zeros(self.n_bonds)
        lib().or_used_standing(self.h, _p(u, C.c_double))
        return u

    def settle(self):
        fallen = C.c_double()
        rounds = C.c_int64()
        gone = np.zeros(self.n_nodes, np.uint8)
        lib().or_settle(self.h, C.byref(fallen), C.byref(rounds), _p(gone, C.c_uint8))
        return fallen.value, rounds.value, gone

    def as_generated(self, generated: "Lattice") -> None:
        """bodies.rs:611-625: each bond's strength no less than MARGIN times what the same
        beam of `generated` uses standing (in place)."""
        lib().or_as_generated(self.h, generated.h)

    def copy(self) -> "Lattice":
        lat = Lattice(lib().or_clone(self.h))
        lat.level = getattr(self, "level", 0)
        return lat

    def gathered(self, against_full: bool = True) -> "Lattice":
        """gather.rs:193-195 (or measured(fine, false), gather.rs:230-395): the next
        level up, each coarse cell's beams measured from this lattice's matter."""
        lat = Lattice(lib().or_gather(self.h, 1 if against_full else 0))
        lat.level = getattr(self, "level", 0) + 1
        return lat

    def materials(self) -> dict:
        """Per node its material (index into STONE..LEAVES, -1 other); per bond its
        material and its strength over the material's own (Mat::stronger)."""
        out = dict(node=np.zeros(self.n_nodes, np.int32), bond=np.zeros(self.n_bonds, np.int32),
                   stronger=np.zeros(self.n_bonds))
        lib().or_materials(self.h, _p(out["node"], C.c_int32), _p(out["bond"], C.c_int32),
                           _p(out["stronger"], C.c_double))
        return out

    def level0_apply(self, x_parts: np.ndarray) -> np.ndarray:
        x_parts = np.ascontiguousarray(x_parts, dtype=np.float64)
        y = np.zeros_like(x_parts)
        lib().or_level0_apply(self.h, x_parts.shape[0], _p(x_parts, C.c_double), _p(y, C.c_double))
        return y


def full(mat: int) -> np.ndarray:
    """gather.rs:203-226: a full cell of `mat` measured a level up, by class (180°,
    90°): rows of (section / s^2, strength / the material's)."""
    out = np.zeros(4)
    lib().or_full(int(mat), _p(out, C.c_double))
    return out.reshape(2, 2)


def invert(m: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(m, dtype=np.float64)
    out = np.zeros((6, 6))
    lib().or_invert(_p(m, C.c_double), _p(out, C.c_double))
    return out


def coarse_site(p, l: int):
    a = np.ascontiguousarray(p, dtype=np.int64)
    out = np.zeros(3, np.int64)
    lib().or_coarse_site(_p(a, C.c_int64), l, _p(out, C.c_int64))
    return tuple(int(v) for v in out)
