"""ORACLE -- test infrastructure only. ctypes access to the CPU restatement of the
engine's solver, mechanics::solve::Solver (mechanics/src/solve.rs), and of the unit cell
element it is assembled from (mechanics/src/element.rs), built into
oracle/_build/liboracle.so (mechanics_oracle.cpp). Only tests may use it, as the
checker of a GPU port."""
import ctypes as C
import os

import numpy as np

from .oracle import lib as _lib  # the one liboracle.so

_I64 = C.POINTER(C.c_int64)
_F64 = C.POINTER(C.c_double)
_U32 = C.POINTER(C.c_uint32)


def _p(a, t):
    return a.ctypes.data_as(t)


def unit_stiffness() -> np.ndarray:
    """K[a][c] (3 x 3) of the unit cube of stiffness 1 between corners a and c (element.rs:44-69)."""
    k = np.zeros((8, 8, 3, 3))
    _lib().mo_unit_stiffness(_p(k, _F64))
    return k


def system(state, e, h=1.0, dt=1.0 / 60.0, mass=1.0) -> dict:
    """The system of a voxel piece at rest (lib.rs:638-676): every free cell an 8-node
    element welded to its free neighbours, corners touching a held cell held; unknowns
    the other nodes in first-touch order; pairs in first-encounter order. Returns sites,
    at, diag (n x 3 x 3), pairs (pi, pj, pb: m x 3 x 3) and b (n x 3)."""
    state = np.ascontiguousarray(state, np.uint8)
    e = np.ascontiguousarray(e, np.float32)
    nx, ny, nz = state.shape
    lib = _lib()
    n, m = C.c_int64(), C.c_int64()
    null = C.c_void_p()
    lib.mo_system(_p(state, C.POINTER(C.c_uint8)), _p(e, C.POINTER(C.c_float)), nx, ny, nz, C.c_double(h),
                  C.c_double(dt), C.c_double(mass), C.byref(n), C.byref(m), None, None, None, None, None, None, None)
    n, m = n.value, m.value
    s = {"sites": np.zeros((n, 3), np.int64), "at": np.zeros((n, 3)), "diag": np.zeros((n, 3, 3)),
         "pi": np.zeros(m, np.uint32), "pj": np.zeros(m, np.uint32), "pb": np.zeros((m, 3, 3)), "b": np.zeros((n, 3)),
         "h": h}
    nn, mm = C.c_int64(), C.c_int64()
    lib.mo_system(_p(state, C.POINTER(C.c_uint8)), _p(e, C.POINTER(C.c_float)), nx, ny, nz, C.c_double(h),
                  C.c_double(dt), C.c_double(mass), C.byref(nn), C.byref(mm), _p(s["sites"], _I64), _p(s["at"], _F64),
                  _p(s["diag"], _F64), _p(s["pi"], _U32), _p(s["pj"], _U32), _p(s["pb"], _F64), _p(s["b"], _F64))
    return s


def _args(s):
    return (C.c_int64(len(s["sites"])), _p(s["sites"], _I64), _p(s["at"], _F64), _p(s["diag"], _F64),
            C.c_int64(len(s["pi"])), _p(s["pi"], _U32), _p(s["pj"], _U32), _p(s["pb"], _F64))


def times(s, x) -> np.ndarray:
    """y = S x (solve.rs:63-73)."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros_like(x)
    _lib().mo_times(*_args(s), _p(x, _F64), _p(y, _F64))
    return y


def solve(s, b=None, x0=None, tol=1e-8, size=None):
    """Solver::new(s, size) then solve(s, b, x, tol) from x0 (zeros by default)
    (solve.rs:356-538). Returns (x, rounds or -1, coarse level sizes, fine step)."""
    b = np.ascontiguousarray(s["b"] if b is None else b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64, copy=True)
    sizes = np.zeros(64, np.int64)
    nl = C.c_int()
    step = C.c_double()
    lib = _lib()
    lib.mo_solve.restype = C.c_int
    rounds = lib.mo_solve(*_args(s), _p(b, _F64), _p(x, _F64), C.c_double(tol), C.c_double(size or s["h"]), 64,
                          _p(sizes, _I64), C.byref(nl), C.byref(step))
    return x, rounds, list(sizes[:nl.value]), step.value


def levels(s, size=None):
    """Solver::new only: (coarse level sizes, steps: the nodes' then each level's, 0 at a
    direct top)."""
    sizes, steps = np.zeros(64, np.int64), np.zeros(65)
    lib = _lib()
    lib.mo_levels.restype = C.c_int
    nl = lib.mo_levels(*_args(s), C.c_double(size or s["h"]), 64, _p(sizes, _I64), _p(steps, _F64))
    return list(sizes[:nl]), list(steps[:nl + 1])
