"""The C-ABI library without a GPU: it loads, exports every entry point
include/statics_cuda.h declares, and its host-only helpers behave."""
import ctypes
import os
import re

import numpy as np
import pytest

import statics_cuda as sc
from oracle import oracle as O

from helpers import oracle_lattice, piece

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "statics_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sc_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(sc.LIB_PATH)
    names = declared()
    assert len(names) >= 13
    for name in names:
        assert hasattr(lib, name), name


def test_generated_pieces():
    st, k = piece(24, 7)
    assert st.shape == (24, 24, 24)
    assert (st[:, :, 0] == sc.CELL_HELD).all()
    assert ((st[:, :, 1:] == sc.CELL_FREE) | (st[:, :, 1:] == sc.CELL_EMPTY)).all()
    occ = k[st > 0]
    assert occ.min() >= 0.5 and occ.max() <= 2.0
    assert (k[st == 0] == 0).all()
    st2, k2 = piece(24, 7)
    assert (st == st2).all() and (k == k2).all()
    st3, _ = piece(24, 8)
    assert (st != st3).any()
    # every kept cell is joined to the support (a 6-connected flood from z = 0)
    keep = st > 0
    seen = np.zeros_like(keep)
    seen[:, :, 0] = True
    frontier = list(zip(*np.nonzero(seen)))
    while frontier:
        nxt = []
        for x, y, z in frontier:
            for dx, dy, dz in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
                a, b, c = x + dx, y + dy, z + dz
                if 0 <= a < 24 and 0 <= b < 24 and 0 <= c < 24 and keep[a, b, c] and not seen[a, b, c]:
                    seen[a, b, c] = True
                    nxt.append((a, b, c))
        frontier = nxt
    assert (seen == keep).all()


def test_lognormal_pieces():
    st, k = piece(16, 3, sc.K_LOGNORMAL)
    occ = k[st > 0]
    assert occ.min() >= 0.1 and occ.max() <= 10.0
    assert 0.7 < np.exp(np.log(occ).mean()) < 1.4


def test_fill_ratio_near_half():
    st, _ = piece(64, 0)
    assert 0.4 < (st[:, :, 1:] > 0).mean() < 0.6


@pytest.mark.parametrize("seed", [0, 1, 5])
def test_grid_count_matches_build(seed):
    st, k = piece(12, seed)
    lat = oracle_lattice(st, k)
    ex = lat.export()
    n, p = sc.grid_count(st)
    assert n == lat.n_nodes
    assert p == int((ex["held"] == 0).sum())


def test_no_device_is_a_status_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sc.StaticsError) as e:
        sc.Solver(0)
    assert e.value.status == sc.NO_DEVICE


def test_status_strings():
    lib = sc.lib()
    for s in range(8):
        assert lib.sc_status_string(s)


def test_mech_levels_rejects_missing_outputs():
    """sc_mech_levels writes steps (and sizes when max_levels > 0): NULL there is
    SC_BAD_INPUT, never a write through a null pointer."""
    st, k = piece(8, 1)
    s = sc.mech_voxel_system(st, k * 1e9, h=0.125, dt=1 / 60, mass=2000 * 0.125 ** 3)
    arrs = [np.ascontiguousarray(s[name], dt) for name, dt in
            (("sites", np.int64), ("at", np.float64), ("diag", np.float64), ("pi", np.uint32), ("pj", np.uint32),
             ("pb", np.float64))]
    ptr = [a.ctypes.data_as(ctypes.c_void_p) for a in arrs]
    n, npairs = len(arrs[0]), len(arrs[3])
    lib = sc.lib()
    nl = ctypes.c_int32()
    sizes, steps = np.zeros(4, np.int64), np.zeros(5)
    args = (n, ptr[0], ptr[1], ptr[2], npairs, ptr[3], ptr[4], ptr[5], ctypes.c_double(0.125))
    assert lib.sc_mech_levels(*args, 4, sizes.ctypes.data_as(ctypes.c_void_p), None, ctypes.byref(nl)) == sc.BAD_INPUT
    assert lib.sc_mech_levels(*args, 4, None, steps.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nl)) == sc.BAD_INPUT
    # a count-only query: no sizes, steps[0] only
    assert lib.sc_mech_levels(*args, 0, None, steps.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nl)) == sc.OK
    assert nl.value >= 1
