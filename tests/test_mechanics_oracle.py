"""The CPU restatement of the engine's solver, mechanics::solve::Solver
(mechanics/src/solve.rs), and of its unit cell element (mechanics/src/element.rs): the
element against the reference's own element test, the assembled system's structure, and
the solver's stopping rule and warm start. (No GPU: this is the checker a GPU port of the
solver will be held to.)"""
import numpy as np
import pytest

import statics_cuda as sc
from oracle import mechanics as M

CORNERS = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]]
NU = 0.3


def _forces(K, u):
    return np.einsum("acij,cj->ai", K, u)


def test_unit_cube_as_the_reference_tests_it():
    """element.rs:171-187: moved rigidly the cube holds nothing back; pulled along x by a
    thousandth, free across, the far face's force over the stretch is E (= 1) within 1e-6.
    (The reference moves the corners and lets the element find its turn; unturned, the
    motion is the corners' displacement.)"""
    K = M.unit_stiffness()
    assert np.allclose(K, K.transpose(1, 0, 3, 2), rtol=0, atol=1e-15)  # K_ac = K_ca'
    t = np.array([3.0, -1.0, 2.0])
    assert np.abs(_forces(K, np.tile(t, (8, 1)))).max() < 1e-14
    w = np.array([0.3, -0.2, 0.5]) * 1e-3  # a small turn: u = w x (p - middle)
    u = np.array([np.cross(w, np.array(c, float) - 0.5) for c in CORNERS])
    assert np.abs(_forces(K, u)).max() < 1e-16
    u = np.array([[(c[0] - 0.5) * 1e-3, -(c[1] - 0.5) * NU * 1e-3, -(c[2] - 0.5) * NU * 1e-3] for c in CORNERS])
    pull = sum(_forces(K, u)[a][0] for a in range(8) if CORNERS[a][0] == 1)
    assert abs(pull / 1e-3 - 1.0) < 1e-6


def test_one_cell_system():
    """A free cell on a held one: its four upper corners are the unknowns, six pairs."""
    st = np.zeros((1, 1, 2), np.uint8)
    st[0, 0, 0], st[0, 0, 1] = 2, 1
    s = M.system(st, np.ones(st.shape, np.float32), h=1.0, dt=1.0, mass=8.0)
    assert len(s["sites"]) == 4 and len(s["pi"]) == 6
    assert (s["sites"][:, 2] == 2).all()  # the corners at z = 2; z = 1 touches the held cell
    assert (s["pi"] < s["pj"]).all()
    # each corner: mass 1 plus its stiffness (dt^2 + 0.3 dt) E h K_aa
    K = M.unit_stiffness()
    assert np.allclose(s["diag"][0], np.eye(3) + 1.3 * K[4, 4])
    assert np.allclose(s["b"], np.tile([0.0, -9.81, 0.0], (4, 1)))


@pytest.mark.parametrize("n,seed", [(8, 0), (12, 3)])
def test_system_symmetric_positive(n, seed):
    st, k = sc.generate_piece(n, n + 2, n, seed, sc.K_UNIFORM)
    s = M.system(st, k * 1e8, h=0.125, dt=1 / 60, mass=4.0)
    rng = np.random.default_rng(seed)
    a, c = rng.standard_normal(s["b"].shape), rng.standard_normal(s["b"].shape)
    sa, sc_ = M.times(s, a), M.times(s, c)
    assert abs(np.sum(c * sa) - np.sum(a * sc_)) <= 1e-12 * abs(np.sum(c * sa))
    assert np.sum(a * sa) > 0


@pytest.mark.parametrize("E", [1e6, 1e9])
def test_solver_converges_and_warm_starts(E):
    """PCG to the energy-norm tolerance (solve.rs:468-538); the levels coarsen to a
    direct top; solved again from its answer it takes no round."""
    st, k = sc.generate_piece(16, 16, 16, 2, sc.K_UNIFORM)
    s = M.system(st, k * E, h=0.125, dt=1 / 60, mass=2000 * 0.125 ** 3)
    x, rounds, sizes, step = M.solve(s, tol=1e-8)
    assert 0 < rounds < 300
    assert all(a > b for a, b in zip([len(s["sites"])] + sizes, sizes))
    assert 0 < step < 4 / 3 * 1.0001
    r = s["b"] - M.times(s, x)
    assert np.linalg.norm(r) <= 1e-6 * np.linalg.norm(s["b"])
    _, again, _, _ = M.solve(s, x0=x, tol=1e-8)
    assert again == 0


@pytest.mark.parametrize("n,seed", [(6, 0), (12, 5)])
def test_library_system_matches_oracle(n, seed):
    """The library's voxel system (sc_mech_voxel_system, host code: no GPU) is the
    oracle's, value for value."""
    st, k = sc.generate_piece(n, n + 1, n, seed, sc.K_UNIFORM)
    a = M.system(st, k * 1e8, h=0.125, dt=1 / 60, mass=2.0)
    b = sc.mech_voxel_system(st, k * 1e8, h=0.125, dt=1 / 60, mass=2.0)
    for key in ("sites", "at", "diag", "pi", "pj", "pb", "b"):
        assert a[key].shape == b[key].shape, key
        assert np.array_equal(a[key], b[key]), key


@pytest.mark.parametrize("n,E,seed", [(10, 1e6, 0), (16, 1e9, 4), (20, 1e9, 7)])
def test_library_levels_match_oracle(n, E, seed):
    """The levels the library makes on the host for the GPU solve (sc_mech_levels, no
    device) are the oracle's Solver::new: the same parts on every level and the same
    smoother steps, bit for bit (the same additions in the same order)."""
    st, k = sc.generate_piece(n, n, n + 2, seed, sc.K_UNIFORM)
    s = sc.mech_voxel_system(st, k * E, h=0.125, dt=1 / 60, mass=2000 * 0.125 ** 3)
    sizes, steps = sc.mech_levels(s)
    want_sizes, want_steps = M.levels(s)
    assert [int(v) for v in sizes] == [int(v) for v in want_sizes]
    assert steps == want_steps
