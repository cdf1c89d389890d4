"""The engine's solver on the GPU (sc_mech_solve: mechanics::solve::Solver, solve.rs)
against its CPU oracle on voxel pieces at rest: the levels made on the device equal the
oracle's (and the library's host copy's) bit for bit, the rounds within two, motions
within 1e-7 of the oracle's solve to 1e-12, a warm start from the answer taking no
round."""
import numpy as np
import pytest

import statics_cuda as sc
from oracle import mechanics as M

pytestmark = pytest.mark.gpu


def _system(n, E, seed=4):
    st, k = sc.generate_piece(n, n, n, seed, sc.K_UNIFORM)
    return M.system(st, k * E, h=0.125, dt=1 / 60, mass=2000 * 0.125 ** 3)


@pytest.mark.parametrize("n,E,seed", [(10, 1e6, 0), (16, 1e9, 4), (20, 1e9, 7), (32, 1e9, 1)])
def test_device_levels_match_oracle(solver, n, E, seed):
    """Solver::new on the device (sc_mech_levels_on): the same parts on every level and
    the same smoother steps as the oracle and as the host copy (sc_mech_levels), bit for
    bit."""
    st, k = sc.generate_piece(n, n, n + 2, seed, sc.K_UNIFORM)
    s = sc.mech_voxel_system(st, k * E, h=0.125, dt=1 / 60, mass=2000 * 0.125 ** 3)
    sizes, steps = solver.mech_levels(s)
    host_sizes, host_steps = sc.mech_levels(s)
    assert [int(v) for v in sizes] == [int(v) for v in host_sizes]
    assert steps == host_steps
    if n <= 20:
        want_sizes, want_steps = M.levels(s)
        assert [int(v) for v in sizes] == [int(v) for v in want_sizes]
        assert steps == want_steps


@pytest.mark.parametrize("n,E", [(10, 1e6), (16, 1e9), (20, 1e9)])
def test_mech_solve_matches_oracle(solver, n, E):
    s = _system(n, E)
    x_ref, r_ref, sizes, _ = M.solve(s, tol=1e-8)
    x_tight, _, _, _ = M.solve(s, tol=1e-12)
    x, rounds, levels = solver.mech_solve(s, tol=1e-8)
    assert levels == len(sizes)
    assert 0 < rounds < 300 and abs(rounds - r_ref) <= 2
    assert np.linalg.norm(x - x_tight) <= 1e-7 * np.linalg.norm(x_tight)
    r = s["b"] - M.times(s, x)
    assert np.linalg.norm(r) <= 1e-6 * np.linalg.norm(s["b"])
    _, again, _ = solver.mech_solve(s, x0=x, tol=1e-8)
    assert again == 0


def test_mech_solve_rejects_bad_pairs(solver):
    s = _system(6, 1e6)
    bad = dict(s, pi=s["pi"].copy())
    bad["pi"][0] = bad["pj"][0]  # a pair with itself
    with pytest.raises(sc.StaticsError):
        solver.mech_solve(bad)
