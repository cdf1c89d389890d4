"""The engine's solver on the GPU (sc_mech_solve: mechanics::solve::Solver, solve.rs)
against its CPU oracle on voxel pieces at rest: the same levels, the rounds within two,
motions within 1e-7 of the oracle's solve to 1e-12, a warm start from the answer taking
no round."""
import numpy as np
import pytest

import statics_cuda as sc
from oracle import mechanics as M

pytestmark = pytest.mark.gpu


def _system(n, E, seed=4):
    st, k = sc.generate_piece(n, n, n, seed, sc.K_UNIFORM)
    return M.system(st, k * E, h=0.125, dt=1 / 60, mass=2000 * 0.125 ** 3)


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
