"""The compliance adjoint (sc_compliance_grad): dC/dk_c = -2 U_c / k_c against central
finite differences of C = f.u (relative step 1e-4) and against the FP64 CPU adjoint the
oracle computes from its own motions (Bond::energy per cell, statics/src/model.rs:132-136).

The central difference (C(k+) - C(k-)) / (k+ - k-) is evaluated as f.(u+ - u-), with
u+ - u- solved directly: K+ (u+ - u-) = (K- - K+) u-, a right-hand side that lives on the
one cell's faces. Subtracting two compliances of a 96^3 piece instead would lose the
difference (one voxel moves C by ~1e-9 of itself) in the rounding of C."""
import numpy as np
import pytest

import statics_cuda as sc

from helpers import oracle_lattice, piece, z_loads

pytestmark = pytest.mark.gpu

H = 1e-4          # relative finite-difference step
FD_TOL = 1e-5     # gradient against finite differences
CPU_TOL = 1e-8    # gradient against the CPU adjoint (same FP64 quantity)


def _fd(solver, st, k, cells, opt, f_nodes, free_nodes):
    out = []
    delta_opt = sc.options(tol=1e-11, max_iter=20000)
    for c in cells:
        kp, km = k.copy(), k.copy()
        kp.flat[c] = np.float32(k.flat[c] * (1 + H))
        km.flat[c] = np.float32(k.flat[c] * (1 - H))
        dk = float(kp.flat[c]) - float(km.flat[c])  # the step k actually took in float32
        u_m, _ = solver.solve_grid(st, km, opt)
        x = u_m[free_nodes]
        rhs = np.zeros_like(u_m)
        rhs[free_nodes] = solver.grid_apply(st, km, x) - solver.grid_apply(st, kp, x)
        delta, info = solver.solve_grid(st, kp, delta_opt, loads=rhs)
        assert info["status"] == sc.OK
        out.append(float((f_nodes * delta).sum()) / dk)
    return np.array(out)


def _check(solver, n, seed, n_cells, with_cpu):
    st, k = piece(n, seed)
    opt = sc.options(tol=1e-13, max_iter=20000)
    C, grad, u, info = solver.compliance_grad(st, k, opt)
    assert info["status"] == sc.OK
    free = np.flatnonzero(st.ravel() == sc.CELL_FREE)
    rng = np.random.default_rng(1000 + seed)
    cells = rng.choice(free, size=min(n_cells, free.size), replace=False)
    lat = oracle_lattice(st, k)
    f_nodes, ex = z_loads(lat)
    fd = _fd(solver, st, k, cells, opt, f_nodes, ex["held"] == 0)
    g = grad.ravel()[cells]
    err = np.abs(g - fd) / np.abs(fd)
    assert err.max() < FD_TOL, err.max()
    assert (grad.ravel()[st.ravel() != sc.CELL_FREE] == 0).all()
    if with_cpu:
        u_ref, _ = lat.motions(f_nodes, tol=1e-12)
        energy = lat.cell_energy(u_ref, st.size)
        want = np.where(st.ravel() == sc.CELL_FREE, -2 * energy / np.where(k.ravel() > 0, k.ravel(), 1), 0)
        assert np.abs(grad.ravel() - want).max() <= CPU_TOL * np.abs(want).max()


def test_adjoint_against_finite_differences(solver):
    _check(solver, 16, 3, 16, with_cpu=True)


@pytest.mark.slow
def test_adjoint_96cubed_64_voxels(solver):
    """The adjoint configuration: a 96^3 piece, 64 seeded occupied voxels."""
    _check(solver, 96, 0, 64, with_cpu=True)
