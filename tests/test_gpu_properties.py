"""Size-independent checks at the benchmark's full size (128^3, ~20 M DOF), where the
oracle would take minutes: the compliance identity of the adjoint and the agreement of
the precisions.

For the solution u of K u = f, C = f.u = u'Ku = 2 sum_c U_c, and dC/dk_c = -2 U_c / k_c
(every cell's stiffness scales its block linearly), so sum_c k_c dC/dk_c = -C: an
identity between the compliance the solve reports and the per-cell strain-energy
gather, off only by the solve's residual."""
import numpy as np
import pytest

import statics_cuda as sc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol,bar", [(sc.FP64, 1e-10, 1e-8), (sc.MIXED, 1e-8, 1e-6)],
                         ids=["fp64", "mixed"])
def test_compliance_identity_128cubed(solver, precision, tol, bar):
    st, k = sc.generate_piece(128, 128, 128, 0, sc.K_UNIFORM)
    C, grad, u, info = solver.compliance_grad(st, k, sc.options(tol=tol, precision=precision, max_iter=20000))
    assert info["status"] == sc.OK
    # CG stops on its recursively updated residual; the FP64 true residual it reports can
    # exceed tol by the recurrence's rounding (1.3e-10 at 1e-10 on this piece)
    assert info["residual"] <= 2 * tol
    s = float((k.astype(np.float64) * grad).sum())
    assert abs(s + C) <= bar * abs(C)


def test_precisions_agree_128cubed(solver):
    """Mixed and FP64 motions at 1e-8 within the displacement bar (1e-6 relative)."""
    st, k = sc.generate_piece(128, 128, 128, 0, sc.K_UNIFORM)
    u64, i64 = solver.solve_grid(st, k, sc.options(tol=1e-10))
    u32, i32 = solver.solve_grid(st, k, sc.options(tol=1e-8, precision=sc.MIXED))
    assert i64["status"] == sc.OK and i32["status"] == sc.OK
    assert np.linalg.norm(u32 - u64) <= 1e-6 * np.linalg.norm(u64)


@pytest.mark.slow
def test_compliance_identity_lognormal_192cubed(solver):
    """The large configuration's generator (lognormal k) at 192^3 (~63 GB of device memory)."""
    st, k = sc.generate_piece(192, 192, 192, 0, sc.K_LOGNORMAL)
    C, grad, u, info = solver.compliance_grad(st, k, sc.options(tol=1e-8, precision=sc.MIXED, max_iter=20000))
    assert info["status"] == sc.OK
    s = float((k.astype(np.float64) * grad).sum())
    assert abs(s + C) <= 1e-6 * abs(C)
