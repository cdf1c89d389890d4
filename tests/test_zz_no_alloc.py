"""sc_compliance_noalloc — compliance of motions already on the device, for callers that
cannot let the library allocate device memory (an engine that owns the GPU's memory,
a frame loop that cannot stall on cudaMalloc). Its result
must match the compliance sc_compliance_grad reports for the same solve, call after
call, although it keeps its partial sums in one array shared by every call.

Named to be collected last, so a run that stops at its first failure has run every
other test before this one."""
import numpy as np
import pytest

import statics_cuda as sc

from helpers import oracle_lattice, piece, z_loads

pytestmark = pytest.mark.gpu


def test_noalloc_compliance_matches_compliance_grad():
    import torch

    st, k = piece(24, 2)
    solver = sc.Solver(0)
    C, _, u, _ = solver.compliance_grad(st, k, sc.options(tol=1e-12, max_iter=5000))
    solver.close()
    loads, _ = z_loads(oracle_lattice(st, k))  # the piece's loads, node order (input data)
    f_d = torch.from_numpy(np.ascontiguousarray(loads.ravel())).cuda()
    u_d = torch.from_numpy(np.ascontiguousarray(u.ravel())).cuda()
    assert f_d.numel() == u_d.numel() > 8192  # several chunks of the shared array
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for i in range(2):  # two calls in a row, the second over the first's partial sums
        s = sc.compliance_noalloc(f_d.data_ptr(), u_d.data_ptr(), f_d.numel(), out.data_ptr() + 8 * i, stream)
        assert s == sc.OK
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert got[0] == pytest.approx(C, rel=1e-9)
    assert got[1] == pytest.approx(C, rel=1e-9)
    assert got[0] == got[1]  # deterministic


def test_noalloc_rejects_sizes_past_its_array():
    import torch

    f = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    s = sc.compliance_noalloc(f.data_ptr(), f.data_ptr(), sc.NOALLOC_MAX_VALUES + 1, out.data_ptr(), 0)
    assert s == sc.BAD_INPUT
