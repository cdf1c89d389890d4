"""GPU path against the oracle, through the C ABI: bit-exact numbering and hierarchy,
operator values, motions, mixed precision, batches, general lattices, statuses."""
import hashlib
import json
import os

import numpy as np
import pytest

import statics_cuda as sc
from oracle import oracle as O

from helpers import lattice_dict, oracle_lattice, piece, rel, z_loads

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))

# FP64 operator values differ from the oracle's only by summation order.
OP_TOL64 = 1e-12
OP_TOL32 = 2e-6
# Displacements at 1e-8 relative residual: both solves are within ~kappa * 1e-8 of the
# exact answer; the GPU's differs from the oracle's by far less.
DISP_TOL = 1e-6


def special_pieces():
    out = []
    st = np.zeros((1, 1, 2), np.uint8)
    st[0, 0, 0], st[0, 0, 1] = 2, 1  # one free cell on the support
    out.append(("one cell", st, np.ones(st.shape, np.float32)))
    st = np.zeros((1, 1, 6), np.uint8)
    st[0, 0, 0], st[0, 0, 1:] = 2, 1  # a column
    out.append(("column", st, np.linspace(0.5, 2, st.size, dtype=np.float32).reshape(st.shape)))
    st = np.zeros((5, 4, 3), np.uint8)
    st[:, :, 0] = 2
    st[1:4, 1:3, 1:] = 1  # a block, empty ring around it
    out.append(("block", st, np.full(st.shape, 1.5, np.float32)))
    st = np.zeros((4, 4, 4), np.uint8)
    st[:, :, 0] = 2
    st[:, :, 1] = 1
    st[1, 1, 2] = 2  # a held cell in the middle of free ones
    st[2, 2, 2:] = 1
    out.append(("held inside", st, np.full(st.shape, 0.7, np.float32)))
    return out


@pytest.mark.parametrize("n,seed", [(8, 0), (12, 3), (16, 1), (20, 5)])
@pytest.mark.parametrize("tile", [0, 1024], ids=["bricks", "per-part"])
def test_operator_matches_level_new_apply(solver, n, seed, tile):
    """The iterations' brick stencil (tile 0) and the setup's per-part stencil (tile
    1024) against the oracle's Level::new + Level::apply."""
    st, k = piece(n, seed, shape=(n, n + 3, n - 2))
    lat = oracle_lattice(st, k)
    _, parts = sc.grid_count(st)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((parts, 6))
    want = lat.level0_apply(x)
    got = solver.grid_apply(st, k, x, sc.FP64, tile=tile)
    assert rel(got, want) < OP_TOL64
    got32 = solver.grid_apply(st, k, x, sc.MIXED, tile=tile)
    assert rel(got32, want) < OP_TOL32


@pytest.mark.parametrize("shape,seed", [((8, 16, 16), 2), ((4, 8, 8), 5), ((9, 17, 15), 1), ((32, 8, 24), 7),
                                        ((3, 5, 70), 4)])
def test_brick_stencil_shapes(solver, shape, seed):
    """The brick stencil on pieces whose edges are multiples of the 4 x 8 x 8 bricks (so
    the last bricks own the + boundary faces as extra slots), one brick, ragged ones, and
    a thin column: every part against the oracle's operator, FP64 and FP32."""
    st, k = piece(0, seed, shape=shape)
    lat = oracle_lattice(st, k)
    _, parts = sc.grid_count(st)
    x = np.random.default_rng(seed).standard_normal((parts, 6))
    want = lat.level0_apply(x)
    got = solver.grid_apply(st, k, x, sc.FP64)
    assert rel(got, want) < OP_TOL64
    # per part, not only in the norm: each row's error against the largest row's size
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    assert rel(solver.grid_apply(st, k, x, sc.MIXED), want) < OP_TOL32


@pytest.mark.parametrize("name,st,k", special_pieces(), ids=[p[0] for p in special_pieces()])
def test_operator_special_pieces(solver, name, st, k):
    lat = oracle_lattice(st, k)
    _, parts = sc.grid_count(st)
    x = np.random.default_rng(1).standard_normal((parts, 6))
    assert rel(solver.grid_apply(st, k, x), lat.level0_apply(x)) < OP_TOL64


def _solve_both(solver, st, k, tol, precision=sc.FP64):
    lat = oracle_lattice(st, k)
    loads, ex = z_loads(lat)
    u_ref, info_ref = lat.motions(loads, tol=tol, hierarchy=True)
    u, info = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=tol, precision=precision))
    return lat, u_ref, info_ref, u, info


@pytest.mark.parametrize("n,seed", [(16, 0), (16, 1), (24, 3), (32, 0), (32, 2)])
def test_hierarchy_bit_exact_and_motions(solver, n, seed):
    st, k = piece(n, seed)
    lat, u_ref, ir, u, info = _solve_both(solver, st, k, 1e-8)
    assert info["status"] == sc.OK
    assert info["parts"] == ir["counts"]
    assert info["blocks"][1:] == [2 * p + c for p, c in zip(ir["pairs"][1:], ir["counts"][1:])]
    for l, up_ref in enumerate(ir["up"]):
        up = solver.last_up(l, len(up_ref))
        assert (up == up_ref).all(), f"level {l}"
    assert np.allclose(info["steps"], ir["steps"], rtol=1e-9)
    assert abs(info["iterations"] - ir["iterations"]) <= 1
    assert rel(u, u_ref) < DISP_TOL
    assert info["residual"] <= 1e-8 * 1.0001


@pytest.mark.parametrize("name,st,k", special_pieces(), ids=[p[0] for p in special_pieces()])
def test_motions_special_pieces(solver, name, st, k):
    lat, u_ref, ir, u, info = _solve_both(solver, st, k, 1e-10)
    assert info["parts"] == ir["counts"]
    assert rel(u, u_ref) < 1e-8


def test_mixed_precision_against_fp64(solver):
    """SC_MIXED (FP64 CG, FP32 V-cycle) and SC_MIXED_FP32_KRYLOV (FP32 CG with FP64
    residual replacement) both reach the tolerance on the FP64 true residual and the
    oracle's FP64 motions; the FP32 V-cycle leaves the iteration count near FP64's."""
    st, k = piece(32, 1)
    lat = oracle_lattice(st, k)
    loads, ex = z_loads(lat)
    u_ref, _ = lat.motions(loads, tol=1e-12)
    u64, i64 = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=1e-8))
    assert rel(u64, u_ref) < DISP_TOL
    u32, i32 = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=1e-8, precision=sc.MIXED))
    assert i32["status"] == sc.OK
    assert i32["residual"] <= 1e-8 * 1.0001
    assert i32["iterations"] <= 1.5 * i64["iterations"] + 2
    assert rel(u32, u_ref) < DISP_TOL
    uk, ik = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=1e-8, precision=sc.MIXED_FP32_KRYLOV))
    assert ik["status"] == sc.OK
    assert ik["residual"] <= 1e-8 * 1.0001
    assert ik["refinements"] >= 1
    assert rel(uk, u_ref) < DISP_TOL


def test_mixed_precision_hard_piece(solver):
    """A 16 x 16 x 24 piece on which the all-FP32 Krylov recurrence breaks down: the
    FP32 V-cycle inside FP64 CG converges like FP64."""
    st, k = sc.generate_piece(16, 16, 24, 10_017, sc.K_UNIFORM)
    _, i64 = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=1e-8))
    u, info = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=1e-8, precision=sc.MIXED))
    assert info["status"] == sc.OK
    assert info["residual"] <= 1e-8 * 1.0001
    assert info["iterations"] <= i64["iterations"] + 5
    lat = oracle_lattice(st, k)
    loads, _ = z_loads(lat)
    u_ref, _ = lat.motions(loads, tol=1e-12)
    assert rel(u, u_ref) < DISP_TOL


def test_golden_large(solver):
    """Pieces whose oracle solve takes minutes, against its committed outputs."""
    cases = [c for c in json.load(open(os.path.join(HERE, "golden", "oracle_pieces.json"))) if c["n"] >= 48]
    for c in cases:
        st, k = piece(c["n"], c["seed"])
        u, info = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=c["tol"]))
        assert info["parts"] == c["counts"], c["n"]
        for l, h in enumerate(c["up_hash"]):
            up = solver.last_up(l, c["counts"][l])
            assert hashlib.sha256(up.astype(np.int32).tobytes()).hexdigest()[:16] == h
        assert abs(info["iterations"] - c["iterations"]) <= 1
        assert np.linalg.norm(u) == pytest.approx(c["u_norm"], rel=DISP_TOL)
        idx = np.asarray(c["sample_idx"])
        assert np.allclose(u.ravel()[idx], c["sample_u"], rtol=0, atol=DISP_TOL * c["u_norm"] / np.sqrt(u.size) * 50)


def test_batch_matches_single_solves(solver):
    rng = np.random.default_rng(7)
    sizes = [16, 24, 32]
    pieces = []
    for i in range(6):
        shape = tuple(int(v) for v in rng.choice(sizes, 3))
        pieces.append(piece(0, 100 + i, shape=shape))
    outs, infos = solver.solve_grid_batch(pieces, sc.options(max_iter=5000, tol=1e-8))
    for (st, k), u, info in zip(pieces, outs, infos):
        lat = oracle_lattice(st, k)
        loads, _ = z_loads(lat)
        u_ref, ir = lat.motions(loads, tol=1e-8)
        assert info["parts"] == ir["counts"]
        assert abs(info["iterations"] - ir["iterations"]) <= 1
        assert rel(u, u_ref) < DISP_TOL


def test_batch_mixed(solver):
    pieces = [piece(0, 200 + i, shape=(16 + 8 * (i % 3), 24, 16 + 16 * (i % 2))) for i in range(8)]
    outs, infos = solver.solve_grid_batch(pieces, sc.options(max_iter=5000, tol=1e-8, precision=sc.MIXED))
    for (st, k), u, info in zip(pieces, outs, infos):
        lat = oracle_lattice(st, k)
        loads, _ = z_loads(lat)
        u_ref, _ = lat.motions(loads, tol=1e-12)
        assert info["residual"] <= 1e-8 * 1.0001
        assert rel(u, u_ref) < DISP_TOL


@pytest.mark.parametrize("env", [{}, {"SC_GALERKIN": "rows"},
                                 {"SC_GALERKIN": "rows", "SC_ROWS_VARIANT": "0"},
                                 {"SC_GALERKIN": "rows", "SC_ROWS_VARIANT": "1"},
                                 {"SC_GALERKIN": "rows", "SC_ROWS_VARIANT": "2"},
                                 {"SC_GALERKIN": "rows", "SC_ROWS_SLOTS": "3", "SC_ROWS_META": "5"},
                                 {"SC_GALERKIN": "sort", "SC_UPPER_SLICE": "20000"}],
                         ids=["default", "rows", "rows-64", "rows-192", "rows-areg", "rows-tiled", "sort-sliced"])
def test_galerkin_rows_match_sorted(solver, monkeypatch, env):
    """The row-by-row Galerkin products (pieces with at most 65536 coarse parts a level)
    and the sorted-candidate ones add the same products in the same order: the same
    bits, for a single piece and a batch, with the default choice per product and with
    every product row by row (level 0's K P then reads the cell template). Tiles of 3
    output blocks and 5 staged entries split a row over many blocks and walk it often.
    The sorted upper products made in slices of coarse rows (at most 20000 candidates a
    slice) give the same bits as made at once."""
    opts = sc.options(max_iter=5000, tol=1e-8)
    st, k = piece(0, 11, shape=(40, 28, 36))
    batch = [piece(0, 300 + i, shape=(16 + 8 * (i % 3), 24, 20)) for i in range(4)]
    for name, v in env.items():
        monkeypatch.setenv(name, v)
    u_rows, i_rows = solver.solve_grid(st, k, opts)
    b_rows, bi_rows = solver.solve_grid_batch(batch, opts)
    for name in env:
        monkeypatch.delenv(name)
    monkeypatch.setenv("SC_GALERKIN", "sort")
    u_sort, i_sort = solver.solve_grid(st, k, opts)
    b_sort, bi_sort = solver.solve_grid_batch(batch, opts)
    assert i_rows["status"] == sc.OK
    assert i_rows["iterations"] == i_sort["iterations"]
    assert i_rows["steps"] == i_sort["steps"]
    assert np.array_equal(u_rows, u_sort)
    for a, b, ia, ib in zip(b_rows, b_sort, bi_rows, bi_sort):
        assert ia["iterations"] == ib["iterations"]
        assert np.array_equal(a, b)


@pytest.mark.parametrize("tile", [1, 2, 32, 1024, 4096])
@pytest.mark.parametrize("precision", [sc.FP64, sc.MIXED], ids=["fp64", "mixed"])
def test_stencil_variants(solver, tile, precision):
    """The level-0 stencils sc_options.tile selects (1: the plane-pencil stencil; 2: the
    two-pass cell-then-part stencil; a power of two: the per-part stencil in the
    reference's part order with that axis-grouping window) apply the same operator as the
    default brick stencil: the
    same hierarchy and iterations as the default, motions within the displacement bar of
    the oracle's. The shape is ragged against the pencil's 16 x 8 x 32 blocks."""
    st, k = piece(0, 41, shape=(37, 21, 45))
    lat = oracle_lattice(st, k)
    loads, _ = z_loads(lat)
    u_ref, _ = lat.motions(loads, tol=1e-12)
    u0, i0 = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=1e-8, precision=precision))
    u, info = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=1e-8, precision=precision, tile=tile))
    assert info["status"] == sc.OK
    assert info["parts"] == i0["parts"]
    assert abs(info["iterations"] - i0["iterations"]) <= 1
    assert rel(u, u_ref) < DISP_TOL
    if precision == sc.FP64:
        x = np.random.default_rng(2).standard_normal((sc.grid_count(st)[1], 6))
        assert rel(solver.grid_apply(st, k, x, tile=tile), lat.level0_apply(x)) < OP_TOL64


@pytest.mark.parametrize("sweeps", [2, 3])
def test_more_sweeps(solver, sweeps):
    """Several block-Jacobi sweeps before and after each coarse correction (the
    reference does one): a different preconditioner, the same solution."""
    st, k = piece(32, 2)
    lat = oracle_lattice(st, k)
    loads, _ = z_loads(lat)
    u_ref, _ = lat.motions(loads, tol=1e-12)
    u, info = solver.solve_grid(st, k, sc.options(max_iter=5000, tol=1e-8, sweeps=sweeps))
    if info["status"] == sc.OK:
        assert rel(u, u_ref) < DISP_TOL
    else:  # more sweeps of the reference's damping can lose definiteness; it must say so
        assert info["status"] in (sc.MAXITER, sc.BREAKDOWN)


def test_autotuned_batch(solver, tmp_path):
    """The autotuner's batched solve: every piece converges (a failed group member is
    solved again with the reference's setting) and matches the oracle."""
    from statics_cuda import autotune
    pieces = [piece(0, 300 + i, shape=(16 + 8 * (i % 2), 16, 24 - 8 * (i % 3 == 0))) for i in range(6)]
    outs, infos = autotune.solve_batch(solver, pieces, sc.MIXED, 1e-8, path=str(tmp_path / "cache.json"))
    for (st, k), u, info in zip(pieces, outs, infos):
        assert info["status"] == sc.OK
        assert info["residual"] <= 1e-8 * 1.0001
        lat = oracle_lattice(st, k)
        loads, _ = z_loads(lat)
        u_ref, _ = lat.motions(loads, tol=1e-12)
        assert rel(u, u_ref) < DISP_TOL


SCENES = [
    ("cantilever", dict(kind="cantilever", mat=O.STONE, a=0.5, b=4.0)),
    ("cantilever 6", dict(kind="cantilever", mat=O.STONE, a=0.5, b=6.0)),
    ("portico", dict(kind="portico", a=1, b=0.5)),
    ("tree 70", dict(kind="tree", a=8.0, b=-1.0, c=0.7)),
]


@pytest.mark.parametrize("name,kw", SCENES, ids=[s[0] for s in SCENES])
def test_general_lattice_motions(solver, name, kw):
    lat = O.Lattice.scene(**kw)
    ex = lat.export()
    loads = np.zeros((lat.n_nodes, 6))
    loads[:, 1] = -ex["m"] * 9.81
    u_ref, ir = lat.motions(loads, tol=1e-10, hierarchy=True)
    w = sc.Work()
    u = solver.motions(lattice_dict(ex), None, None, loads, w, sc.options(max_iter=5000, tol=1e-10))
    assert w.status == sc.OK
    assert w.info["parts"] == ir["counts"]
    assert rel(u, u_ref) < 1e-7


def test_general_lattice_alive_and_gone(solver):
    lat = O.Lattice.scene("pendant", a=0)
    ex = lat.export()
    rng = np.random.default_rng(4)
    alive = np.ones(lat.n_bonds, np.uint8)
    beams = rng.choice(lat.n_bonds // 4, size=lat.n_bonds // 40, replace=False)
    for b in beams:
        alive[4 * b:4 * b + 4] = 0
    gone = np.zeros(lat.n_nodes, np.uint8)
    loads = np.zeros((lat.n_nodes, 6))
    loads[:, 1] = -ex["m"] * 9.81
    u_ref, ir = lat.motions(loads, alive=alive, gone=gone, tol=1e-10, hierarchy=True)
    w = sc.Work()
    u = solver.motions(lattice_dict(ex), alive, gone, loads, w, sc.options(max_iter=5000, tol=1e-10))
    assert w.info["parts"] == ir["counts"]
    assert rel(u, u_ref) < 1e-7


def test_compliance_gradient(solver):
    st, k = piece(12, 2)
    C, grad, u, info = solver.compliance_grad(st, k, sc.options(max_iter=5000, tol=1e-12))
    lat = oracle_lattice(st, k)
    loads, ex = z_loads(lat)
    u_ref, _ = lat.motions(loads, tol=1e-12)
    assert C == pytest.approx(float((loads * u_ref).sum()), rel=1e-9)
    energy = lat.cell_energy(u_ref, st.size).reshape(st.shape)
    free = st == 1
    want = np.where(free, -2 * energy / np.where(free, k, 1), 0)
    assert rel(grad, want) < 1e-8


def test_statuses(solver):
    st, k = piece(12, 0)
    u, info = solver.solve_grid(st, k, sc.options(tol=1e-8, max_iter=0))
    assert info["status"] == sc.MAXITER
    assert np.abs(u).max() == 0.0
    bad = k.copy()
    bad[st == 1] = np.nan
    u, info = solver.solve_grid(st, bad, sc.options(max_iter=5000, tol=1e-8))
    assert info["status"] in (sc.BREAKDOWN, sc.NOT_SPD)
    with pytest.raises(sc.StaticsError) as e:
        solver.solve_grid(st, k, sc.options(max_iter=5000, tol=-1.0))
    assert e.value.status == sc.BAD_INPUT


def test_timeout_status(solver):
    """A 64^3 solve given 1 ms ends with SC_TIMEOUT (the host looks at the clock between
    launches of the device-side loop), and the context still solves afterwards."""
    st, k = piece(64, 0)
    with pytest.raises(sc.StaticsError) as e:
        solver.solve_grid(st, k, sc.options(tol=1e-8, timeout_ms=1))
    assert e.value.status == sc.TIMEOUT
    _, info = solver.solve_grid(*piece(16, 0), sc.options(tol=1e-8))
    assert info["status"] == sc.OK


@pytest.mark.parametrize("precision", [sc.FP64, sc.MIXED])
def test_unsupported_piece_is_not_ok(solver, precision):
    """Nothing held: K is singular (every rigid motion strains no bond) and gravity has a
    part along those motions, so no x meets the tolerance. The solve must say so (a
    non-positive pivot at the top, a breakdown or the cap), never SC_OK."""
    st = np.ones((8, 8, 8), np.uint8)
    k = np.full(st.shape, 1.0, np.float32)
    try:
        _, info = solver.solve_grid(st, k, sc.options(tol=1e-8, max_iter=300, precision=precision))
        status = info["status"]
    except sc.StaticsError as e:
        status = e.status
    assert status in (sc.NOT_SPD, sc.BREAKDOWN, sc.MAXITER)


def test_solve_grid_into_caller_buffer(solver):
    """solve_grid(out=...) writes the motions into the caller's array (a larger one too)
    and gives the same values as a new array; the C ABI turns down one too small
    (SC_BAD_INPUT)."""
    st, k = piece(16, 0)
    opt = sc.options(max_iter=5000, tol=1e-8)
    u, _ = solver.solve_grid(st, k, opt)
    buf = np.full((u.shape[0] + 3, 6), np.nan)
    u2, info = solver.solve_grid(st, k, opt, out=buf)
    assert info["status"] == sc.OK
    assert np.shares_memory(u2, buf)
    assert np.array_equal(u, u2)
    with pytest.raises(sc.StaticsError):
        solver.solve_grid(st, k, opt, out=np.zeros((2, 6)))


@pytest.mark.parametrize("precision", [sc.FP64, sc.MIXED], ids=["fp64", "mixed"])
def test_residual_replacement_and_fp64_floor(solver, precision):
    """Two pieces of the bench's batch (edges 16 x 24 x 64, seed 10256; 16 x 16 x 48, seed
    10324). On the first the CG recursion drifts from b - K x: the recursive residual meets
    1e-8 while the true one does not, so the solve replaces it by the true residual and
    goes on, ending below 1e-8. On the second no FP64 vector of motions has a residual
    below about 5e-8 |b| (the oracle's own solve at a recursive 1e-13 ends there, and
    moving x by one unit in the last place gives as much): the solve stops at that floor,
    which it reports, with status OK. Both against the oracle's motions at 1e-12."""
    for shape, seed, floored in (((16, 24, 64), 10256, False), ((16, 16, 48), 10324, True)):
        st, k = sc.generate_piece(*shape, seed, sc.K_UNIFORM)
        u, info = solver.solve_grid(st, k, sc.options(max_iter=20000, tol=1e-8, precision=precision))
        assert info["status"] == sc.OK
        assert info["residual"] <= max(1e-8, info["residual_floor"]) * (1 + 1e-9)
        if floored:
            assert info["residual_floor"] > 1e-8
        else:
            assert info["residual"] <= 1e-8 * (1 + 1e-9)
        lat = oracle_lattice(st, k)
        loads, _ = z_loads(lat)
        u_ref, _ = lat.motions(loads, tol=1e-12, max_iter=20000)
        assert rel(u, u_ref) < DISP_TOL
