"""statics_cuda — Python host side of the B200 statics solver.

A ctypes front end over libstatics_cuda.so (include/statics_cuda.h), mirroring the
reference's solve API (SupraSummus/parallax-world, statics/src/bodies.rs):

* ``motions(lattice, alive, gone, loads, work)`` answers ``statics::bodies::motions``
  (bodies.rs:429): each node's 6-DOF motion, held and gone nodes at rest. Like the
  reference it returns the motions even when the solve stops at the iteration cap or
  breaks down; the outcome is on ``work.status`` (the reference has no error channel).
* ``Work`` mirrors bodies.rs:331 (``work.v`` is the reference's counter).
* ``solve_grid`` / ``solve_grid_batch`` / ``compliance_grad`` are the voxel-piece fast
  path, the batched path and the compliance adjoint.

There is no CPU fallback: without the built library or an sm_100 device these raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstatics_cuda.so")

OK, MAXITER, BREAKDOWN, NOT_SPD, BAD_INPUT, TIMEOUT, CUDA, NO_DEVICE = range(8)
CELL_EMPTY, CELL_FREE, CELL_HELD = 0, 1, 2
K_UNIFORM, K_LOGNORMAL = 0, 1
FP64, MIXED, MIXED_FP32_KRYLOV = 0, 1, 2
MAX_LEVELS = 24
(FAM_STENCIL64, FAM_STENCIL32, FAM_SPMV64, FAM_SPMV32, FAM_TRANSFER64, FAM_TRANSFER32, FAM_SMOOTH64,
 FAM_SMOOTH32, FAM_TOP) = range(9)
FAM_NAMES = ["stencil64", "stencil32", "spmv64", "spmv32", "transfer64", "transfer32", "smooth64", "smooth32",
             "top"]

STATUS_NAMES = {OK: "ok", MAXITER: "maxiter", BREAKDOWN: "breakdown", NOT_SPD: "not_spd",
                BAD_INPUT: "bad_input", TIMEOUT: "timeout", CUDA: "cuda", NO_DEVICE: "no_device"}


class StaticsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Options(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_int64), ("few", C.c_int64), ("precision", C.c_int32),
                ("sweeps", C.c_int32), ("inner_tol", C.c_double), ("timeout_ms", C.c_int64), ("tile", C.c_int32),
                ("reserved", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("refinements", C.c_int64), ("levels", C.c_int32),
                ("status", C.c_int32), ("parts", C.c_int64 * MAX_LEVELS), ("blocks", C.c_int64 * MAX_LEVELS),
                ("steps", C.c_double * MAX_LEVELS), ("residual", C.c_double), ("work", C.c_double),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double), ("n_nodes", C.c_int64),
                ("n_parts", C.c_int64), ("peak_bytes", C.c_int64), ("residual_floor", C.c_double)]

    def as_dict(self) -> dict:
        nl = self.levels
        return dict(iterations=self.iterations, refinements=self.refinements, levels=nl, status=self.status,
                    parts=list(self.parts[:nl]), blocks=list(self.blocks[:nl]), steps=list(self.steps[:nl]),
                    residual=self.residual, work=self.work, setup_ms=self.setup_ms, solve_ms=self.solve_ms,
                    n_nodes=self.n_nodes, n_parts=self.n_parts, peak_bytes=self.peak_bytes,
                    residual_floor=self.residual_floor)


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("state", C.c_void_p), ("k", C.c_void_p),
                ("g_over_e", C.c_double), ("rho", C.c_double), ("gravity", C.c_double * 3),
                ("on_device", C.c_int32), ("loads", C.c_void_p)]


class LatticeC(C.Structure):
    _fields_ = [("level", C.c_int32), ("n_nodes", C.c_int64), ("n_bonds", C.c_int64), ("x", C.c_void_p),
                ("held", C.c_void_p), ("around", C.c_void_p), ("bond_i", C.c_void_p), ("bond_j", C.c_void_p),
                ("bond_p", C.c_void_p), ("bond_n", C.c_void_p), ("bond_a", C.c_void_p), ("bond_d", C.c_void_p),
                ("bond_e", C.c_void_p), ("bond_g", C.c_void_p)]


class Strength(C.Structure):
    _fields_ = [("m", C.c_void_p), ("ft", C.c_void_p), ("fc", C.c_void_p), ("fs", C.c_void_p)]


class SettleInfo(C.Structure):
    _fields_ = [("fell", C.c_double), ("rounds", C.c_int64), ("work", C.c_double), ("status", C.c_int32),
                ("pad", C.c_int32)]


_lib = None


def lib():
    """The loaded C-ABI library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built: run __graft_entry__.build() (make -C csrc)")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.sc_default_options.argtypes = [C.POINTER(Options)]
        L.sc_status_string.restype = C.c_char_p
        L.sc_status_string.argtypes = [C.c_int]
        L.sc_create.argtypes = [C.c_int32, C.POINTER(P)]
        L.sc_destroy.argtypes = [P]
        L.sc_last_error.restype = C.c_char_p
        L.sc_last_error.argtypes = [P]
        L.sc_generate_piece.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, P, P]
        L.sc_grid_count.argtypes = [C.POINTER(Grid), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.sc_solve_grid.argtypes = [P, C.POINTER(Grid), C.POINTER(Options), P, C.c_int64, C.c_int32,
                                    C.POINTER(SolveInfo)]
        L.sc_solve_grid_batch.argtypes = [P, C.c_int32, C.POINTER(Grid), C.POINTER(Options), C.POINTER(P),
                                          C.POINTER(SolveInfo)]
        L.sc_compliance_grad.argtypes = [P, C.POINTER(Grid), C.POINTER(Options), C.POINTER(C.c_double), P, P,
                                         C.c_int64, C.POINTER(SolveInfo)]
        L.sc_grid_apply.argtypes = [P, C.POINTER(Grid), C.c_int32, P, P]
        L.sc_grid_apply_tile.argtypes = [P, C.POINTER(Grid), C.c_int32, C.c_int32, P, P]
        L.sc_last_up.argtypes = [P, C.c_int32, P, C.c_int64]
        L.sc_motions.argtypes = [P, C.POINTER(LatticeC), P, P, P, C.POINTER(Options), P, C.POINTER(SolveInfo)]
        L.sc_profile.argtypes = [P, C.c_uint32]
        L.sc_profile_read.argtypes = [P, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]
        L.sc_launches.restype = C.c_int64
        L.sc_launches.argtypes = []
        L.sc_context_stream.argtypes = [P, C.POINTER(P)]
        L.sc_mech_voxel_system.argtypes = [P, P, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                           C.c_double, C.POINTER(C.c_int64), C.POINTER(C.c_int64), P, P, P, P, P,
                                           P, P]
        L.sc_gather.argtypes = [P, C.POINTER(LatticeC), C.POINTER(Strength), P, P, C.c_int32, C.c_int32, C.c_int32,
                                C.POINTER(C.c_void_p), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.sc_gathered_read.argtypes = [P, C.POINTER(C.c_int32)] + [P] * 17
        L.sc_gathered_free.argtypes = [P]
        L.sc_gathered_free.restype = None
        L.sc_gather_full.argtypes = [P, P]
        L.sc_mech_levels.argtypes = [C.c_int64, P, P, P, C.c_int64, P, P, P, C.c_double, C.c_int32, P, P,
                                     C.POINTER(C.c_int32)]
        L.sc_mech_solve.argtypes = [P, C.c_int64, P, P, P, C.c_int64, P, P, P, P, P, C.c_double, C.c_double,
                                    C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.sc_mech_levels_on.argtypes = [P, C.c_int64, P, P, P, C.c_int64, P, P, P, C.c_double, C.c_int32, P, P,
                                        C.POINTER(C.c_int32)]
        L.sc_used_standing.argtypes = [P, C.POINTER(LatticeC), C.POINTER(Strength), C.POINTER(Options), P,
                                       C.POINTER(SolveInfo)]
        L.sc_settle.argtypes = [P, C.POINTER(LatticeC), C.POINTER(Strength), C.POINTER(Options), P,
                                C.POINTER(SettleInfo)]
        L.sc_as_generated.argtypes = [P, C.POINTER(LatticeC), C.POINTER(Strength), C.POINTER(LatticeC),
                                      C.POINTER(Strength), C.POINTER(Options), P, P, P]
        L.sc_as_generated.restype = C.c_int
        L.sc_compliance_noalloc.argtypes = [P, P, C.c_int64, P, P]
        L.sc_compliance_noalloc.restype = C.c_int
        for name in ("sc_profile", "sc_profile_read", "sc_context_stream"):
            getattr(L, name).restype = C.c_int
        for name in ("sc_create", "sc_generate_piece", "sc_grid_count", "sc_solve_grid", "sc_solve_grid_batch",
                     "sc_compliance_grad", "sc_grid_apply", "sc_grid_apply_tile", "sc_last_up", "sc_motions",
                     "sc_used_standing",
                     "sc_settle"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def options(tol=1e-6, max_iter=100000, few=64, precision=FP64, sweeps=1, inner_tol=1e-4, timeout_ms=0,
            tile=0) -> Options:
    """The reference's constants by default (bodies.rs:430-432, 351)."""
    o = Options()
    lib().sc_default_options(C.byref(o))
    o.tol, o.max_iter, o.few, o.precision = tol, max_iter, few, precision
    o.sweeps, o.inner_tol, o.timeout_ms, o.tile = sweeps, inner_tol, timeout_ms, tile
    return o


def generate_piece(nx: int, ny: int, nz: int, seed: int, k_dist: int = K_UNIFORM):
    """Seeded synthetic piece: (state uint8, k float32), each shaped (nx, ny, nz)."""
    state = np.zeros((nx, ny, nz), np.uint8)
    k = np.zeros((nx, ny, nz), np.float32)
    s = lib().sc_generate_piece(nx, ny, nz, C.c_uint64(seed), k_dist, _ptr(state), _ptr(k))
    if s != OK:
        raise StaticsError(s, "sc_generate_piece")
    return state, k


def make_grid(state: np.ndarray, k: np.ndarray, g_over_e=0.4, rho=512.0, gravity=(0.0, 0.0, -1.0),
              loads: np.ndarray | None = None) -> Grid:
    nx, ny, nz = state.shape
    g = Grid()
    g.nx, g.ny, g.nz = nx, ny, nz
    g.state, g.k = _ptr(state), _ptr(k)
    g.g_over_e, g.rho = g_over_e, rho
    g.gravity[0], g.gravity[1], g.gravity[2] = gravity
    g.on_device = 0
    g.loads = _ptr(loads)
    g._keep = (state, k, loads)
    return g


def mech_voxel_system(state, e, h: float = 0.125, dt: float = 1.0 / 60.0, mass: float = 1.0) -> dict:
    """A voxel piece at rest as the engine's system (sc_mech_voxel_system): sites, at,
    diag (n x 3 x 3), pi, pj, pb (m x 3 x 3) for the pairs, b (n x 3), h."""
    state = np.ascontiguousarray(state, np.uint8)
    e = np.ascontiguousarray(e, np.float32)
    nx, ny, nz = state.shape
    n, m = C.c_int64(), C.c_int64()
    s = lib().sc_mech_voxel_system(_ptr(state), _ptr(e), nx, ny, nz, h, dt, mass, C.byref(n), C.byref(m), None, None,
                                   None, None, None, None, None)
    if s != OK:
        raise StaticsError(s, "sc_mech_voxel_system")
    out = {"sites": np.zeros((n.value, 3), np.int64), "at": np.zeros((n.value, 3)), "diag": np.zeros((n.value, 3, 3)),
           "pi": np.zeros(m.value, np.uint32), "pj": np.zeros(m.value, np.uint32), "pb": np.zeros((m.value, 3, 3)),
           "b": np.zeros((n.value, 3)), "h": h}
    s = lib().sc_mech_voxel_system(_ptr(state), _ptr(e), nx, ny, nz, h, dt, mass, C.byref(n), C.byref(m),
                                   _ptr(out["sites"]), _ptr(out["at"]), _ptr(out["diag"]), _ptr(out["pi"]),
                                   _ptr(out["pj"]), _ptr(out["pb"]), _ptr(out["b"]))
    if s != OK:
        raise StaticsError(s, "sc_mech_voxel_system")
    return out


def mech_levels(system: dict, size: float | None = None):
    """Only the levels the engine's solver makes for `system` (sc_mech_levels, host code):
    (parts of each coarse level, smoother steps: the nodes' then each level's, 0 at the
    direct top)."""
    sites = np.ascontiguousarray(system["sites"], np.int64)
    at = np.ascontiguousarray(system["at"], np.float64)
    diag = np.ascontiguousarray(system["diag"], np.float64)
    pi = np.ascontiguousarray(system["pi"], np.uint32)
    pj = np.ascontiguousarray(system["pj"], np.uint32)
    pb = np.ascontiguousarray(system["pb"], np.float64)
    sizes, steps, nl = np.zeros(64, np.int64), np.zeros(65), C.c_int32()
    s = lib().sc_mech_levels(len(sites), _ptr(sites), _ptr(at), _ptr(diag), len(pi), _ptr(pi), _ptr(pj), _ptr(pb),
                             size or system["h"], 64, _ptr(sizes), _ptr(steps), C.byref(nl))
    if s != OK:
        raise StaticsError(s, "sc_mech_levels")
    return list(sizes[:nl.value]), list(steps[:nl.value + 1])


# The reference's materials (statics/src/model.rs:53-58): E, G, and the tensile,
# compressive and shear strengths, in the order sc_gather's tables take them.
MATERIALS = {
    "stone": (30e9, 12e9, 5e6, 100e6, 10e6),
    "wood": (10e9, 4e9, 40e6, 30e6, 6e6),
    "masonry": (5e9, 2e9, 0.2e6, 10e6, 0.4e6),
    "soil": (50e6, 20e6, 5e3, 0.3e6, 20e3),
    "steel": (200e9, 80e9, 250e6, 250e6, 145e6),
    "leaves": (0.2e9, 0.08e9, 5e6, 5e6, 1e6),
}


def _material_table(materials) -> np.ndarray:
    rows = [MATERIALS[m] if isinstance(m, str) else tuple(m) for m in materials]
    return np.ascontiguousarray(np.array(rows, np.float64).reshape(-1, 5))


def gather(lattice: dict, materials, against_full: bool = True, threads: int = 0, solver=None) -> dict:
    """statics::gather::gathered (statics/src/gather.rs:193-195), or measured(fine, false)
    with against_full=False: the next level up of `lattice` (a lattice dict with masses m,
    bond strengths ft/fc/fs and each node's material index `mat` into `materials`, a list
    of names of MATERIALS or (E, G, ft, fc, fs) rows), by sc_gather: the cells measured on
    `solver`'s device, or on the host's cores without one.
    Returns a lattice dict of the same keys, the gathered level's, with each bond's
    material index as `bmat`."""
    L, keep = _lattice_c(lattice)
    S, keep_s = _strength_c(lattice)
    table = _material_table(materials)
    node_mat = np.ascontiguousarray(lattice["mat"], np.int32)
    h, nn, nb = C.c_void_p(), C.c_int64(), C.c_int64()
    s = lib().sc_gather(solver.h if solver is not None else None, C.byref(L), C.byref(S), _ptr(node_mat), _ptr(table), len(table), 1 if against_full else 0,
                        int(threads), C.byref(h), C.byref(nn), C.byref(nb))
    if s != OK:
        if solver is not None:
            solver._check(s, "sc_gather", soft=())
        raise StaticsError(s, "sc_gather")
    try:
        n, b = nn.value, nb.value
        out = dict(x=np.zeros((n, 3)), m=np.zeros(n), held=np.zeros(n, np.uint8), around=np.zeros((n, 2, 3), np.int64),
                   mat=np.zeros(n, np.int32), bi=np.zeros(b, np.int64), bj=np.zeros(b, np.int64),
                   bmat=np.zeros(b, np.int32), p=np.zeros((b, 3)),
                   n=np.zeros((b, 3)), a=np.zeros(b), d=np.zeros(b), e=np.zeros(b), g=np.zeros(b), ft=np.zeros(b),
                   fc=np.zeros(b), fs=np.zeros(b))
        level = C.c_int32()
        lib().sc_gathered_read(h, C.byref(level), *(_ptr(out[k]) for k in
                                                     ("x", "m", "held", "around", "mat", "bi", "bj", "bmat", "p", "n", "a",
                                                      "d", "e", "g", "ft", "fc", "fs")))
        out["level"] = level.value
        return out
    finally:
        lib().sc_gathered_free(h)


def gather_full(material) -> np.ndarray:
    """gather.rs:203-226: a full cell of `material` (a name of MATERIALS or an (E, G, ft,
    fc, fs) row) measured a level up; rows (180°, 90°) of (section / s^2, strength / the
    material's). The calibration `gather` applies against a full cell."""
    table = _material_table([material])
    out = np.zeros(4)
    s = lib().sc_gather_full(_ptr(table), _ptr(out))
    if s != OK:
        raise StaticsError(s, "sc_gather_full")
    return out.reshape(2, 2)


def launches() -> int:
    """Kernels the library has launched in this process."""
    return int(lib().sc_launches())


NOALLOC_MAX_VALUES = 8192 * 65536


def compliance_noalloc(loads_ptr: int, motions_ptr: int, n_values: int, out_ptr: int, stream: int = 0) -> int:
    """C = f . u of two device arrays into a device double, allocating no device memory
    (sc_compliance_noalloc). For callers that cannot let the library allocate: engines
    that own the GPU's memory, frame loops. Returns the status; the result is ready
    when `stream` gets there."""
    return int(lib().sc_compliance_noalloc(C.c_void_p(loads_ptr), C.c_void_p(motions_ptr), n_values,
                                           C.c_void_p(out_ptr), C.c_void_p(stream or None)))


def grid_count(state: np.ndarray):
    st = np.ascontiguousarray(state, np.uint8)
    g = make_grid(st, np.zeros(st.shape, np.float32))
    n, p = C.c_int64(), C.c_int64()
    s = lib().sc_grid_count(C.byref(g), C.byref(n), C.byref(p))
    if s != OK:
        raise StaticsError(s, "sc_grid_count")
    return n.value, p.value


@dataclass
class Work:
    """The reference's Work (bodies.rs:331): parts + pairs per level apply, plus the
    outcome the reference does not report."""
    v: float = 0.0
    status: int = OK
    info: dict = field(default_factory=dict)


class Solver:
    """One solver context on one CUDA device (sc_create / sc_destroy)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        s = lib().sc_create(device, C.byref(h))
        if s != OK:
            raise StaticsError(s, "sc_create: no usable sm_100 device")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().sc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def gather(self, lattice: dict, materials, against_full: bool = True) -> dict:
        """statics::gather::gathered with the cells measured on this solver's device."""
        return gather(lattice, materials, against_full, solver=self)

    def _check(self, s: int, what: str, soft=(OK, MAXITER, BREAKDOWN, NOT_SPD)):
        if s not in soft:
            raise StaticsError(s, f"{what}: {lib().sc_last_error(self.h).decode()}")
        return s

    # ---- measurement ----------------------------------------------------------------
    def profile(self, mask: int) -> None:
        """Time the kernel families in `mask` with CUDA events on the solver's stream."""
        self._check(lib().sc_profile(self.h, mask), "sc_profile", soft=(OK,))

    def profile_read(self) -> dict:
        out = {}
        for f, name in enumerate(FAM_NAMES):
            n, ms, by = C.c_int64(), C.c_double(), C.c_double()
            self._check(lib().sc_profile_read(self.h, f, C.byref(n), C.byref(ms), C.byref(by)), "sc_profile_read",
                        soft=(OK,))
            out[name] = dict(launches=n.value, ms=ms.value, bytes=by.value)
        return out

    def stream(self) -> int:
        s = C.c_void_p()
        self._check(lib().sc_context_stream(self.h, C.byref(s)), "sc_context_stream", soft=(OK,))
        return s.value or 0

    def solve_grid_device(self, grid: Grid, opt: Options, motions_ptr: int, capacity: int):
        """A solve whose inputs (grid.state, grid.k, on_device=1) and output live in HBM."""
        info = SolveInfo()
        s = lib().sc_solve_grid(self.h, C.byref(grid), C.byref(opt), C.c_void_p(motions_ptr), capacity, 1,
                                C.byref(info))
        self._check(s, "sc_solve_grid")
        d = info.as_dict()
        d["status"] = s
        return d

    # ---- voxel pieces -------------------------------------------------------------
    def solve_grid(self, state, k, opt: Options | None = None, gravity=(0.0, 0.0, -1.0), rho=512.0, loads=None,
                   out: np.ndarray | None = None):
        """Motions of every node of a voxel piece (n_nodes x 6, reference node order);
        `loads` (n_nodes x 6) replaces mass * gravity when given. `out`, a C-contiguous
        float64 array of at least n_nodes x 6 values, receives the motions (a repeated
        solve then writes into memory it has written before); by default a new array."""
        state = np.ascontiguousarray(state, np.uint8)
        k = np.ascontiguousarray(k, np.float32)
        if loads is not None:
            loads = np.ascontiguousarray(loads, np.float64)
        g = make_grid(state, k, rho=rho, gravity=gravity, loads=loads)
        if out is None:
            n_nodes, _ = grid_count(state)
            out = np.zeros((max(n_nodes, 1), 6))
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size % 6:
            raise ValueError("out must be a C-contiguous float64 array of n x 6 values")
        out = out.reshape(-1, 6) if out.ndim != 2 else out
        info = SolveInfo()
        # the call checks out's capacity against the piece's node count (SC_BAD_INPUT)
        s = lib().sc_solve_grid(self.h, C.byref(g), C.byref(opt or options()), _ptr(out), out.size, 0,
                                C.byref(info))
        self._check(s, "sc_solve_grid")
        d = info.as_dict()
        d["status"] = s
        return out[:d["n_nodes"]], d

    def mech_levels(self, system: dict, size: float | None = None):
        """The levels the engine's solver makes on this context's device for `system`
        (sc_mech_levels_on, as mech_solve makes them): (parts of each coarse level,
        smoother steps: the nodes' then each level's, 0 at the direct top)."""
        sites = np.ascontiguousarray(system["sites"], np.int64)
        at = np.ascontiguousarray(system["at"], np.float64)
        diag = np.ascontiguousarray(system["diag"], np.float64)
        pi = np.ascontiguousarray(system["pi"], np.uint32)
        pj = np.ascontiguousarray(system["pj"], np.uint32)
        pb = np.ascontiguousarray(system["pb"], np.float64)
        sizes, steps, nl = np.zeros(64, np.int64), np.zeros(65), C.c_int32()
        s = lib().sc_mech_levels_on(self.h, len(sites), _ptr(sites), _ptr(at), _ptr(diag), len(pi), _ptr(pi),
                                    _ptr(pj), _ptr(pb), size or system["h"], 64, _ptr(sizes), _ptr(steps),
                                    C.byref(nl))
        self._check(s, "sc_mech_levels_on")
        return list(sizes[:nl.value]), list(steps[:nl.value + 1])

    def mech_solve(self, system: dict, b=None, x0=None, tol: float = 1e-3, size: float | None = None):
        """The engine's solver (mechanics::solve::Solver::new then solve, solve.rs:356-538)
        on a system given as arrays: sites (n x 3 int64), at (n x 3), diag (n x 3 x 3),
        pi, pj (uint32) and pb (m x 3 x 3) for the pairs, h (the cells' size, the
        default `size`). Solves from x0 (zeros by default) for b (the system's "b" by
        default). Returns (x, rounds or -1, coarse levels)."""
        n = len(system["sites"])
        sites = np.ascontiguousarray(system["sites"], np.int64)
        at = np.ascontiguousarray(system["at"], np.float64)
        diag = np.ascontiguousarray(system["diag"], np.float64)
        pi = np.ascontiguousarray(system["pi"], np.uint32)
        pj = np.ascontiguousarray(system["pj"], np.uint32)
        pb = np.ascontiguousarray(system["pb"], np.float64)
        b = np.ascontiguousarray(system["b"] if b is None else b, np.float64)
        x = np.zeros((n, 3)) if x0 is None else np.array(x0, np.float64, copy=True)
        rounds, levels = C.c_int32(), C.c_int32()
        s = lib().sc_mech_solve(self.h, n, _ptr(sites), _ptr(at), _ptr(diag), len(pi), _ptr(pi), _ptr(pj), _ptr(pb),
                                _ptr(b), _ptr(x), tol, size or system["h"], C.byref(rounds), C.byref(levels))
        self._check(s, "sc_mech_solve")
        return x, rounds.value, levels.value

    def solve_grid_batch(self, pieces, opt: Options | None = None):
        """pieces: list of (state, k). Returns ([motions], [info])."""
        n = len(pieces)
        grids = (Grid * n)()
        outs, keep = [], []
        for i, (st, k) in enumerate(pieces):
            st = np.ascontiguousarray(st, np.uint8)
            k = np.ascontiguousarray(k, np.float32)
            keep.append((st, k))
            g = make_grid(st, k)
            grids[i] = g
            outs.append(np.zeros((max(grid_count(st)[0], 1), 6)))
        ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        infos = (SolveInfo * n)()
        s = lib().sc_solve_grid_batch(self.h, n, grids, C.byref(opt or options()), ptrs, infos)
        self._check(s, "sc_solve_grid_batch")
        return [o[:grid_count(p[0])[0]] for o, p in zip(outs, keep)], [i.as_dict() for i in infos]

    def compliance_grad(self, state, k, opt: Options | None = None):
        """(C, dC/dk per cell (shape of the grid), motions, info)."""
        state = np.ascontiguousarray(state, np.uint8)
        k = np.ascontiguousarray(k, np.float32)
        g = make_grid(state, k)
        n_nodes, _ = grid_count(state)
        grad = np.zeros(state.shape)
        mot = np.zeros((max(n_nodes, 1), 6))
        comp = C.c_double()
        info = SolveInfo()
        s = lib().sc_compliance_grad(self.h, C.byref(g), C.byref(opt or options()), C.byref(comp), _ptr(grad),
                                     _ptr(mot), mot.size, C.byref(info))
        self._check(s, "sc_compliance_grad")
        return comp.value, grad, mot[:n_nodes], info.as_dict()

    def grid_apply(self, state, k, x_parts: np.ndarray, precision=FP64, tile: int = 0) -> np.ndarray:
        """Level 0's operator y = K x over the free nodes (n_parts x 6, part order), by the
        stencil `tile` selects (0: the brick stencil the iterations use)."""
        state = np.ascontiguousarray(state, np.uint8)
        k = np.ascontiguousarray(k, np.float32)
        g = make_grid(state, k)
        x = np.ascontiguousarray(x_parts, np.float64)
        y = np.zeros_like(x)
        s = lib().sc_grid_apply_tile(self.h, C.byref(g), precision, tile, _ptr(x), _ptr(y))
        self._check(s, "sc_grid_apply_tile", soft=(OK,))
        return y

    def last_up(self, level: int, n_parts: int) -> np.ndarray:
        up = np.zeros(n_parts, np.int32)
        s = lib().sc_last_up(self.h, level, _ptr(up), n_parts)
        self._check(s, "sc_last_up", soft=(OK,))
        return up

    # ---- general lattices: the drop-in for bodies.rs:429 ----------------------------
    def motions(self, lattice: dict, alive=None, gone=None, loads=None, work: Work | None = None,
                opt: Options | None = None) -> np.ndarray:
        """statics::bodies::motions (bodies.rs:429) for a lattice given as a dict of
        arrays: x (n,3), held (n,), around (n,2,3), bi, bj (b,), p, n (b,3), a, d, e, g (b,),
        level. `loads` is (n, 6) or a callable of the node index, as in the reference."""
        nn = int(lattice["x"].shape[0])
        if callable(loads):
            loads = np.array([loads(v) for v in range(nn)], dtype=np.float64)
        loads = np.ascontiguousarray(loads, np.float64).reshape(nn, 6)
        L, arr = _lattice_c(lattice)
        al = None if alive is None else np.ascontiguousarray(alive, np.uint8)
        gn = None if gone is None else np.ascontiguousarray(gone, np.uint8)
        out = np.zeros((nn, 6))
        info = SolveInfo()
        s = lib().sc_motions(self.h, C.byref(L), _ptr(al), _ptr(gn), _ptr(loads), C.byref(opt or options()),
                             _ptr(out), C.byref(info))
        self._check(s, "sc_motions")
        if work is not None:
            work.v += info.work
            work.status = s
            work.info = info.as_dict()
        return out


    def used_standing(self, lattice: dict, opt: Options | None = None):
        """statics::bodies::used_standing (bodies.rs:550-554): each bond's used fraction
        of its strength with everything standing under the nodes' weights. The lattice
        dict also carries m (n,) and ft, fc, fs (b,). Returns (used, info)."""
        L, arr = _lattice_c(lattice)
        S, keep = _strength_c(lattice)
        used = np.zeros(max(L.n_bonds, 1))
        info = SolveInfo()
        s = lib().sc_used_standing(self.h, C.byref(L), C.byref(S), C.byref(opt or options()), _ptr(used),
                                   C.byref(info))
        self._check(s, "sc_used_standing", soft=(OK, MAXITER))
        return used[:L.n_bonds], info.as_dict()

    def as_generated(self, lattice: dict, generated: dict, opt: Options | None = None) -> dict:
        """statics::bodies::as_generated (bodies.rs:611-625): `lattice` with each bond's
        strengths (ft, fc, fs) made what its world as generated (`generated`, a lattice
        dict with m, ft, fc, fs) needs, twice. Returns a new dict; the inputs are kept."""
        L, arr = _lattice_c(lattice)
        S, keep = _strength_c(lattice)
        G, garr = _lattice_c(generated)
        GS, gkeep = _strength_c(generated)
        nb = max(L.n_bonds, 1)
        ft, fc, fs = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        s = lib().sc_as_generated(self.h, C.byref(L), C.byref(S), C.byref(G), C.byref(GS),
                                  C.byref(opt or options()), _ptr(ft), _ptr(fc), _ptr(fs))
        self._check(s, "sc_as_generated", soft=(OK, MAXITER))
        out = dict(lattice)
        out.update(ft=ft[:L.n_bonds], fc=fc[:L.n_bonds], fs=fs[:L.n_bonds])
        return out

    def settle(self, lattice: dict, opt: Options | None = None):
        """statics::bodies::settle (bodies.rs:511-541): (fallen fraction of the free mass,
        rounds, gone flags per node, info)."""
        L, arr = _lattice_c(lattice)
        S, keep = _strength_c(lattice)
        gone = np.zeros(L.n_nodes, np.uint8)
        out = SettleInfo()
        s = lib().sc_settle(self.h, C.byref(L), C.byref(S), C.byref(opt or options()), _ptr(gone), C.byref(out))
        self._check(s, "sc_settle", soft=(OK, MAXITER))
        return out.fell, out.rounds, gone, dict(work=out.work, status=out.status)


def _lattice_c(lattice: dict):
    """The sc_lattice view of a lattice dict (and the arrays it points into)."""
    nn = int(lattice["x"].shape[0])
    nb = int(lattice["bi"].shape[0])
    arr = {}
    for key, dt in (("x", np.float64), ("held", np.uint8), ("around", np.int64), ("bi", np.int64),
                    ("bj", np.int64), ("p", np.float64), ("n", np.float64), ("a", np.float64),
                    ("d", np.float64), ("e", np.float64), ("g", np.float64)):
        arr[key] = np.ascontiguousarray(lattice[key], dt)
    L = LatticeC()
    L.level, L.n_nodes, L.n_bonds = int(lattice.get("level", 0)), nn, nb
    L.x, L.held, L.around = _ptr(arr["x"]), _ptr(arr["held"]), _ptr(arr["around"])
    L.bond_i, L.bond_j, L.bond_p, L.bond_n = _ptr(arr["bi"]), _ptr(arr["bj"]), _ptr(arr["p"]), _ptr(arr["n"])
    L.bond_a, L.bond_d, L.bond_e, L.bond_g = _ptr(arr["a"]), _ptr(arr["d"]), _ptr(arr["e"]), _ptr(arr["g"])
    return L, arr


def _strength_c(lattice: dict):
    keep = {k: np.ascontiguousarray(lattice[k], np.float64) for k in ("m", "ft", "fc", "fs")}
    S = Strength()
    S.m, S.ft, S.fc, S.fs = (_ptr(keep[k]) for k in ("m", "ft", "fc", "fs"))
    return S, keep


_default: Solver | None = None


def motions(lattice: dict, alive=None, gone=None, loads=None, work: Work | None = None, opt=None) -> np.ndarray:
    """Module-level drop-in for statics::bodies::motions on device 0."""
    global _default
    if _default is None:
        _default = Solver(0)
    return _default.motions(lattice, alive, gone, loads, work, opt)
