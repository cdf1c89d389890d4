#!/usr/bin/env python
"""Benchmark of the statics solve (statics::bodies::motions on a voxel piece).

Workload (one step): one full solve -- hierarchy setup plus preconditioned conjugate
gradients to 1e-8 relative residual -- of a seeded synthetic 128^3 piece (value noise of
period 8, threshold 0.5, bottom layer held, k uniform in [0.5, 2], load -1 along z per
unit mass). `value` is solves/s with the piece already in HBM (mixed precision: FP64
conjugate gradients preconditioned by the V-cycle in FP32); `fp64` is the same for the
plain FP64 solve and `mixed_fp32_krylov` for the all-FP32 Krylov recurrence with FP64
residual replacement; `e2e` is the C-ABI call with host buffers (copies inside the
timed region).
Each rank solves its own piece (seed + rank): weak scaling, no collective on the data
path. The working set (vectors ~0.1-0.2 GB each, coarse operators GBs) exceeds the
126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "parallax-world_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "DOF·iters/s & solves/s to 1e-8 rel residual: mixed vs FP64 GPU vs CPU ref"
N = 128
TOL = 1e-8
SAMPLE_N, SAMPLE_SEED = 48, 5  # the CPU legs' bounded sample
EDGES = (16, 24, 32, 48, 64)   # edge lengths of the batched pieces


def peaks():
    try:
        m = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def rank_seed(base, rank):
    """Each rank solves its own piece: weak scaling, no collective on the data path."""
    return base + rank


def workload(seed):
    return {"workload": f"{N}^3 voxel piece, value noise period 8 thr 0.5, seed {seed}+rank, k U[0.5,2], "
                        f"gravity -z, solve to {TOL:g} rel residual (setup + PCG per step)",
            "grid": [N, N, N], "seed": seed, "tol": TOL, "l2": "inputs larger than L2 (no flush)"}


# ---- clocks ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.path = tempfile.mktemp(suffix=".csv")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], [], set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- distributed plumbing -----------------------------------------------------------------
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---- the CPU legs (the oracle: a restatement of the reference's Rust) ------------------------
# Their inputs come from the oracle's own generator (oracle/generate_oracle.cpp, byte-equal
# to the library's, tests/test_oracle_generator.py): the CPU legs load no product library.
def oracle_solve(n, seed, threads=None):
    """One oracle `motions` (setup + PCG, timed by std::chrono inside the oracle) of the
    seeded n^3 piece under -1 along z per unit mass, to TOL, on `threads` host threads
    (all of them by default)."""
    import numpy as np

    from oracle import oracle as O
    st, k = O.generate_piece(n, n, n, seed, O.K_UNIFORM)
    lat = O.Lattice.grid(st, k, g_over_e=0.4, rho=512.0)
    ex = lat.export()
    loads = np.zeros((lat.n_nodes, 6))
    loads[:, 2] = -ex["m"]
    before = O.threads()
    if threads:
        O.set_threads(threads)
    try:
        _, info = lat.motions(loads, tol=TOL)
        used = O.threads()
    finally:
        O.set_threads(before)
    return dict(seconds=info["seconds"], setup_seconds=info["setup_seconds"], solve_seconds=info["solve_seconds"],
                dof=6 * info["counts"][0], iterations=info["iterations"], threads=used, n=n, seed=seed)


def cpu_sample():
    """The bounded sample of our arm's CPU baseline: one oracle solve of a 48^3 piece on
    all host threads (about 5 s on 16 threads)."""
    return oracle_solve(SAMPLE_N, SAMPLE_SEED)


def cpu_baseline_obj(s, dof_iters_target):
    rate = s["dof"] * s["iterations"] / s["seconds"]
    return {"value": rate / dof_iters_target, "unit": "solves/s", "cores": s["threads"], "kind": "port",
            "dof_iters_per_s": rate, "sample_solves_per_s": 1.0 / s["seconds"],
            "sample": f"oracle (C++ restatement of statics/src/bodies.rs) solving a {SAMPLE_N}^3 piece "
                      f"(seed {SAMPLE_SEED}, {s['dof']} DOF, {s['iterations']} iterations) to {TOL:g} in "
                      f"{s['seconds']:.2f} s on {s['threads']} threads (sample_solves_per_s); value is that "
                      f"DOF*iters/s over the {N}^3 solve's DOF*iters. The reference arm "
                      f"(bench.py --impl reference) times whole {N}^3 solves instead"}


def run_reference(args):
    """The reference's algorithm on the host's cores: the oracle's `motions` (setup + PCG)
    of the same 128^3 piece, timed whole. Warm-up: W solves of a 24^3 piece. Timed: whole
    128^3 solves, at least one and at most K, no new one started once --ref-budget
    seconds have passed. Beside it, one 48^3 solve on one thread."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    for w in range(args.warmup):
        oracle_solve(24, 100 + w)
    solves = []
    t_start = time.perf_counter()
    while len(solves) < max(1, args.steps):
        solves.append(oracle_solve(N, args.seed))
        spent = time.perf_counter() - t_start
        if spent + solves[-1]["seconds"] > args.ref_budget:
            break
    one = oracle_solve(SAMPLE_N, SAMPLE_SEED, threads=1)
    secs = statistics.mean(s["seconds"] for s in solves)
    s0 = solves[0]
    value = 1.0 / secs
    cores = s0["threads"]
    sample = (f"{len(solves)} whole oracle motions (setup + PCG) of the {N}^3 piece (seed {args.seed}, "
              f"{s0['dof']} DOF, {s0['iterations']} iterations to {TOL:g}) on {cores} host threads, "
              f"std::chrono inside the oracle: mean {secs:.1f} s")
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": len(solves),
            "warmup": args.warmup, "ms_per_step": 1000.0 * secs, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload(args.seed),
            "impl": "reference",
            "steps_note": f"--steps {args.steps} asked; {len(solves)} whole {N}^3 solves timed within "
                          f"--ref-budget {args.ref_budget:g} s (warm-up: {args.warmup} solves of a 24^3 piece)",
            "dof_iters_per_s": s0["dof"] * s0["iterations"] / secs,
            "setup_s": statistics.mean(s["setup_seconds"] for s in solves),
            "solve_s": statistics.mean(s["solve_seconds"] for s in solves),
            "seconds_each": [round(s["seconds"], 3) for s in solves],
            "one_core": {"grid": [SAMPLE_N] * 3, "seed": SAMPLE_SEED, "seconds": one["seconds"],
                         "dof": one["dof"], "iterations": one["iterations"], "threads": one["threads"],
                         "solves_per_s": 1.0 / one["seconds"],
                         "dof_iters_per_s": one["dof"] * one["iterations"] / one["seconds"]},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def golden_piece(seed):
    """The oracle's committed record of the bench piece (n, seed, TOL), if there is one."""
    try:
        for c in json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_pieces.json"))):
            if c["n"] == N and c["seed"] == seed and c["tol"] == TOL:
                return c
    except (OSError, ValueError):
        pass
    return None


# ---- our arm -----------------------------------------------------------------------------
def run_ours(args):
    import numpy as np
    import torch

    import statics_cuda as sc

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    solver = sc.Solver(local)
    seed = rank_seed(args.seed, rank)
    state, k = sc.generate_piece(N, N, N, seed, sc.K_UNIFORM)
    n_nodes, n_parts = sc.grid_count(state)
    st_d = torch.from_numpy(state).cuda()
    k_d = torch.from_numpy(k).cuda()
    out_d = torch.empty(6 * n_nodes, dtype=torch.float64, device="cuda")
    grid = sc.make_grid(state, k)
    grid.state, grid.k, grid.on_device = st_d.data_ptr(), k_d.data_ptr(), 1
    stream = torch.cuda.ExternalStream(solver.stream())
    hbm, hbm_kind = peaks()

    def timed(precision, steps, warmup):
        """K solves on the solver's stream, CUDA events around them, profiling off (the
        CG iterations run as CUDA graphs)."""
        opt = sc.options(tol=TOL, precision=precision, tile=args.tile)
        for _ in range(warmup):
            solver.solve_grid_device(grid, opt, out_d.data_ptr(), out_d.numel())
        barrier(world)
        torch.cuda.synchronize()
        l0 = sc.launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        infos = [solver.solve_grid_device(grid, opt, out_d.data_ptr(), out_d.numel()) for _ in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        return ms, infos, sc.launches() - l0

    def profiled(precision, mask):
        """One more solve of the same workload with per-launch CUDA events on the
        solver's stream for the kernel families in `mask` (kernels launched one by one)."""
        opt = sc.options(tol=TOL, precision=precision, tile=args.tile)
        barrier(world)
        torch.cuda.synchronize()
        solver.profile(mask)
        solver.solve_grid_device(grid, opt, out_d.data_ptr(), out_d.numel())
        torch.cuda.synchronize()
        prof = solver.profile_read()
        solver.profile(0)
        return prof

    golden = golden_piece(seed)

    def error_vs_oracle():
        """The motions the last solve wrote (out_d) against the oracle's FP64 solve of the
        same piece at the same tolerance (tests/golden/oracle_pieces.json: its norm and 256
        sampled values)."""
        if golden is None:
            return None
        idx = torch.tensor(golden["sample_idx"], dtype=torch.int64, device="cuda")
        got = out_d[idx].cpu().numpy()
        want = np.array(golden["sample_u"])
        norm = float(torch.linalg.vector_norm(out_d).item())
        return {"sample_l2_rel": float(np.linalg.norm(got - want) / np.linalg.norm(want)),
                "sample_max_abs_over_max": float(np.abs(got - want).max() / np.abs(want).max()),
                "norm_rel_diff": abs(norm - golden["u_norm"]) / golden["u_norm"],
                "oracle": f"oracle FP64 solve of the same piece to {golden['tol']:g} "
                          f"({golden['iterations']} iterations), 256 sampled motions and the norm"}

    clocks = Clocks(local)
    ms_mixed, infos_m, launches = timed(sc.MIXED, args.steps, args.warmup)
    clk = clocks.stop()
    err_mixed = error_vs_oracle()
    ms_64, infos_64, _ = timed(sc.FP64, args.steps, max(3, args.warmup // 2))
    err_64 = error_vs_oracle()
    ms_k, infos_k, _ = timed(sc.MIXED_FP32_KRYLOV, args.steps, max(3, args.warmup // 2))
    # which kernel family dominates a mixed solve, and each family's time per launch
    all_fams = (1 << len(sc.FAM_NAMES)) - 1
    prof = profiled(sc.MIXED, all_fams)
    prof64 = profiled(sc.FP64, all_fams)
    dominant = max(prof, key=lambda f: prof[f]["ms"])
    stencil = "stencil32"

    # e2e through the C ABI with host buffers: the piece's state and k uploaded and the
    # motions (n_nodes x 6 FP64) downloaded every step, into the caller's output array; all
    # three in pinned (page-locked) host memory, which the copies reach at full speed
    opt = sc.options(tol=TOL, precision=sc.MIXED)
    state_h = torch.from_numpy(state).pin_memory().numpy()
    k_h = torch.from_numpy(k).pin_memory().numpy()
    u_host = torch.empty((n_nodes, 6), dtype=torch.float64, pin_memory=True).numpy()
    solver.solve_grid(state_h, k_h, opt, out=u_host)  # warm-up
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        u, _ = solver.solve_grid(state_h, k_h, opt, out=u_host)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), world)

    K = args.steps
    dof = 6 * n_parts
    it_m = infos_m[-1]["iterations"]
    it_64 = infos_64[-1]["iterations"]
    value = world * K / (ms_mixed / 1000.0)
    solve_ms_m = statistics.mean(i["solve_ms"] for i in infos_m)
    solve_ms_64 = statistics.mean(i["solve_ms"] for i in infos_64)

    def roof(p, name):
        f = p[name]
        if not f["launches"]:
            return None
        avg_ms = f["ms"] / f["launches"]
        achieved = f["bytes"] / f["launches"] / (avg_ms / 1000.0) / 1e9
        return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": hbm_kind, "launches": f["launches"], "avg_ms": avg_ms,
                "bytes_per_launch": f["bytes"] / f["launches"], "traffic": None}

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": ms_mixed / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 CG, f32 V-cycle", "data": "synthetic", "config": workload(args.seed),
        "dof": dof, "iterations": it_m, "refinements": infos_m[-1]["refinements"],
        "error_vs_oracle": err_mixed,
        "levels": infos_m[-1]["parts"], "residual": infos_m[-1]["residual"],
        "setup_ms": statistics.mean(i["setup_ms"] for i in infos_m), "solve_ms": solve_ms_m,
        "dof_iters_per_s": world * dof * it_m / (solve_ms_m / 1000.0),
        "fp64": {"value": world * K / (ms_64 / 1000.0), "unit": "solves/s", "ms_per_step": ms_64 / K,
                 "iterations": it_64, "solve_ms": solve_ms_64,
                 "dof_iters_per_s": world * dof * it_64 / (solve_ms_64 / 1000.0),
                 "residual": infos_64[-1]["residual"], "error_vs_oracle": err_64,
                 "stencil_roofline": roof(prof64, "stencil64")},
        "mixed_fp32_krylov": {"value": world * K / (ms_k / 1000.0), "unit": "solves/s", "ms_per_step": ms_k / K,
                              "iterations": infos_k[-1]["iterations"],
                              "refinements": infos_k[-1]["refinements"],
                              "solve_ms": statistics.mean(i["solve_ms"] for i in infos_k),
                              "residual": infos_k[-1]["residual"]},
        "roofline": roof(prof, dominant),
        "stencil_roofline": roof(prof, stencil),
        "kernel_ms": {f: round(prof[f]["ms"], 3) for f in prof if prof[f]["launches"]},
        # the whole CG phase against HBM: the algorithmic bytes of every timed kernel family
        # of the profiled solve over the timed solves' CG time (dots and axpys not counted)
        "solve_roofline": {"bytes_per_solve": sum(prof[f]["bytes"] for f in prof),
                           "achieved": sum(prof[f]["bytes"] for f in prof) / (solve_ms_m / 1000.0) / 1e9,
                           "peak": hbm, "unit": "GB/s",
                           "frac": sum(prof[f]["bytes"] for f in prof) / (solve_ms_m / 1000.0) / 1e9 / hbm},
        "setup_roofline": setup_roofline(infos_m[-1], state.size, statistics.mean(i["setup_ms"] for i in infos_m),
                                         hbm),
        "roofline_method": "per-launch CUDA events on the solver's stream during one profiled solve of the same "
                           "workload after the timed region (the timed region runs CUDA graphs, no events)",
        "e2e": {"value": world * K / (ms_e2e / 1000.0), "unit": "solves/s",
                "h2d_bytes_per_step": int(state.nbytes + k.nbytes), "d2h_bytes_per_step": int(8 * 6 * n_nodes)},
        "gpu_launches": launches,
        "clocks": clk,
        "peak_hbm_bytes": infos_m[-1]["peak_bytes"],
    }
    if not args.no_batch:
        line["batch"] = batch_section(solver, sc, rank, world, args)
    if rank == 0 and world == 1 and not args.no_large:
        line["large"] = large_section(solver, sc, args)
    if rank == 0 and world == 1 and not args.no_cpu:
        s = cpu_sample()
        line["cpu_baseline"] = cpu_baseline_obj(s, dof * it_64)
    if rank == 0:
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_probe(args):
    """One kernel or one solve alone, for profiling: `stencil` applies the level-0
    stencil to the bench's piece (FP64 then FP32, two launches each); `solve` runs FP64,
    mixed, FP64, mixed solves of it (SC_TIMING=1 prints the setup's phases)."""
    import numpy as np

    import statics_cuda as sc
    if args.probe == "mech":
        # the engine's solver (sc_mech_solve) on voxel pieces at rest (E = 1e9 U[0.5, 2],
        # h = 1/8 m, dt = 1/60 s), to 1e-8 in its energy norm; beside it, the CPU baseline:
        # the oracle's restatement of the same solver on one host core (pieces up to 48^3)
        solver = sc.Solver(0)
        for n in (32, 48, 64):
            st, k = sc.generate_piece(n, n, n, 4, sc.K_UNIFORM)
            s = sc.mech_voxel_system(st, k * 1e9, h=0.125, dt=1 / 60, mass=2000 * 0.125 ** 3)
            solver.mech_solve(s, tol=1e-8)  # warm-up
            t = time.perf_counter()
            x, rounds, levels = solver.mech_solve(s, tol=1e-8)
            out = {"probe": "mech", "grid": [n, n, n], "unknowns": len(s["sites"]), "pairs": len(s["pi"]),
                   "rounds": rounds, "levels": levels, "gpu_s": time.perf_counter() - t}
            if n <= 48:
                from oracle import mechanics as M
                t = time.perf_counter()
                xr, rr, _, _ = M.solve(s, tol=1e-8)
                out.update(cpu_s=time.perf_counter() - t, cpu_rounds=rr,
                           rel_diff=float(np.linalg.norm(x - xr) / np.linalg.norm(xr)))
            print(json.dumps(out), flush=True)
        solver.close()
        return
    if args.probe == "gather":
        # statics::gather (sc_gather, the host's cores) on the reference's timing scene, an
        # uncut tree (statics/examples/statics.rs:373-391), gathered to levels 1-4; beside it
        # the oracle's restatement on the same cores, and whether the two levels are the
        # same bit for bit. The tree itself is built by the oracle's lattice.rs restatement
        # (the library builds level 0 of voxel pieces only, on the device).
        from oracle import oracle as O
        names = list(sc.MATERIALS)
        keys = ("x", "m", "held", "around", "bi", "bj", "p", "n", "a", "d", "e", "g", "ft", "fc", "fs")
        sc.gather_full("stone"), O.full(O.STONE)  # both full-cell calibrations made once
        ora = O.Lattice.scene("tree", O.STONE, 8.0, 1.0, 0.0)
        lat = dict(ora.export(), **ora.strengths(), mat=ora.materials()["node"], level=0)
        try:  # the device leg: the cells measured by k_gather_cells, one thread block a cell
            solver = sc.Solver(0)
            solver.gather(lat, names)  # warm-up: module load, the other materials' calibrations
        except Exception:
            solver = None
        for level in range(1, 5):
            t = time.perf_counter()
            nxt = sc.gather(lat, names)
            lib_s = time.perf_counter() - t
            dev_s = dev_same = None
            if solver is not None:
                t = time.perf_counter()
                dev = solver.gather(lat, names)
                dev_s = time.perf_counter() - t
                dev_same = all(np.array_equal(nxt[k], dev[k]) for k in keys)
            t = time.perf_counter()
            ora = ora.gathered()
            ora_s = time.perf_counter() - t
            want = dict(ora.export(), **ora.strengths())
            same = all(np.array_equal(nxt[k], want[k]) for k in keys)
            print(json.dumps({"probe": "gather", "scene": "tree(8, 1, 0)", "level": level,
                              "fine_nodes": int(len(lat["m"])), "fine_bonds": int(len(lat["bi"])),
                              "nodes": int(len(nxt["m"])), "bonds": int(len(nxt["bi"])), "library_s": lib_s,
                              "device_s": dev_s, "oracle_s": ora_s, "cores": os.cpu_count(),
                              "identical": bool(same), "device_identical": dev_same}), flush=True)
            lat = nxt
        if solver is not None:
            solver.close()
        return
    if args.probe == "large":
        solver = sc.Solver(0)
        print(json.dumps(large_section(solver, sc, args)), flush=True)
        solver.close()
        return
    if args.probe == "batch":
        pieces = batch_pieces(sc, args.batch)
        solver = sc.Solver(0)
        names = {sc.FP64: "fp64", sc.MIXED: "mixed", sc.MIXED_FP32_KRYLOV: "mixed_fp32_krylov"}
        slow = None
        for prec in (sc.MIXED, sc.MIXED, sc.MIXED_FP32_KRYLOV, sc.FP64):
            opt = sc.options(tol=TOL, precision=prec, max_iter=20000)
            t = time.perf_counter()
            _, infos = solver.solve_grid_batch(pieces, opt)
            dt = time.perf_counter() - t
            groups = sorted({(i["setup_ms"], i["solve_ms"]) for i in infos})
            print(json.dumps({"probe": "batch", "pieces": len(pieces), "precision": names[prec],
                              "seconds": dt, "groups": len(groups),
                              "setup_ms": sum(g[0] for g in groups), "solve_ms": sum(g[1] for g in groups),
                              "iterations_max": max(i["iterations"] for i in infos),
                              "iterations_mean": sum(i["iterations"] for i in infos) / len(infos),
                              "bad": sum(1 for i in infos if i["status"] != 0)}), flush=True)
            if slow is None:
                slow = sorted(range(len(infos)), key=lambda i: -infos[i]["iterations"])[:4]
        for i in slow:
            st, k = pieces[i]
            alone = {}
            for prec in (sc.MIXED, sc.MIXED_FP32_KRYLOV, sc.FP64):
                _, inf = solver.solve_grid(st, k, sc.options(tol=TOL, precision=prec, max_iter=20000))
                alone[names[prec]] = {"status": inf["status"], "iterations": inf["iterations"],
                                      "residual": inf["residual"]}
            print(json.dumps({"piece": i, "shape": list(st.shape), "parts": inf["parts"][:inf["levels"]],
                              "steps": inf["steps"][:inf["levels"]], "alone": alone}), flush=True)
        t = time.perf_counter()
        for st, k in pieces[:32]:
            solver.solve_grid(st, k, sc.options(tol=TOL, precision=sc.FP64))
        print(json.dumps({"probe": "fp64 single", "pieces": 32, "seconds": time.perf_counter() - t}), flush=True)
        solver.close()
        return
    pn = args.probe_n
    state, k = sc.generate_piece(pn, pn, pn, args.seed, sc.K_UNIFORM)
    if args.probe == "solve":
        solver = sc.Solver(0)
        order = {"all": (sc.FP64, sc.MIXED, sc.MIXED_FP32_KRYLOV) * 2, "mixed": (sc.MIXED,) * 2,
                 "fp64": (sc.FP64,) * 2}[args.precision]
        for prec in order:
            _, info = solver.solve_grid(state, k, sc.options(tol=TOL, precision=prec, tile=args.tile))
            print(json.dumps({"probe": "solve", "precision": prec, "tile": args.tile, "iterations": info["iterations"],
                              "setup_ms": info["setup_ms"], "solve_ms": info["solve_ms"]}))
        solver.close()
        return
    _, parts = sc.grid_count(state)
    x = np.random.default_rng(0).standard_normal((parts, 6))
    solver = sc.Solver(0)
    for prec in (sc.FP64, sc.MIXED):
        for _ in range(2):
            y = solver.grid_apply(state, k, x, prec)
    print(json.dumps({"probe": "stencil", "parts": parts, "y_norm": float(np.linalg.norm(y))}))
    solver.close()


def large_section(solver, sc, args):
    """The large configuration: a 256^3 piece, k lognormal (mu 0, sigma 0.5) clipped to
    [0.1, 10], the mixed-precision forward solve to 1e-8 plus the compliance adjoint, and
    the FP64 solve to 1e-10 with its adjoint as the gradient's reference (the CPU oracle
    does not fit this size in host memory; the FP64 GPU solve is checked against it up to
    128^3 by the parity tests). Times are the solver's own (setup + CG, device work,
    synchronised), and the wall time of the C-ABI call with its host copies."""
    import numpy as np
    n = args.large_n
    ws, wk = sc.generate_piece(48, 48, 48, 1, sc.K_LOGNORMAL)
    for prec in (sc.MIXED, sc.FP64):  # warm-up: the library's kernels loaded once
        solver.compliance_grad(ws, wk, sc.options(tol=TOL, precision=prec))
    st, k = sc.generate_piece(n, n, n, args.seed, sc.K_LOGNORMAL)
    nodes, parts = sc.grid_count(st)
    out = {"workload": f"{n}^3 piece, value noise period 8 thr 0.5, k lognormal (mu 0, sigma 0.5) clipped to "
                       f"[0.1, 10], seed {args.seed}: mixed forward + compliance adjoint to {TOL:g}; FP64 to 1e-10 "
                       f"as the gradient's reference",
           "grid": [n, n, n], "free_cells": int((st == sc.CELL_FREE).sum()), "dof": 6 * parts, "tol": TOL}
    res = {}
    # the mixed solve twice: the first call also grows the device's memory pool to this
    # size's peak (the driver maps new memory at tens of ms a GB), the second is the
    # steady state a caller that keeps its context sees
    for name, prec, tol, calls in (("mixed", sc.MIXED, TOL, 2), ("fp64", sc.FP64, 1e-10, 1)):
        first = None
        for call in range(calls):
            t = time.perf_counter()
            try:
                C, grad, u, info = solver.compliance_grad(st, k, sc.options(tol=tol, precision=prec,
                                                                            max_iter=20000))
            except sc.StaticsError as e:  # e.g. the device's memory: report it, keep the bench line
                out[name] = {"error": str(e)}
                return out
            wall = time.perf_counter() - t
            if call == 0 and calls > 1:
                first = {"setup_ms": info["setup_ms"], "solve_ms": info["solve_ms"],
                         "time_to_tol_ms": info["setup_ms"] + info["solve_ms"], "wall_s_with_copies": wall}
        res[name] = grad
        out[name] = {"tol": tol, "status": info["status"], "iterations": info["iterations"],
                     "refinements": info["refinements"], "residual": info["residual"],
                     "setup_ms": info["setup_ms"], "solve_ms": info["solve_ms"],
                     "time_to_tol_ms": info["setup_ms"] + info["solve_ms"], "wall_s_with_copies": wall,
                     "peak_hbm_bytes": info["peak_bytes"], "levels": info["parts"][:info["levels"]],
                     "compliance": C}
        if first:
            out[name]["first_call"] = first
    g, g64 = res["mixed"].ravel(), res["fp64"].ravel()
    free = st.ravel() == sc.CELL_FREE
    err = np.abs(g[free] - g64[free])
    out["grad_err_vs_fp64"] = {"max_abs_over_max": float(err.max() / np.abs(g64[free]).max()),
                               "l2_rel": float(np.linalg.norm(err) / np.linalg.norm(g64[free])),
                               "max_rel_per_voxel": float((err / np.abs(g64[free])).max())}
    out["compliance_rel_diff"] = abs(out["mixed"]["compliance"] - out["fp64"]["compliance"]) / abs(
        out["fp64"]["compliance"])
    return out


def setup_roofline(info, grid_cells, setup_ms, hbm):
    """The hierarchy setup against HBM, by its compulsory bytes: the piece read once (state
    and k, 5 B a grid cell), every coarse level's 6x6 blocks written once in FP64 and once
    in FP32 (SC_MIXED keeps both until the FP64 copies are dropped), and each coarse level
    but the top read once more in FP64 to make the next one's Galerkin product (level 0 is
    matrix-free: its operator comes from the cell template). A lower bound: the sorts,
    candidate lists and the level-0 K P blocks the setup moves besides are not counted."""
    blocks = [int(b) for b in info["blocks"][1:info["levels"]]]
    block64, block32 = 36 * 8, 36 * 4
    nbytes = 5 * grid_cells + sum(b * (block64 + block32) for b in blocks) + sum(b * block64 for b in blocks[:-1])
    achieved = nbytes / (setup_ms / 1000.0) / 1e9
    return {"bound": "hbm", "bytes_per_setup": nbytes, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "setup_ms": setup_ms, "traffic": None}


def batch_pieces(sc, count, seed0=10_000):
    """`count` pieces with edges drawn from EDGES per axis, seeds seed0 + i. Every rank
    makes the same batch; batch_share picks its part."""
    import numpy as np
    rng = np.random.default_rng(777)
    pieces = []
    for i in range(count):
        nx, ny, nz = (int(v) for v in rng.choice(EDGES, 3))
        pieces.append(sc.generate_piece(nx, ny, nz, seed0 + i, sc.K_UNIFORM))
    return pieces


def batch_share(sc, pieces, rank, world):
    """This rank's indices into `pieces`: one batch split across the ranks, longest
    pieces (by unknowns) first (statics_cuda.shard.lpt_split)."""
    from statics_cuda import shard
    dof = [6 * sc.grid_count(st)[1] for st, _ in pieces]
    return shard.lpt_split(dof, world)[rank], dof


def batch_stats(infos, tol, world):
    """Counts and extremes of this rank's solves, summed / maxed over the ranks (one
    all-reduce each, the same on every rank)."""
    import torch
    import torch.distributed as dist

    from statics_cuda import autotune
    sums = [len(infos), sum(1 for i in infos if i["status"] != 0),
            sum(1 for i in infos if i["status"] == 0 and not autotune.converged(i, tol)),
            sum(1 for i in infos if i["refinements"] > 0), sum(1 for i in infos if i.get("retried")),
            sum(i["iterations"] for i in infos),
            sum(1 for i in infos if autotune.above_tol_at_floor(i, tol))]
    worst = max([i["residual"] for i in infos] or [0.0])
    if world > 1:
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor(sums, dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        sums = [float(v) for v in t.tolist()]
        worst = max_over_ranks(worst, world)
    return {"pieces": int(sums[0]), "failed": int(sums[1]), "above_tol": int(sums[2]), "replaced": int(sums[3]),
            "retried": int(sums[4]), "iterations_mean": sums[5] / max(sums[0], 1), "max_true_residual": worst,
            "at_fp64_floor": int(sums[6])}


def batch_section(solver, sc, rank, world, args):
    """One batch of BATCH pieces whose edges are drawn from EDGES per axis, split across
    the ranks (longest first by unknowns) and solved by the autotuned mixed-precision
    batched solve on each; against the plain FP64 drop-in solving a sample of them one
    call at a time (the sample split the same way). Time: the max over ranks."""
    import torch

    from statics_cuda import autotune
    pieces = batch_pieces(sc, args.batch)
    mine, dof_all = batch_share(sc, pieces, rank, world)
    mine_p = [pieces[i] for i in mine]
    t = time.perf_counter()
    setting = autotune.choose(solver, mine_p, sc.MIXED, TOL)
    tune_s = time.perf_counter() - t
    stream = torch.cuda.ExternalStream(solver.stream())
    # warm-up: the same batch once, so the timed run finds the device pool grown to its peak
    autotune.solve_batch(solver, mine_p, sc.MIXED, TOL, setting=setting)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = sc.launches()
    e0.record(stream)
    _, infos = autotune.solve_batch(solver, mine_p, sc.MIXED, TOL, setting=setting)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = sc.launches() - l0
    ms_b = max_over_ranks(e0.elapsed_time(e1), world)
    stats = batch_stats(infos, TOL, world)
    sample_all = pieces[: min(args.batch_sample, len(pieces))]
    sample = [sample_all[i] for i in batch_share(sc, sample_all, rank, world)[0]]
    opt64 = sc.options(tol=TOL, precision=sc.FP64)
    solver.solve_grid(*sample[0], opt64)  # warm-up
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    for st, k in sample:
        solver.solve_grid(st, k, opt64)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_1 = max_over_ranks(e0.elapsed_time(e1), world)
    batched = len(pieces) / (ms_b / 1000.0)
    single = len(sample_all) / (ms_1 / 1000.0)
    groups = len({(i["setup_ms"], i["solve_ms"]) for i in infos})
    return {"workload": f"one batch of {len(pieces)} pieces split across {world} rank(s) (longest first by "
                        f"unknowns), edges from {list(EDGES)} per axis, seeds 10000+; value noise period 8 "
                        f"thr 0.5, k U[0.5,2], tol {TOL:g}",
            "scaling": "strong", "pieces": len(pieces), "dof": int(sum(dof_all)),
            "pieces_this_rank": len(mine_p), "dof_this_rank": int(sum(dof_all[i] for i in mine)),
            "mixed_batched_solves_per_s": batched,
            "fp64_single_solves_per_s": single, "fp64_single_sample": len(sample_all),
            "speedup_batched_mixed_vs_fp64_single": batched / single,
            "mixed_batched_ms": ms_b, "iterations_mean": stats["iterations_mean"],
            "pieces_failed": stats["failed"], "pieces_true_residual_above_tol_and_floor": stats["above_tol"],
            "pieces_above_tol_at_fp64_floor": stats["at_fp64_floor"],
            "pieces_residual_replaced": stats["replaced"], "max_true_residual": stats["max_true_residual"],
            "pieces_retried": stats["retried"], "groups_this_rank": groups, "gpu_launches_this_rank": launches,
            "autotune": {"sweeps": setting["sweeps"], "tile": setting["tile"]}, "autotune_seconds": tune_s}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--ref-budget", type=float, default=300.0,
                    help="--impl reference: seconds after which no further whole solve is started")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-pieces section")
    ap.add_argument("--no-large", action="store_true", help="skip the 256^3 forward + adjoint section")
    ap.add_argument("--batch", type=int, default=512, help="pieces in the batched section")
    ap.add_argument("--batch-sample", type=int, default=64, help="pieces the one-at-a-time FP64 leg solves")
    ap.add_argument("--large-n", type=int, default=256, help="edge of the --probe large piece")
    ap.add_argument("--tile", type=int, default=0, help="sc_options.tile of the solves (0: the default stencil)")
    ap.add_argument("--probe-n", type=int, default=N, help="edge of the --probe solve / stencil piece")
    ap.add_argument("--precision", choices=["all", "mixed", "fp64"], default="all",
                    help="the --probe solve precisions: all three twice, or two solves of one")
    ap.add_argument("--probe", choices=["stencil", "solve", "batch", "large", "mech", "gather"],
                    help="run one kernel or one solve alone (profiling); mech: the engine's solver; "
                         "gather: statics::gather on the host's cores")
    args = ap.parse_args()
    if args.probe:
        run_probe(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
