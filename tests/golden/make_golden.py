"""Generates tests/golden/oracle_pieces.json: the oracle's outputs on seeded synthetic
pieces (value noise period 8, threshold 0.5, bottom layer held, k uniform [0.5, 2],
load -1 along z per unit mass), so GPU parity at sizes where the oracle takes minutes
runs against committed numbers. The pieces come from sc_generate_piece; the oracle is
the CPU restatement of statics/src/bodies.rs. Usage:

    python tests/golden/make_golden.py [n:seed:tol ...]   (default: the committed set)
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "parallax-world_b200"), os.path.dirname(HERE)]

import statics_cuda as sc  # noqa: E402
from oracle import oracle as O  # noqa: E402

DEFAULT = ["16:0:1e-8", "16:1:1e-8", "24:3:1e-8", "32:0:1e-8", "32:1:1e-8", "32:2:1e-8", "32:0:1e-12",
           "48:5:1e-8", "64:0:1e-8", "96:0:1e-8", "128:0:1e-8"]


def up_hash(up):
    return hashlib.sha256(np.ascontiguousarray(up, np.int32).tobytes()).hexdigest()[:16]


def run(n, seed, tol):
    st, k = sc.generate_piece(n, n, n, seed, sc.K_UNIFORM)
    lat = O.Lattice.grid(st, k, g_over_e=0.4, rho=512.0)
    ex = lat.export()
    loads = np.zeros((lat.n_nodes, 6))
    loads[:, 2] = -ex["m"]
    t = time.time()
    u, info = lat.motions(loads, tol=tol, hierarchy=True)
    secs = time.time() - t
    rng = np.random.default_rng(1000 + n + seed)
    idx = np.sort(rng.choice(u.size, size=min(256, u.size), replace=False))
    return dict(n=n, seed=seed, tol=tol, n_nodes=lat.n_nodes, free_cells=int((st == 1).sum()),
                counts=info["counts"], pairs=info["pairs"], steps=info["steps"], iterations=info["iterations"],
                work=info["work"], up_sums=[int(np.asarray(x, np.int64).sum()) for x in info["up"]],
                up_hash=[up_hash(x) for x in info["up"]], u_norm=float(np.linalg.norm(u)),
                sample_idx=idx.tolist(), sample_u=u.ravel()[idx].tolist(), seconds=secs,
                threads=O.threads())


def main():
    specs = sys.argv[1:] or DEFAULT
    path = os.path.join(HERE, "oracle_pieces.json")
    cases = json.load(open(path)) if os.path.exists(path) else []
    for spec in specs:
        n, seed, tol = spec.split(":")
        c = run(int(n), int(seed), float(tol))
        cases = [x for x in cases if not (x["n"] == c["n"] and x["seed"] == c["seed"] and x["tol"] == c["tol"])]
        cases.append(c)
        cases.sort(key=lambda x: (x["n"], x["seed"], -x["tol"]))
        json.dump(cases, open(path, "w"), indent=1)
        print(f"{spec}: levels {c['counts']} iterations {c['iterations']} in {c['seconds']:.1f}s", flush=True)


if __name__ == "__main__":
    main()
