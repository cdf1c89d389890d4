"""Generates tests/golden/oracle_gather.json: the oracle's gathered levels (statics::gather,
statics/src/gather.rs) of scenes restated from the reference's statics/examples/statics.rs
and its bar test (gather.rs:403-405), three levels each, measured against a full cell and as
it is: per level the node and bond counts, the total weight, and a hash of every array. The
oracle is the CPU restatement of gather.rs; the hashes pin it (and through the parity tests
the library) to these exact bits. Usage:

    python tests/golden/make_gather_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT]

from oracle import oracle as O  # noqa: E402

KEYS = ("x", "m", "held", "around", "bi", "bj", "p", "n", "a", "d", "e", "g")
SCENES = {
    "bar": lambda: O.Lattice.block(O.STEEL, [-4.5, -1.0, -1.0], [4.5, 1.0, 1.0], [4.0, 0.2, 0.2]),
    "cantilever": lambda: O.Lattice.scene("cantilever", O.STONE, 0.5, 3.0),
    "pendant_apart": lambda: O.Lattice.scene("pendant", O.STONE, 1),
}


def digest(lat) -> dict:
    e = lat.export()
    e.update(lat.strengths())
    h = hashlib.sha256()
    for k in KEYS + ("ft", "fc", "fs"):
        h.update(np.ascontiguousarray(e[k]).tobytes())
    return {"nodes": lat.n_nodes, "bonds": lat.n_bonds, "weight": float(e["m"].sum()), "sha256": h.hexdigest()[:32]}


def main():
    out = []
    for name, make in SCENES.items():
        for against in (True, False):
            lat = make()
            for level in (1, 2, 3):
                lat = lat.gathered(against)
                out.append(dict(scene=name, against_full=against, level=level, **digest(lat)))
    path = os.path.join(HERE, "oracle_gather.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out)} levels to {path}")


if __name__ == "__main__":
    main()
