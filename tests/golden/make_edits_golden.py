"""Generates tests/golden/oracle_edits.json: the oracle's run of the reference's edits
experiment (`exp_edits`, statics/examples/statics.rs:310-344), whose outcomes the
reference publishes as its per-level verdicts (docs/statics.md:236-247).

For each (generated, edited) pair of scenes (restated in oracle/scenes.cpp from
statics/examples/statics.rs), at levels 0 to 4 (each level gathered from the one below,
gather.rs:193-195): both lattices made as strong as the generated one needs
(as_generated, bodies.rs:611-625), then settled (bodies.rs:511-541). Recorded per level:
the fallen share of each, the rounds, and a hash of each gone array, so GPU runs of the
same chain are checked against it bit for bit without the oracle's minutes-long level-0
settles. Usage:

    python tests/golden/make_edits_golden.py [case ...]   (default: every case)
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "parallax-world_b200")]

from oracle import oracle as O  # noqa: E402

# name: (generated scene, edited scene, the docs' verdicts at levels 0..4 for the edited one)
CASES = {
    "cantilever 4 m": (("cantilever", dict(mat=O.STONE, a=0.5, b=3.0)), ("cantilever", dict(mat=O.STONE, a=0.5, b=4.0)),
                       ["stands"] * 5),
    "cantilever 6 m": (("cantilever", dict(mat=O.STONE, a=0.5, b=3.0)), ("cantilever", dict(mat=O.STONE, a=0.5, b=6.0)),
                       ["stands"] * 5),
    "slab, one column cut": (("portico", dict(a=0, b=0.5)), ("portico", dict(a=1, b=0.5)), ["stands"] * 5),
    "slab, two columns cut": (("portico", dict(a=0, b=0.5)), ("portico", dict(a=2, b=0.5)),
                              ["falls", "falls", "falls", "falls", "stands"]),
    "tower, a leg cut": (("tower", dict(mat=O.STEEL, a=0)), ("tower", dict(mat=O.STEEL, a=1)),
                         ["stands", "stands", "stands", "stands", "falls"]),
    "tower, two legs cut": (("tower", dict(mat=O.STEEL, a=0)), ("tower", dict(mat=O.STEEL, a=2)),
                            ["stands", "stands", "two fifths fall", "two fifths fall", "falls"]),
    "tree cut 30 %": (("tree", dict(a=8.0, b=1.0, c=0.0)), ("tree", dict(a=8.0, b=-1.0, c=0.3)), ["stands"] * 5),
    "tree cut 70 %": (("tree", dict(a=8.0, b=1.0, c=0.0)), ("tree", dict(a=8.0, b=-1.0, c=0.7)),
                      ["falls", "falls", "stands", "stands", "stands"]),
    "tree cut through": (("tree", dict(a=8.0, b=1.0, c=0.0)), ("tree", dict(a=8.0, b=-1.0, c=1.0)),
                         ["falls", "falls", "falls", "stands", "stands"]),
    "block hanging let go": (("pendant", dict(a=0)), ("pendant", dict(a=1)), ["falls"] * 5),
}


def gone_hash(gone):
    return hashlib.sha256(np.ascontiguousarray(gone, np.uint8).tobytes()).hexdigest()[:16]


def run(name):
    (gk, gkw), (ek, ekw), verdicts = CASES[name]
    g, e = O.Lattice.scene(gk, **gkw), O.Lattice.scene(ek, **ekw)
    levels = []
    for level in range(5):
        t = time.time()
        if level > 0:
            g, e = g.gathered(), e.gathered()
        gs, es = g.copy(), e.copy()
        gs.as_generated(g)
        es.as_generated(g)
        fb, rb, gb = gs.settle()
        fa, ra, ga = es.settle()
        levels.append(dict(level=level, nodes=[g.n_nodes, e.n_nodes], bonds=[g.n_bonds, e.n_bonds],
                           fallen=[fb, fa], rounds=[rb, ra], gone_hash=[gone_hash(gb), gone_hash(ga)],
                           seconds=time.time() - t))
    return dict(name=name, generated=[gk, gkw], edited=[ek, ekw], docs=verdicts, levels=levels, threads=O.threads())


def main():
    names = sys.argv[1:] or list(CASES)
    path = os.path.join(HERE, "oracle_edits.json")
    out = json.load(open(path)) if os.path.exists(path) else []
    for name in names:
        c = run(name)
        out = [x for x in out if x["name"] != name] + [c]
        print(name, [(lv["level"], round(lv["fallen"][1], 3)) for lv in c["levels"]], flush=True)
    out.sort(key=lambda x: list(CASES).index(x["name"]))
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
