"""The reference's edits experiment on the GPU chain (exp_edits,
statics/examples/statics.rs:310-344): a generated scene and its edit, both gathered
level after level (sc_gather on the device), made as strong as the generated one needs
(sc_as_generated, statics/src/bodies.rs:611-625) and settled (sc_settle). Checked bit
for bit against the oracle's run of the same chain (tests/golden/oracle_edits.json,
made by tests/golden/make_edits_golden.py: fallen shares, rounds, a hash of every gone
array) and against the verdicts the reference publishes per level
(docs/statics.md:236-247: stands, falls, two fifths fall)."""
import hashlib
import json
import os

import numpy as np
import pytest

import statics_cuda as sc
from oracle import oracle as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "oracle_edits.json")))


def verdict(fallen):
    if fallen == 0.0:
        return "stands"
    if 0.35 <= fallen <= 0.45:
        return "two fifths fall"
    return "falls"


def _dict(lat):
    return dict(lat.export(), **lat.strengths(), mat=lat.materials()["node"], level=0)


def _hash(gone):
    return hashlib.sha256(np.ascontiguousarray(gone, np.uint8).tobytes()).hexdigest()[:16]


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_edits_chain_matches_oracle(solver, case):
    (gk, gkw), (ek, ekw) = case["generated"], case["edited"]
    names = list(sc.MATERIALS)
    g, e = _dict(O.Lattice.scene(gk, **gkw)), _dict(O.Lattice.scene(ek, **ekw))
    for want in case["levels"]:
        if want["level"] > 0:
            g, e = solver.gather(g, names), solver.gather(e, names)
        assert [len(g["m"]), len(e["m"])] == want["nodes"]
        assert [len(g["bi"]), len(e["bi"])] == want["bonds"]
        gs, es = solver.as_generated(g, g), solver.as_generated(e, g)
        got = []
        for lat in (gs, es):
            fell, rounds, gone, _ = solver.settle(lat)
            got.append((fell, rounds, _hash(gone)))
        for i in range(2):
            assert got[i][0] == pytest.approx(want["fallen"][i], abs=1e-12), (want["level"], i)
            assert got[i][1] == want["rounds"][i], (want["level"], i)
            assert got[i][2] == want["gone_hash"][i], (want["level"], i)
        assert verdict(got[1][0]) == case["docs"][want["level"]], want["level"]
