"""The callers of motions on the GPU (sc_used_standing, sc_settle) against the oracle's
used_standing (statics/src/bodies.rs:550-554) and settle (bodies.rs:511-541) on the
reference's edit scenes (statics/examples/statics.rs), and the published "Used at 0"
values they give (docs/statics.md:236-247)."""
import numpy as np
import pytest

import statics_cuda as sc
from oracle import oracle as O

from helpers import lattice_dict

pytestmark = pytest.mark.gpu

SCENES = [
    ("a stone beam made 4 m", dict(kind="cantilever", mat=O.STONE, a=0.5, b=4.0), 0.43),
    ("made 6 m", dict(kind="cantilever", mat=O.STONE, a=0.5, b=6.0), 0.97),
    ("a slab, one column cut", dict(kind="portico", a=1, b=0.5), 1.03),
    ("two columns cut", dict(kind="portico", a=2, b=0.5), 7.3),
    ("a tree cut 30 %", dict(kind="tree", a=8.0, b=-1.0, c=0.3), 0.37),
    ("cut 70 %", dict(kind="tree", a=8.0, b=-1.0, c=0.7), 3.3),
]
USED_TOL = 1e-6  # both solves stop at the reference's 1e-6 residual; they differ by far less


def _full(lat):
    ex = lat.export()
    d = lattice_dict(ex)
    d["m"] = ex["m"]
    d.update(lat.strengths())
    return d


def _two_figures(v, want):
    decimals = len(repr(want).split(".")[1])
    return round(v, decimals) == pytest.approx(want)


@pytest.mark.parametrize("name,kw,want", SCENES, ids=[s[0] for s in SCENES])
def test_used_standing(solver, name, kw, want):
    lat = O.Lattice.scene(**kw)
    used, info = solver.used_standing(_full(lat), sc.options(max_iter=20000))
    ref = lat.used_standing()
    assert info["status"] == sc.OK
    assert np.abs(used - ref).max() <= USED_TOL * max(ref.max(), 1.0)
    assert _two_figures(used.max(), want)


@pytest.mark.parametrize("name,kw,want", SCENES, ids=[s[0] for s in SCENES])
def test_settle(solver, name, kw, want):
    lat = O.Lattice.scene(**kw)
    fell, rounds, gone, info = solver.settle(_full(lat), sc.options(max_iter=20000))
    ref_fell, ref_rounds, ref_gone = lat.settle()
    assert info["status"] == sc.OK
    assert rounds == ref_rounds
    assert (gone == ref_gone).all()
    assert fell == pytest.approx(ref_fell, rel=1e-12, abs=1e-15)
    if want < 1.0:  # nothing is over its strength: the first round breaks nothing
        assert rounds == 1 and fell == 0.0
