"""statics::gather with the cells measured on the GPU (sc_gather with a context: one thread
block a cell, k_gather_cells) against the CPU restatement of statics/src/gather.rs: the same
gathered lattice, array for array and bit for bit, level after level."""
import numpy as np
import pytest

import statics_cuda as sc
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NAMES = list(sc.MATERIALS)
KEYS = ("x", "m", "held", "around", "bi", "bj", "p", "n", "a", "d", "e", "g", "ft", "fc", "fs")


def _dict(lat, level):
    d = lat.export()
    d.update(lat.strengths())
    mats = lat.materials()
    d["mat"], d["bmat"] = mats["node"], mats["bond"]
    d["level"] = level
    return d


@pytest.mark.parametrize("against_full", [True, False])
@pytest.mark.parametrize("scene", [("cantilever", O.STONE, 0.5, 3.0, 0.0), ("portico", O.STONE, 1, 0.5, 0.0),
                                   ("tree", O.STONE, 8.0, 1.0, 0.0)])
def test_device_gather_is_the_oracles(solver, scene, against_full):
    ora = O.Lattice.scene(*scene)
    lib = _dict(ora, 0)
    launched = sc.launches()
    for level in (1, 2, 3):
        ora = ora.gathered(against_full)
        lib = solver.gather(lib, NAMES, against_full)
        want = _dict(ora, level)
        for key in KEYS + ("mat", "bmat"):
            assert lib[key].shape == np.asarray(want[key]).shape, (level, key)
            assert np.array_equal(lib[key], want[key]), (level, key)
    assert sc.launches() >= launched + 3  # one kernel a level: the device measured the cells


def test_device_bar_weighs_as_much(solver):
    """gather.rs:401-412 with the cells measured on the GPU."""
    lat = _dict(O.Lattice.block(O.STEEL, [-4.5, -1.0, -1.0], [4.5, 1.0, 1.0], [4.0, 0.2, 0.2]), 0)
    whole = lat["m"].sum()
    for _ in range(3):
        lat = solver.gather(lat, NAMES)
        assert abs(lat["m"].sum() / whole - 1.0) < 1e-9
