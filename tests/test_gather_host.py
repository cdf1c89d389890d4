"""The library's statics::gather (sc_gather on the host's cores, no device) against the CPU
restatement of statics/src/gather.rs: the same gathered lattice, array for array and bit for
bit, level after level, on the reference's own bar (gather.rs:403-405) and example scenes
(statics/examples/statics.rs), measured against a full cell and as it is; and the same for
the device kernel's per-cell code run on the host (SC_GATHER_EMULATE)."""
import numpy as np
import pytest

import statics_cuda as sc
from oracle import oracle as O

NAMES = list(sc.MATERIALS)  # the oracle's material indexes (STONE..LEAVES) in the same order
KEYS = ("x", "m", "held", "around", "bi", "bj", "p", "n", "a", "d", "e", "g", "ft", "fc", "fs")


def _dict(lat, level):
    d = lat.export()
    d.update(lat.strengths())
    mats = lat.materials()
    d["mat"], d["bmat"] = mats["node"], mats["bond"]
    d["level"] = level
    return d


def _scene(name):
    if name == "bar":
        return O.Lattice.block(O.STEEL, [-4.5, -1.0, -1.0], [4.5, 1.0, 1.0], [4.0, 0.2, 0.2])
    if name == "cantilever":
        return O.Lattice.scene("cantilever", O.STONE, 0.5, 3.0)
    if name == "rock":  # statics.rs:114-133: stone over soil, two materials a cell may mix
        return O.Lattice.scene("rock", O.STONE, 1.0, 0.5)
    if name.startswith("pendant"):
        # statics.rs:285-303: a held wall; let go, a layer gone, so a cell's matter no longer
        # joins all its faces and beams go only between the faces it joins
        return O.Lattice.scene("pendant", O.STONE, 1 if name.endswith("apart") else 0)
    return O.Lattice.scene("portico", O.STONE, 1, 0.5)


@pytest.mark.parametrize("emulated", [False, True])
@pytest.mark.parametrize("against_full", [True, False])
@pytest.mark.parametrize("name", ["bar", "cantilever", "portico", "pendant", "pendant_apart", "rock"])
def test_library_gather_is_the_oracles(name, against_full, emulated, monkeypatch):
    """emulated: the cells measured by the device kernel's own code (gf_measure_cell) run by
    one host thread a cell, so the CPU checks the kernel's indexing and order of operations."""
    if emulated:
        monkeypatch.setenv("SC_GATHER_EMULATE", "1")
    ora = _scene(name)
    lib = _dict(ora, 0)
    for level in (1, 2, 3):
        ora = ora.gathered(against_full)
        lib = sc.gather(lib, NAMES, against_full)
        want = _dict(ora, level)
        assert lib["level"] == level
        for key in KEYS + ("mat", "bmat"):
            assert lib[key].shape == np.asarray(want[key]).shape, (level, key)
            assert np.array_equal(lib[key], want[key]), (level, key)


def test_library_full_is_the_oracles():
    """gather.rs:203-226 for every reference material, bit for bit."""
    for k, name in enumerate(NAMES):
        assert np.array_equal(sc.gather_full(name), O.full(k)), name


def test_library_bar_weighs_as_much():
    """gather.rs:401-412 through the library."""
    lat = _dict(_scene("bar"), 0)
    whole = lat["m"].sum()
    for _ in range(3):
        lat = sc.gather(lat, NAMES)
        assert abs(lat["m"].sum() / whole - 1.0) < 1e-9


def test_library_gather_on_any_threads():
    lat = _dict(_scene("portico"), 0)
    one = sc.gather(lat, NAMES, threads=1)
    many = sc.gather(lat, NAMES, threads=7)
    for key in KEYS + ("mat",):
        assert np.array_equal(one[key], many[key]), key


def test_library_gather_rejects_bad_input():
    lat = _dict(_scene("cantilever"), 0)
    bad = dict(lat, mat=lat["mat"].copy())
    bad["mat"][0] = len(NAMES)  # a material not in the table
    with pytest.raises(sc.StaticsError):
        sc.gather(bad, NAMES)
    bad = dict(lat, a=lat["a"].copy())
    bad["a"][5] = 0.0  # a bond without section
    with pytest.raises(sc.StaticsError):
        sc.gather(bad, NAMES)
    # a bond between two nodes that share no cell (the reference panics: "a beam is inside a cell")
    around = lat["around"]
    far = next(v for v in range(len(around))
               if not ({tuple(s) for s in around[v]} & {tuple(s) for s in around[lat["bi"][0]]}))
    bad = dict(lat, bj=lat["bj"].copy())
    bad["bj"][0] = far
    with pytest.raises(sc.StaticsError):
        sc.gather(bad, NAMES)
    bad = dict(lat, bi=lat["bi"].copy())
    bad["bi"][0] = len(around)  # out of range
    with pytest.raises(sc.StaticsError):
        sc.gather(bad, NAMES)


def test_library_gather_of_nothing():
    """An empty lattice gathers to an empty level one up."""
    z = np.zeros
    lat = dict(x=z((0, 3)), held=z(0, np.uint8), around=z((0, 2, 3), np.int64), bi=z(0, np.int64),
               bj=z(0, np.int64), p=z((0, 3)), n=z((0, 3)), a=z(0), d=z(0), e=z(0), g=z(0), m=z(0), ft=z(0),
               fc=z(0), fs=z(0), mat=z(0, np.int32), level=2)
    out = sc.gather(lat, NAMES)
    assert out["level"] == 3 and out["x"].shape == (0, 3) and out["bi"].shape == (0,)


def test_library_gather_matches_committed_levels():
    """The library's gathered levels are the oracle's committed ones
    (tests/golden/oracle_gather.json), hashed array by array."""
    from test_gather_oracle import GOLDEN_SCENES, _digest, _golden
    rows = _golden()
    for name, make in GOLDEN_SCENES.items():
        for against in (True, False):
            lat = _dict(make(), 0)
            for level in (1, 2, 3):
                lat = sc.gather(lat, NAMES, against)
                want = next(r for r in rows if r["scene"] == name and r["against_full"] == against
                            and r["level"] == level)
                got = _digest(lat, len(lat["m"]), len(lat["bi"]))
                assert got == {k: want[k] for k in got}, (name, against, level)
