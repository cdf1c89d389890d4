"""The CPU restatement of statics::gather (statics/src/gather.rs): a coarser level measured
from a finer one. Pinned by the reference's own test (a_bar_weighs_as_much, gather.rs:401-412)
and by the figures its docs give for a full cell of stone (docs/statics.md:166-175, made by
`statics full`, statics/examples/statics.rs:348-369)."""
import numpy as np
import pytest

from oracle import oracle as O

SECTION = 0.336  # lattice.rs:25, both classes


def _origin_cell(lat, level):
    """statics.rs:355-366: the beams of the cell keyed by the origin, by class (0: 180°,
    1: 90°), as (section / s^2, strength / the material's)."""
    e, mats = lat.export(), lat.materials()
    s = 0.125 * 2 ** level
    mid = np.full(3, 0.5 * s)
    out = {0: [], 1: []}
    for q in range(0, lat.n_bonds, 4):
        x, y = e["x"][e["bi"][q]], e["x"][e["bj"][q]]
        if abs(np.linalg.norm(x - mid) - s / 2) > 1e-9 or abs(np.linalg.norm(y - mid) - s / 2) > 1e-9:
            continue
        u, v = x - mid, y - mid
        k = int(round(1 + u @ v / (np.linalg.norm(u) * np.linalg.norm(v))))
        out[k].append((4 * e["a"][q] / s ** 2, mats["stronger"][q]))
    return {k: np.array(v) for k, v in out.items()}


def test_a_bar_weighs_as_much():
    """gather.rs:401-412: a bar of steel, gathered three times, weighs as much at every level."""
    lat = O.Lattice.block(O.STEEL, [-4.5, -1.0, -1.0], [4.5, 1.0, 1.0], [4.0, 0.2, 0.2])
    whole = lat.export()["m"].sum()
    for _ in range(3):
        lat = lat.gathered()
        assert abs(lat.export()["m"].sum() / whole - 1.0) < 1e-9


def test_full_cell_of_stone_as_the_docs_give():
    """docs/statics.md:166-172: measured as it is, a full cell of stone a level up has beams
    between faces at right angles two and a half times the section of a full cell's, those
    between opposite faces three quarters, its strength within a tenth."""
    f = O.full(O.STONE)
    assert 0.7 < f[0, 0] / SECTION < 0.8
    assert 2.4 < f[1, 0] / SECTION < 2.6
    assert np.all(np.abs(f[:, 1] - 1.0) < 0.1)


def test_full_cell_is_its_material_at_every_level():
    """docs/statics.md:173-177: measured against a full cell, a full cell is its material a
    level up and two levels up (3 beams at 180°, 12 at 90°, each SECTION, strength as the
    material's); measured as it is, two levels up the right-angle beams are nearly six times
    SECTION (docs/statics.md:168-170)."""
    for against, levels in ((True, (1, 2)), (False, (2,))):
        lat = O.Lattice.block(O.STONE, [-1.0] * 3, [1.0] * 3, [9.0] * 3)
        for level in (1, 2):
            lat = lat.gathered(against)
            if level not in levels:
                continue
            cell = _origin_cell(lat, level)
            assert len(cell[0]) == 3 and len(cell[1]) == 12
            if against:
                for k in (0, 1):
                    assert np.allclose(cell[k][:, 0], SECTION, rtol=1e-12, atol=0)
                    assert np.allclose(cell[k][:, 1], 1.0, rtol=1e-12, atol=0)
            else:
                assert 5.0 < cell[1][:, 0].mean() / SECTION < 6.0


def test_gathered_level_structure():
    """gather.rs:230-395 as a level of its own: one node per face between coarse cells
    (their sites keyed to the level, lesser first), beams of four bonds inside one coarse
    cell each, no beam between two held faces, a held cell's faces held."""
    lat = O.Lattice.scene("cantilever", O.STONE, 0.5, 3.0)
    for level in (1, 2):
        lat = lat.gathered()
        e = lat.export()
        a = e["around"]
        assert np.all(a % (2 ** level) == 0)
        assert all(tuple(p) < tuple(q) for p, q in zip(a[:, 0], a[:, 1]))
        assert len({(tuple(p), tuple(q)) for p, q in zip(a[:, 0], a[:, 1])}) == lat.n_nodes
        assert lat.n_bonds % 4 == 0
        bi, bj = e["bi"].reshape(-1, 4), e["bj"].reshape(-1, 4)
        assert np.all(bi == bi[:, :1]) and np.all(bj == bj[:, :1])
        for i, j in zip(bi[:, 0], bj[:, 0]):
            shared = {tuple(s) for s in a[i]} & {tuple(s) for s in a[j]}
            assert len(shared) >= 1
            assert not (e["held"][i] and e["held"][j])
        assert e["held"].any() and not e["held"].all()


def test_gather_is_the_same_twice_and_on_any_threads():
    """docs/statics.md:186: every level gives the same answer twice; the cells are measured
    in parallel (bodies.rs:51-69) with no effect on the result."""
    base = O.Lattice.scene("portico", O.STONE, 1, 0.5)
    outs = []
    for threads in (1, 0, 1):
        O.set_threads(threads)
        try:
            outs.append(base.gathered().export())
        finally:
            O.set_threads(0)
    for other in outs[1:]:
        for key in outs[0]:
            assert np.array_equal(outs[0][key], other[key]), key


def _digest(d: dict, nodes: int, bonds: int) -> dict:
    """tests/golden/make_gather_golden.py's digest of a gathered level."""
    import hashlib
    h = hashlib.sha256()
    for k in ("x", "m", "held", "around", "bi", "bj", "p", "n", "a", "d", "e", "g", "ft", "fc", "fs"):
        h.update(np.ascontiguousarray(d[k]).tobytes())
    return {"nodes": nodes, "bonds": bonds, "weight": float(d["m"].sum()), "sha256": h.hexdigest()[:32]}


GOLDEN_SCENES = {
    "bar": lambda: O.Lattice.block(O.STEEL, [-4.5, -1.0, -1.0], [4.5, 1.0, 1.0], [4.0, 0.2, 0.2]),
    "cantilever": lambda: O.Lattice.scene("cantilever", O.STONE, 0.5, 3.0),
    "pendant_apart": lambda: O.Lattice.scene("pendant", O.STONE, 1),
}


def _golden():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_gather.json")
    return json.load(open(path))


def test_oracle_gather_matches_committed_levels():
    """The oracle's gathered levels are the committed ones (tests/golden/oracle_gather.json),
    bit for bit: any change to the restatement shows here."""
    rows = _golden()
    assert len(rows) == 18
    for name, make in GOLDEN_SCENES.items():
        for against in (True, False):
            lat = make()
            for level in (1, 2, 3):
                lat = lat.gathered(against)
                e = lat.export()
                e.update(lat.strengths())
                want = next(r for r in rows if r["scene"] == name and r["against_full"] == against
                            and r["level"] == level)
                got = _digest(e, lat.n_nodes, lat.n_bonds)
                assert got == {k: want[k] for k in got}, (name, against, level)
