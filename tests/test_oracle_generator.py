"""The checker's own piece generator (oracle/generate_oracle.cpp) makes the same pieces
as the library's sc_generate_piece, byte for byte: the CPU reference arm builds its
inputs with the former and never loads the product library."""
import numpy as np
import pytest

import statics_cuda as sc
from oracle import oracle as O


@pytest.mark.parametrize("dims", [(16, 16, 16), (24, 32, 48), (48, 16, 24), (64, 64, 64), (17, 9, 33), (1, 1, 2)])
@pytest.mark.parametrize("k_dist", [sc.K_UNIFORM, sc.K_LOGNORMAL])
def test_generator_matches_library(dims, k_dist):
    for seed in (0, 7, 10_000 + 511):
        st_lib, k_lib = sc.generate_piece(*dims, seed, k_dist)
        st_or, k_or = O.generate_piece(*dims, seed, k_dist)
        assert st_lib.tobytes() == st_or.tobytes()
        assert k_lib.tobytes() == k_or.tobytes()


def test_generator_definition():
    """The definition itself: bottom layer held, every kept cell joined to it, k in
    range and zero off the piece."""
    st, k = O.generate_piece(32, 32, 32, 3, O.K_LOGNORMAL)
    assert (st[:, :, 0] == O.CELL_HELD).all()
    assert ((st[:, :, 1:] == O.CELL_FREE) | (st[:, :, 1:] == O.CELL_EMPTY)).all()
    kept = st != O.CELL_EMPTY
    assert (k[~kept] == 0).all()
    assert ((k[kept] >= 0.1) & (k[kept] <= 10.0)).all()
    # every kept cell reaches the bottom layer through kept cells (a flood from it)
    seen = np.zeros_like(kept)
    seen[:, :, 0] = True
    while True:
        grow = seen.copy()
        for a in range(3):
            for s in (1, -1):
                grow |= np.roll(seen, s, axis=a) & kept & ~_wrapped(a, s, kept.shape)
        if (grow == seen).all():
            break
        seen = grow
    assert (seen == kept).all()
    _, ku = O.generate_piece(16, 16, 16, 3, O.K_UNIFORM)
    assert ((ku[ku > 0] >= 0.5) & (ku[ku > 0] <= 2.0)).all()


def _wrapped(axis, shift, shape):
    """The cells np.roll filled from the opposite edge."""
    m = np.zeros(shape, bool)
    idx = [slice(None)] * 3
    idx[axis] = 0 if shift == 1 else -1
    m[tuple(idx)] = True
    return m
