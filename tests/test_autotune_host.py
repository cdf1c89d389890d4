"""Host logic of the batch autotuner (no GPU): the sample spread over the batch's sizes,
cache keys that do not depend on the pieces' order."""
import numpy as np

from statics_cuda import autotune


def _pieces(sizes):
    return [(np.zeros((n, 1, 1), np.uint8), np.ones((n, 1, 1), np.float32)) for n in sizes]


def test_sample_spans_sizes():
    pieces = _pieces(range(1, 101))
    got = [p[0].size for p in autotune.sample(pieces, 5)]
    assert got == [1, 26, 50, 75, 100] or got == [1, 26, 51, 75, 100]
    assert [p[0].size for p in autotune.sample(_pieces([3, 1, 2]), 5)] == [1, 2, 3]


def test_key_ignores_order_and_repeats():
    a = autotune._key([4096, 512, 512], 1, 1e-8)
    b = autotune._key([512, 4096], 1, 1e-8)
    assert a == b
    assert a != autotune._key([512, 4096], 0, 1e-8)
    assert autotune.size_class(np.zeros((3, 5, 7))) == 128
