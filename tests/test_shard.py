"""The batch split across GPUs (statics_cuda.shard): longest processing time first."""
import numpy as np
import pytest

from statics_cuda import shard


@pytest.mark.parametrize("ranks", [1, 2, 3, 8])
def test_lpt_covers_and_balances(ranks):
    w = [int(v) for v in np.random.default_rng(ranks).integers(1, 10_000, size=512)]
    split = shard.lpt_split(w, ranks)
    assert len(split) == ranks
    assert sorted(i for s in split for i in s) == list(range(len(w)))
    loads = shard.loads(w, split)
    assert max(loads) <= sum(w) / ranks + max(w)
    # the 4/3 bound against the best split's lower bound (the mean load, the heaviest piece)
    assert max(loads) <= 4 / 3 * max(sum(w) / ranks, max(w)) + 1e-9


def test_lpt_known_split():
    # a case where LPT misses the best split (14: 5 + 5 + 4 against 4 + 3 + 3 + 3) but
    # stays within 4/3 of it: 5, 4, 3, 3 to one rank, 5, 4, 3 to the other
    w = [5, 5, 4, 4, 3, 3, 3]
    split = shard.lpt_split(w, 2)
    assert split == [[0, 2, 4, 6], [1, 3, 5]]
    assert shard.loads(w, split) == [15, 12]
    assert 15 <= 4 / 3 * 14
    assert shard.lpt_split([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard.lpt_split(w, 0)
