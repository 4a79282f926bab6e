"""Host logic of the batched launch (no GPU): part sizes, seeds, and the
split of a union's values by the vertex offset table."""
import numpy as np

from ipregel_b200 import batch as B


def test_log_uniform_sizes_deterministic_and_bounded():
    a = B.log_uniform_sizes(4096, 1024, 65536, seed=1)
    b = B.log_uniform_sizes(4096, 1024, 65536, seed=1)
    np.testing.assert_array_equal(a, b)
    assert a.min() >= 1024 and a.max() <= 65536
    # log-uniform: about half the parts below the geometric midpoint 8192
    assert 0.45 < np.mean(a < 8192) < 0.55
    assert not np.array_equal(a, B.log_uniform_sizes(4096, 1024, 65536, seed=2))


def test_part_seeds_distinct():
    seeds = {B.part_seed(1, i) for i in range(4096)}
    assert len(seeds) == 4096


def test_split_by_offsets_relabels():
    voff = np.array([0, 3, 3, 7], dtype=np.uint64)
    labels = np.array([0, 0, 2, 3, 3, 5, 6], dtype=np.uint32)
    parts = B.split_by_offsets(labels, voff, relabel=True)
    assert [p.tolist() for p in parts] == [[0, 0, 2], [], [0, 0, 2, 3]]
    dist = np.array([0, 1, 2, 0, 4, 4, 9], dtype=np.uint32)
    parts = B.split_by_offsets(dist, voff)
    assert [p.tolist() for p in parts] == [[0, 1, 2], [], [0, 4, 4, 9]]
