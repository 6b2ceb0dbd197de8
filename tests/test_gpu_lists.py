"""The list sorts of the pair-to-table step (gsj_place.cu) at the sizes where
the algorithm changes: a warp network per list up to 256 entries (32, 64, 128,
256-entry networks), a CTA network up to 4096 (512 ... 4096 entries), CTA
radix passes above.  Clusters of m coincident points make lists of exactly m
entries (the cluster's ids, ascending), with the ids of all clusters shuffled
so every list is unordered before its sort."""
import numpy as np
import pytest

from gpu_self_join_b200 import JoinConfig, SelfJoin

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513, 1023, 1024, 1025, 2047,
         2048, 2049, 4095, 4096, 4097, 6000]


def clusters(n, dtype, seed):
    rng = np.random.default_rng(seed)
    sizes = np.array([m for m in SIZES for _ in range(2)])  # two clusters of every size
    centres = np.arange(sizes.size, dtype=np.float64)[:, None] * 10.0 + np.zeros((1, n))
    pts = np.repeat(centres, sizes, axis=0)
    label = np.repeat(np.arange(sizes.size), sizes)
    perm = rng.permutation(pts.shape[0])
    return pts[perm].astype(dtype), label[perm], sizes


@pytest.mark.parametrize("n,dtype,ilp", [(6, np.float32, 0), (3, np.float32, 2), (5, np.float64, 0)])
def test_lists_sorted_at_every_size_class(n, dtype, ilp):
    pts, label, sizes = clusters(n, dtype, 7 + n)
    with SelfJoin(0) as sj:
        st = sj.run(pts, 1.0, JoinConfig(indexed_dims=min(n, 3), ilp=ilp, plain=True))
        counts, table = sj.counts(), sj.table()
    assert st["join_path"] in (0, 2)
    assert np.array_equal(counts, sizes[label])
    order = np.argsort(label, kind="stable")  # ids of each cluster, ascending
    members = np.split(order.astype(np.uint32), np.cumsum(sizes)[:-1])
    off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    for q in range(pts.shape[0]):
        assert np.array_equal(table[off[q]:off[q + 1]], members[label[q]]), f"list of point {q}"
