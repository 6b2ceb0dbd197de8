"""CPU tests of the oracle's SORT restatement (GPU.cu:351-395 per-cell sort,
kernel.cu:400-467 pruned scans): the pruned scans report only pairs the full
scan reports, evaluate fewer candidates, and on seeded uniform inputs find
every pair; the reference SORT=1 builds pin it in test_ref_pins."""
import numpy as np
import pytest


def _lists(oracle, pts, eps, **kw):
    return oracle.join_lists(pts, eps, oracle.OracleConfig(**kw))


@pytest.mark.parametrize("n,k,dtype,eps", [(2, 2, np.float32, 1.0), (3, 2, np.float32, 1.5),
                                           (5, 3, np.float64, 2.0), (6, 6, np.float32, 2.5),
                                           (4, 1, np.float32, 0.8)])
def test_sort_finds_the_full_scans_pairs(oracle, n, k, dtype, eps):
    rng = np.random.default_rng(3)
    pts = rng.uniform(0, 20, size=(6000, n)).astype(dtype)
    c0, o0, l0 = _lists(oracle, pts, eps, k=k)
    c1, o1, l1 = _lists(oracle, pts, eps, k=k, sort=True)
    assert np.array_equal(c0, c1) and np.array_equal(l0, l1)
    _, _, cand0 = oracle.join_counts(pts, eps, oracle.OracleConfig(k=k))
    _, _, cand1 = oracle.join_counts(pts, eps, oracle.OracleConfig(k=k, sort=True))
    assert cand1 < cand0


def test_sort_subset_with_ties(oracle):
    # many equal values in the sort dimension: the window still reports only
    # pairs within eps, never a pair the full scan misses
    rng = np.random.default_rng(11)
    pts = rng.integers(0, 12, size=(4000, 3)).astype(np.float32) * 0.5
    eps = 1.0
    c0, o0, l0 = _lists(oracle, pts, eps, k=2)
    c1, o1, l1 = _lists(oracle, pts, eps, k=2, sort=True)
    assert np.all(c1 <= c0)
    for q in range(0, pts.shape[0], 37):
        assert set(l1[o1[q]:o1[q + 1]].tolist()) <= set(l0[o0[q]:o0[q + 1]].tolist())


def test_sort_indexed_break_is_exact(oracle):
    # sort dimension indexed (n == k): the scan stops at the first point more
    # than eps away in dim 0, which no later point of the cell can beat
    rng = np.random.default_rng(5)
    pts = rng.normal(0, 3, size=(5000, 2)).astype(np.float32)
    for eps in (0.3, 0.9):
        c0, _, l0 = _lists(oracle, pts, eps, k=2)
        c1, _, l1 = _lists(oracle, pts, eps, k=2, sort=True)
        assert np.array_equal(c0, c1) and np.array_equal(l0, l1)


def test_sort_empty_and_single(oracle):
    for N in (0, 1):
        pts = np.zeros((N, 3), np.float32)
        c, o, l = _lists(oracle, pts, 1.0, k=2, sort=True)
        assert c.size == N and l.size == N
