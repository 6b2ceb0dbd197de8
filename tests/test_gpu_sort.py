"""Parity of the GPU SORT path (params.h:46 SORT=1: GPU.cu:351-395 per-cell
sort, kernel.cu:400-467 pruned neighbour scans) with the oracle's SORT
restatement: identical per-point neighbour sets and the same number of
candidate evaluations, for the indexed (n == k) and unindexed (n > k) sort
dimension, both dtypes and every distance model."""
import numpy as np
import pytest

from gpu_self_join_b200 import JoinConfig, SelfJoin

pytestmark = pytest.mark.gpu


def canon(counts, table):
    counts = np.asarray(counts, dtype=np.int64)
    seg = np.repeat(np.arange(counts.size), counts)
    return np.asarray(table)[np.lexsort((np.asarray(table), seg))]


def check(oracle, pts, eps, k, reorder=False, ilp=0, sc=False, qr=False, host=False):
    ocfg = oracle.OracleConfig(k=k, reorder=reorder, ilp=ilp, shortcircuit=sc, sort=True)
    oc, _, on = oracle.join_lists(pts, eps, ocfg)
    _, _, ocand = oracle.join_counts(pts, eps, ocfg)
    cfg = JoinConfig(indexed_dims=k, reorder=reorder, ilp=ilp, shortcircuit=sc, query_reorder=qr, sort=True)
    with SelfJoin(0) as sj:
        if host:
            st, gc, gt = sj.run_host(pts, eps, cfg)
        else:
            st = sj.run(pts, eps, cfg)
            gc, gt = sj.counts(), sj.table()
    if pts.shape[0]:
        assert st["join_path"] == 4
    assert np.array_equal(gc, oc), f"counts differ at {np.flatnonzero(gc != oc)[:10]}"
    assert np.array_equal(canon(gc, gt), on)
    assert st["candidates"] == ocand
    return st


@pytest.mark.parametrize("n,k,dtype,eps", [(2, 2, np.float32, 1.0), (3, 2, np.float32, 1.5),
                                           (5, 3, np.float64, 2.0), (6, 6, np.float32, 2.5),
                                           (4, 1, np.float32, 0.8), (7, 7, np.float64, 3.0)])
def test_sort_matches_oracle(oracle, n, k, dtype, eps):
    rng = np.random.default_rng(3 + n)
    pts = rng.uniform(0, 20, size=(20000, n)).astype(dtype)
    check(oracle, pts, eps, k)


@pytest.mark.parametrize("reorder,ilp,sc,qr", [(True, 0, False, False), (False, 2, False, True),
                                               (True, 4, True, True)])
def test_sort_with_switches(oracle, reorder, ilp, sc, qr):
    rng = np.random.default_rng(17)
    pts = (rng.normal(0, 1, size=(15000, 5)) * np.array([5, 1, 3, 0.5, 2])).astype(np.float64)
    check(oracle, pts, 0.6, 3, reorder=reorder, ilp=ilp, sc=sc, qr=qr)


def test_sort_ties_and_clusters(oracle):
    rng = np.random.default_rng(23)
    pts = rng.integers(0, 16, size=(12000, 3)).astype(np.float32) * 0.25
    check(oracle, pts, 0.5, 2)
    check(oracle, pts, 0.5, 3)


def test_sort_host_result(oracle):
    rng = np.random.default_rng(29)
    pts = rng.uniform(0, 10, size=(20000, 3)).astype(np.float32)
    check(oracle, pts, 0.4, 2, host=True)


@pytest.mark.parametrize("N", [0, 1, 2])
def test_sort_tiny(oracle, N):
    pts = np.arange(N * 3, dtype=np.float32).reshape(N, 3) * 0.1
    check(oracle, pts, 1.0, 2)


def test_sort_exact_gap_window(oracle):
    # partners exactly eps apart in the sort dimension: the strict window of
    # the pruned scan drops one direction, the GPU drops the same pairs
    rng = np.random.default_rng(31)
    m, eps = 10000, 0.5
    base = rng.uniform(0, 20, size=(m, 3))
    base[:, 2] = rng.integers(0, 80, m) * eps
    partner = base.copy()
    partner[:, 2] += eps
    pts = np.concatenate([base, partner]).astype(np.float32)[rng.permutation(2 * m)]
    full, _, _ = oracle.join_counts(pts, eps, oracle.OracleConfig(k=2))
    st = check(oracle, pts, eps, 2)
    assert st["total_pairs"] < int(full.sum())
