"""Parity on the benchmarked workloads at their full sizes.

The oracle cannot join 20M points within a test, so every workload is checked
on a seeded sample of queries: the CUDA path (through the C ABI) joins the
whole workload, and each sampled query's neighbour list must equal the
oracle's list for that query exactly (integers, bit-exact: the oracle
restates the reference's algorithm 3 with the reference's arithmetic).

The second oracle is the double-precision decision on the same float inputs.
The FP32 result of the reference's arithmetic differs from it only on pairs
whose distance lies within the FP32 rounding of the sum from eps; the test
counts those boundary flips per workload and checks that every flipped pair
is such a boundary pair.
"""
import numpy as np
import pytest

from gpu_self_join_b200 import JoinConfig, SelfJoin, synth

pytestmark = pytest.mark.gpu

SAMPLE = 2000


def _config(w):
    return JoinConfig(indexed_dims=w.k, reorder=w.reorder, shortcircuit=w.shortcircuit, ilp=w.ilp, stamp=w.stamp,
                      query_reorder=w.query_reorder)


def _lists_of(counts, table, q):
    starts = np.zeros(counts.size + 1, dtype=np.int64)
    np.cumsum(counts, dtype=np.int64, out=starts[1:])
    return [np.sort(table[starts[i]:starts[i + 1]]) for i in q]


@pytest.mark.parametrize("name", ["c2_gmm2d", "c3_gmm6d", "c4_derived18d", "c5_heavy90d"])
def test_full_size_sampled_lists(oracle, name):
    w = synth.WORKLOADS[name]
    pts = synth.generate(name)
    with SelfJoin(0) as sj:
        st = sj.run(pts, w.eps, _config(w))
        counts = sj.counts()
        table = sj.table()
    assert st["total_pairs"] == int(counts.sum(dtype=np.uint64)) == table.size
    q = np.sort(np.random.default_rng(4242 + w.index).choice(pts.shape[0], SAMPLE, replace=False)).astype(np.uint32)
    ocfg = oracle.OracleConfig(k=w.k, reorder=w.reorder, ilp=w.ilp, shortcircuit=w.shortcircuit)
    oc, ol = oracle.sample_lists(pts, w.eps, ocfg, q)
    assert np.array_equal(counts[q], oc), f"list lengths differ at queries {q[np.flatnonzero(counts[q] != oc)][:10]}"
    got = np.concatenate(_lists_of(counts, table, q))
    assert np.array_equal(got, ol)

    # second oracle: the double-precision decision on the same inputs
    fc, fl = oracle.sample_lists(pts, w.eps, oracle.OracleConfig(k=w.k, model=oracle.MODEL_FP64), q)
    f_starts = np.concatenate([[0], np.cumsum(fc, dtype=np.int64)])
    o_starts = np.concatenate([[0], np.cumsum(oc, dtype=np.int64)])
    eps = float(np.float32(w.eps))
    tol = (2 * pts.shape[1] + 8) * 2.0 ** -24  # relative rounding room of the FP32 sum
    flips_in, flips_out = 0, 0
    for j, i in enumerate(q):
        a = ol[o_starts[j]:o_starts[j + 1]]
        b = fl[f_starts[j]:f_starts[j + 1]]
        for c in np.setxor1d(a, b):
            d2 = float(np.sum((pts[c].astype(np.float64) - pts[i].astype(np.float64)) ** 2))
            assert abs(d2 - eps * eps) <= tol * eps * eps, f"pair ({i}, {c}) flips away from the boundary"
        flips_in += np.setdiff1d(a, b).size   # within eps in FP32 only
        flips_out += np.setdiff1d(b, a).size  # within eps in FP64 only
    print(f"\n{name}: {SAMPLE} queries, {ol.size} pairs; FP64 boundary flips: {flips_in} FP32-only, "
          f"{flips_out} FP64-only")
    assert flips_in + flips_out <= max(4, ol.size // 10000)


@pytest.mark.parametrize("case", ["warp", "tile", "screen"])
def test_rerun_after_short_buffer(oracle, case):
    """GSJ_FLAG_EXACT_SIZE runs the first pass with no pair buffer at all, so
    the pass is always repeated at the counted size: the path a short
    estimate takes.  The lists must not change."""
    rng = np.random.default_rng(77)
    if case == "warp":
        pts = rng.uniform(0, 5, size=(15000, 7)).astype(np.float32)
        kw = dict(indexed_dims=6, stamp=True)
        eps, path = 1.0, 0
    else:
        n = 12 if case == "tile" else 18
        base = rng.uniform(0, 10, size=(4, n))[rng.integers(0, 4, 12000)]
        pts = (base + rng.standard_normal((12000, n)) * 0.8).astype(np.float32)
        kw = dict(indexed_dims=6, stamp=(case == "screen"))
        eps, path = 3.0, (2 if case == "tile" else 3)
    with SelfJoin(0) as sj:
        st0 = sj.run(pts, eps, JoinConfig(**kw))
        c0, t0 = sj.counts(), sj.table()
        st1 = sj.run(pts, eps, JoinConfig(exact_size=True, **kw))
        c1, t1 = sj.counts(), sj.table()
    assert st0["join_path"] == st1["join_path"] == path
    assert st1["reruns"] >= 1
    assert np.array_equal(c0, c1) and np.array_equal(t0, t1)
    oc, _, on = oracle.join_lists(pts, eps, oracle.OracleConfig(k=6))
    assert np.array_equal(c1, oc)
    seg = np.repeat(np.arange(c1.size), c1.astype(np.int64))
    assert np.array_equal(t1[np.lexsort((t1, seg))], on)
