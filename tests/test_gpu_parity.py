"""Parity of the CUDA path (through the C ABI) with the oracle, which restates
the reference's algorithm 3 with the reference's arithmetic.  Integer output:
the per-point neighbour sets must be identical (bit-exact), compared as
per-point sorted lists."""
import json
import os

import numpy as np
import pytest

from gpu_self_join_b200 import JoinConfig, SelfJoin, gdsjoin, synth

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def canon(counts, table):
    """Per-point lists sorted ascending (list order is not part of the output)."""
    counts = np.asarray(counts, dtype=np.int64)
    seg = np.repeat(np.arange(counts.size), counts)
    return np.asarray(table)[np.lexsort((np.asarray(table), seg))]


def run_gpu(points, eps, **kw):
    with SelfJoin(0) as sj:
        st = sj.run(points, eps, JoinConfig(**kw))
        return sj.counts(), sj.table(), st


def oracle_cfg(oracle, k, reorder=False, ilp=0, shortcircuit=False):
    return oracle.OracleConfig(k=k, reorder=reorder, ilp=ilp, shortcircuit=shortcircuit)


def assert_same(oracle, pts, eps, **kw):
    k = min(kw.get("indexed_dims", 6), pts.shape[1])
    ocfg = oracle_cfg(oracle, k, kw.get("reorder", False), kw.get("ilp", 0), kw.get("shortcircuit", False))
    oc, _, on = oracle.join_lists(pts, eps, ocfg)
    gc, gt, st = run_gpu(pts, eps, **kw)
    assert gc.shape == oc.shape
    assert np.array_equal(gc, oc), f"counts differ at {np.flatnonzero(gc != oc)[:10]}"
    assert int(gc.sum(dtype=np.uint64)) == st["total_pairs"] == gt.size
    assert np.array_equal(canon(gc, gt), on)
    return st


def test_readme_known_answer_through_gdsjoin():
    pts = np.load(os.path.join(GOLD, "test_dat_f32.npy"))
    with open(os.path.join(GOLD, "known_answers.json")) as f:
        known = json.load(f)
    num, table = gdsjoin(pts.reshape(-1).tolist(), 1.0, 2, "float")
    assert int(num.sum(dtype=np.uint64)) == known["readme_known_answer"] == 27982028
    from tests.golden.make_golden import lists_digest

    assert lists_digest(num, canon(num, table)) == known["lists_sha256_device"]


def test_reference_signatures_through_ctypes():
    """The drop-in pair with the reference's exact C signatures, bound the way
    a caller of the reference's library binds them: GDSJoinPy(float*, unsigned
    int, float, unsigned int, int, unsigned int*) (main.cu:360) then
    copyResultIntoPythonArray(unsigned int*, unsigned int) (main.cu:507), on
    the reference's test input (README.md:82 known answer)."""
    import ctypes

    import numpy.ctypeslib as npct

    from gpu_self_join_b200 import _native
    from tests.golden.make_golden import lists_digest

    _native.lib()  # the product library is built and loads
    L = ctypes.CDLL(_native.LIB_PATH)
    f32 = npct.ndpointer(dtype=np.float32, ndim=1, flags="CONTIGUOUS")
    u32 = npct.ndpointer(dtype=np.uint32, ndim=1, flags="CONTIGUOUS")
    L.GDSJoinPy.argtypes = [f32, ctypes.c_uint, ctypes.c_float, ctypes.c_uint, ctypes.c_int, u32]
    L.GDSJoinPy.restype = None
    L.copyResultIntoPythonArray.argtypes = [u32, ctypes.c_uint]
    L.copyResultIntoPythonArray.restype = None
    pts = np.load(os.path.join(GOLD, "test_dat_f32.npy"))
    with open(os.path.join(GOLD, "known_answers.json")) as f:
        known = json.load(f)
    data = np.ascontiguousarray(pts.reshape(-1), dtype=np.float32)
    num = np.zeros(pts.shape[0], dtype=np.uint32)
    L.GDSJoinPy(data, ctypes.c_uint(pts.shape[0]), ctypes.c_float(1.0), ctypes.c_uint(2), ctypes.c_int(0), num)
    total = int(num.sum(dtype=np.uint64))
    assert total == known["readme_known_answer"] == 27982028
    table = np.zeros(total, dtype=np.uint32)
    L.copyResultIntoPythonArray(table, ctypes.c_uint(total))
    assert lists_digest(num, canon(num, table)) == known["lists_sha256_device"]


@pytest.mark.parametrize("stamp", [False, True])
def test_c1_uniform_100k(oracle, stamp):
    w = synth.WORKLOADS["c1_uniform2d"]
    pts = synth.generate("c1_uniform2d")
    st = assert_same(oracle, pts, w.eps, indexed_dims=2, stamp=stamp)
    assert st["total_pairs"] > 3_000_000


CASES = [
    # n, k, dtype, reorder, ilp, sc, stamp, qr, N, eps
    (2, 2, np.float64, False, 0, False, False, False, 20000, 1.0),
    (3, 2, np.float32, False, 0, False, True, True, 20000, 1.5),
    (4, 4, np.float64, False, 0, False, True, False, 20000, 2.5),
    (5, 3, np.float64, True, 2, True, False, True, 20000, 2.0),
    (6, 6, np.float32, False, 0, False, True, False, 30000, 3.0),
    (7, 3, np.float32, True, 0, True, True, True, 20000, 2.5),
    (8, 1, np.float32, False, 4, False, False, False, 5000, 2.0),
    (18, 6, np.float32, True, 8, True, False, True, 20000, 4.0),
    (18, 6, np.float32, True, 8, False, False, True, 20000, 4.0),
    (18, 6, np.float32, False, 4, True, True, False, 20000, 4.0),
    (90, 6, np.float32, True, 8, True, False, True, 5000, 20.0),
]


@pytest.mark.parametrize("case", CASES, ids=[f"n{c[0]}k{c[1]}{np.dtype(c[2]).name}r{int(c[3])}i{c[4]}s{int(c[5])}"
                                             f"u{int(c[6])}q{int(c[7])}" for c in CASES])
def test_configs_match_oracle(oracle, case):
    n, k, dt, reorder, ilp, sc, stamp, qr, N, eps = case
    rng = np.random.default_rng(1000 + n * 10 + k)
    centres = rng.uniform(0, 20, size=(8, n))
    pts = (centres[rng.integers(0, 8, N)] + rng.standard_normal((N, n)) * rng.uniform(0.5, 3, n)).astype(dt)
    st = assert_same(oracle, pts, eps, indexed_dims=k, reorder=reorder, ilp=ilp, shortcircuit=sc, stamp=stamp,
                     query_reorder=qr)
    assert st["total_pairs"] > N  # more than the self pairs


# Tile join (float, 5 <= n <= 128, k <= 6, populated cells): every distance
# model with and without unicomp, ILP that does not divide n, the largest n.
TILE_CASES = [
    # n, k, reorder, ilp, sc, stamp, qr, N
    (5, 5, False, 0, False, False, False, 20000),
    (18, 6, True, 8, True, False, True, 20000),
    (18, 6, True, 8, False, True, False, 20000),
    (18, 6, False, 4, True, True, True, 20000),
    (33, 4, False, 3, False, False, False, 12000),
    (90, 6, True, 8, True, False, True, 8000),
    (90, 6, True, 8, True, True, False, 8000),
    (128, 6, False, 0, False, True, False, 6000),
]


def tile_points(n, N, eps, seed):
    """Clusters that fill their cells (sigma 1 in six dims, 0.1 in the rest)
    plus partners placed at distance eps, so many pairs sit on the boundary."""
    rng = np.random.default_rng(seed)
    sig = np.full(n, 0.1)
    sig[: min(6, n)] = 1.0
    nb = N // 2
    centres = rng.uniform(0, 10, size=(4, n))
    base = centres[rng.integers(0, 4, nb)] + rng.standard_normal((nb, n)) * sig
    d = rng.standard_normal((N - nb, n))
    d *= eps / np.linalg.norm(d, axis=1, keepdims=True)
    partner = base[rng.integers(0, nb, N - nb)] + d
    return np.concatenate([base, partner]).astype(np.float32)[rng.permutation(N)]


@pytest.mark.parametrize("plain", [False, True], ids=["screen", "plain"])
@pytest.mark.parametrize("case", TILE_CASES, ids=[f"n{c[0]}k{c[1]}r{int(c[2])}i{c[3]}s{int(c[4])}u{int(c[5])}q{int(c[6])}"
                                                  for c in TILE_CASES])
def test_tile_join_matches_oracle(oracle, case, plain):
    """Plain tile join and, from 16 dimensions on, the BF16 tensor-core
    screen: both must give the oracle's lists exactly."""
    n, k, reorder, ilp, sc, stamp, qr, N = case
    eps = 3.0
    pts = tile_points(n, N, eps, 2000 + n)
    st = assert_same(oracle, pts, eps, indexed_dims=k, reorder=reorder, ilp=ilp, shortcircuit=sc, stamp=stamp,
                     query_reorder=qr, plain=plain)
    screened = 16 <= n <= 126 and not plain  # n + 2 columns (the folded norm) within 128
    assert st["join_path"] == (3 if screened else 2)  # GSJ_PATH_SCREEN / GSJ_PATH_TILE
    assert st["total_pairs"] > N
    if screened:
        # every exact pair is among the rechecked ones; the screen rejects the rest
        assert st["total_pairs"] <= 2 * st["screen_rechecks"]
        assert st["screen_rechecks"] < st["candidates"]


@pytest.mark.parametrize("stamp", [False, True])
def test_screen_with_nonfinite_points(oracle, stamp):
    """A NaN and an infinite coordinate in non-indexed dimensions (the six
    indexed ones are the high-variance dims 0-5; rows 5 and 17 are outside
    REORDER's every-100th sample): those points have no neighbours, not even
    themselves, in the reference's arithmetic; every other list is unchanged,
    and the screen still rejects the bulk of the candidates."""
    pts = tile_points(18, 20000, 3.0, 77)
    pts[5, 8] = np.nan
    pts[17, 12] = np.inf
    st = assert_same(oracle, pts, 3.0, indexed_dims=6, reorder=True, ilp=8, shortcircuit=True, stamp=stamp)
    assert st["join_path"] == 3
    assert st["screen_rechecks"] < st["candidates"] // 4


@pytest.mark.parametrize("n", [6, 16, 18, 126])
def test_tiny_and_degenerate_inputs(oracle, n):
    """One point, eight identical points (one cell: the tile and screen paths
    with a single item) and exact duplicates at every dimensionality the
    paths switch on."""
    c, t, _ = run_gpu(np.full((1, n), 0.5, dtype=np.float32), 0.5, indexed_dims=6)
    assert list(c) == [1] and list(t) == [0]
    c, t, st = run_gpu(np.full((8, n), 2.0, dtype=np.float32), 0.5, indexed_dims=6, stamp=True)
    assert list(c) == [8] * 8 and st["total_pairs"] == 64
    # lattice points (distinct ones at least 1 apart), 40 cells per indexed dim
    rng = np.random.default_rng(40 + n)
    base = rng.integers(0, 20, size=(300, n)).astype(np.float32)
    pts = np.concatenate([base, base, base[:50]])
    assert_same(oracle, pts, 0.5, indexed_dims=6)


@pytest.mark.parametrize("n", [16, 126])
def test_screen_dimension_bounds(oracle, n):
    """The smallest and the largest dimensionality the tensor-core screen
    takes (n + 2 columns, the folded norm, within one 128-wide tile)."""
    pts = tile_points(n, 6000, 3.0, 300 + n)
    st = assert_same(oracle, pts, 3.0, indexed_dims=6, stamp=(n == 16))
    assert st["join_path"] == 3


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("stamp", [False, True])
def test_warp_path_sparse_cells(oracle, dtype, stamp):
    """Mostly one point per cell in 6 indexed dims: a warp's 32 candidates
    come from up to 32 different neighbour ranges (the candidate-slot search
    across ranges), mixed with a few dense cells of many ranges' worth."""
    rng = np.random.default_rng(21)
    sparse = rng.uniform(0, 5, size=(15000, 7))  # about one point per cell, ~460 non-empty neighbours
    dense = rng.uniform(0, 1.5, size=(3000, 7)) + 2.0
    pts = np.concatenate([sparse, dense]).astype(dtype)[rng.permutation(18000)]
    st = assert_same(oracle, pts, 1.0, indexed_dims=6, stamp=stamp)
    assert st["join_path"] == 0  # GSJ_PATH_WARP
    # lists come out of the pair sort ascending
    c, t, _ = run_gpu(pts, 1.0, indexed_dims=6, stamp=stamp)
    starts = np.concatenate([[0], np.cumsum(c.astype(np.int64))])
    assert all(np.all(np.diff(t[starts[i]:starts[i + 1]].astype(np.int64)) > 0) for i in range(0, c.size, 61))


def test_tile_join_deterministic():
    pts = tile_points(18, 20000, 3.0, 7)
    c1, t1, s1 = run_gpu(pts, 3.0, indexed_dims=6, stamp=True)
    c2, t2, _ = run_gpu(pts, 3.0, indexed_dims=6, stamp=True)
    c3, t3, s3 = run_gpu(pts, 3.0, indexed_dims=6, stamp=True, plain=True)
    assert s1["join_path"] == 3 and s3["join_path"] == 2
    assert np.array_equal(c1, c3) and np.array_equal(t1, t3)
    assert np.array_equal(c1, c2) and np.array_equal(t1, t2)
    # lists come out of the pair sort ascending
    starts = np.concatenate([[0], np.cumsum(c1.astype(np.int64))])
    assert all(np.all(np.diff(t1[starts[i]:starts[i + 1]].astype(np.int64)) > 0) for i in range(0, c1.size, 97))


@pytest.mark.parametrize("stamp", [False, True])
def test_dense_cell_many_chunks(oracle, stamp):
    # 3000 points in few cells: query cells span many 32-query chunks
    rng = np.random.default_rng(5)
    pts = rng.uniform(0, 2.0, size=(3000, 2)).astype(np.float32)
    assert_same(oracle, pts, 1.0, indexed_dims=2, stamp=stamp)


def test_duplicates_and_eps_zero(oracle):
    rng = np.random.default_rng(6)
    base = rng.uniform(0, 50, size=(500, 3)).astype(np.float32)
    pts = np.concatenate([base, base, base[:100]])
    assert_same(oracle, pts, 1e-3, indexed_dims=3)
    assert_same(oracle, pts, 2e-3, indexed_dims=3, stamp=True)


def test_single_point_and_tiny():
    c, t, st = run_gpu(np.array([[1.0, 2.0]], dtype=np.float32), 0.5, indexed_dims=2)
    assert list(c) == [1] and list(t) == [0]
    c, t, st = run_gpu(np.zeros((0, 2), dtype=np.float32), 0.5, indexed_dims=2)
    assert c.size == 0 and t.size == 0


def test_negative_and_offset_coordinates(oracle):
    rng = np.random.default_rng(8)
    pts = (rng.uniform(-500, -400, size=(20000, 2)) + np.float32(1.0e5)).astype(np.float32)
    assert_same(oracle, pts, 0.8, indexed_dims=2, stamp=True)
    pts2 = rng.uniform(-50, 50, size=(20000, 3)).astype(np.float32)
    assert_same(oracle, pts2, 2.0, indexed_dims=2)


def test_collinear_k1(oracle):
    x = np.sort(np.random.default_rng(9).uniform(0, 1000, 30000)).astype(np.float32)
    pts = np.stack([x, np.zeros_like(x)], 1)
    assert_same(oracle, pts, 0.05, indexed_dims=1, stamp=True)


@pytest.mark.parametrize("case", ["rows_2d_stamp", "warp_3d_f64"])
def test_sort_lists_flag(case):
    """GSJ_FLAG_SORT_LISTS: the same lists, each ascending."""
    if case == "rows_2d_stamp":
        pts = synth.generate("c1_uniform2d")
        kw = dict(indexed_dims=2, stamp=True)
        eps = 1.0
    else:
        pts = np.random.default_rng(12).uniform(0, 40, size=(30000, 3))
        kw = dict(indexed_dims=3)
        eps = 1.5
    c0, t0, s0 = run_gpu(pts, eps, **kw)
    c1, t1, s1 = run_gpu(pts, eps, sort_lists=True, **kw)
    assert s1["join_path"] == s0["join_path"] and s0["join_path"] in (0, 1)
    assert np.array_equal(c0, c1)
    assert np.array_equal(t1, canon(c0, t0))


@pytest.mark.parametrize("case", [(3, np.float32, 20000, 1.5), (5, np.float64, 6000, 2.0), (90, np.float32, 3000, 20.0)])
def test_bruteforce_matches_oracle_and_join(oracle, case):
    """gsj_bruteforce_count (the reference's GPU algorithm 1) gives the oracle's
    brute-force counts exactly, and the grid join's counts on these inputs."""
    n, dt, N, eps = case
    rng = np.random.default_rng(40 + n)
    pts = (rng.uniform(0, 10, size=(N, n)) * rng.uniform(0.5, 2.0, n)).astype(dt)
    with SelfJoin(0) as sj:
        bc, bt = sj.bruteforce(pts, eps)
    oc, ot = oracle.bruteforce_counts(pts, eps, oracle_cfg(oracle, min(6, n)))
    assert bt == ot and np.array_equal(bc, oc)
    gc, _, st = run_gpu(pts, eps, indexed_dims=min(6, n))
    assert np.array_equal(gc, bc) and st["total_pairs"] == bt


def test_deterministic_without_stamp():
    pts = synth.generate("c1_uniform2d")
    c1, t1, _ = run_gpu(pts, 1.0, indexed_dims=2)
    c2, t2, _ = run_gpu(pts, 1.0, indexed_dims=2)
    assert np.array_equal(c1, c2) and np.array_equal(t1, t2)


def test_large_properties():
    """At 4M points of the 2-D mixture workload (too large for the oracle in a
    test): lists are symmetric, contain the point itself, and the unicomp
    traversal yields the same sets as the full traversal."""
    w = synth.WORKLOADS["c2_gmm2d"]
    pts = synth.generate("c2_gmm2d", 4_000_000)
    eps = w.eps if w.eps > 0 else 0.5
    c0, t0, s0 = run_gpu(pts, eps, indexed_dims=2, stamp=False)
    c1, t1, s1 = run_gpu(pts, eps, indexed_dims=2, stamp=True)
    assert np.array_equal(c0, c1)
    assert np.array_equal(canon(c0, t0), canon(c1, t1))
    seg = np.repeat(np.arange(c0.size, dtype=np.int64), c0.astype(np.int64))
    q, c = seg, t0.astype(np.int64)
    assert np.count_nonzero(q == c) == c0.size  # self pairs
    fwd = np.sort(q * c0.size + c)
    rev = np.sort(c * c0.size + q)
    assert np.array_equal(fwd, rev)  # (q,c) present iff (c,q) present
    # the count pass may use either traversal on low-dimensional grids
    assert s1["candidates"] <= s0["candidates"]


@pytest.mark.parametrize("dims,k", [(2, 2), (5, 5)])
def test_extent_rounding_is_rejected(dims, k):
    """eps below the float resolution of the data: max + eps rounds to max, so
    the largest coordinate's cell index equals the grid's extent (the
    reference would index past its grid).  The join fails with a status, on
    the dense (2-D: slot-prefix table) and the sparse (5-D, 2^30 cells: hash
    table) grids."""
    from gpu_self_join_b200._native import GsjError

    rng = np.random.default_rng(5)
    pts = (1e8 - 8.0 * rng.integers(0, 9, size=(2000, dims))).astype(np.float32)
    with pytest.raises(GsjError, match="extent"):
        run_gpu(pts, 1.0, indexed_dims=k)
    # a representable eps on the same data joins normally
    c, t, st = run_gpu(pts, 16.0, indexed_dims=k)
    assert st["total_pairs"] == t.size > 0
