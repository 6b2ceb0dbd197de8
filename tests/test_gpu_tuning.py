"""Launch-shape autotuning: the tuner picks a shape per (path, dim, density),
later joins of the same key launch with it, and no shape changes a result."""
import numpy as np
import pytest

from gpu_self_join_b200 import JoinConfig, SelfJoin, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["rows_2d", "warp_6d", "tile_12d", "screen_18d"])
def test_autotune_keeps_results(case):
    rng = np.random.default_rng(31)
    if case == "rows_2d":
        pts, kw, eps, path = synth.generate("c2_gmm2d", 400_000), dict(indexed_dims=2, stamp=True), 0.5, 1
    elif case == "warp_6d":
        pts, kw, eps, path = synth.generate("c3_gmm6d", 200_000), dict(indexed_dims=6, stamp=True), 2.1, 0
    else:
        n = 12 if case == "tile_12d" else 18
        base = rng.uniform(0, 10, size=(4, n))[rng.integers(0, 4, 20000)]
        pts = (base + rng.standard_normal((20000, n)) * 0.8).astype(np.float32)
        kw, eps, path = dict(indexed_dims=6), 3.0, (2 if n == 12 else 3)
    with SelfJoin(0) as sj:
        st0 = sj.run(pts, eps, JoinConfig(**kw))
        c0, t0 = sj.counts(), sj.table()
        assert st0["join_path"] == path and st0["tuned"] == 0
        best = sj.autotune(pts, eps, JoinConfig(**kw), repeats=1)
        assert sj.tuning(path, pts.shape[1], int(st0["density_log2"])) == best
        st1 = sj.run(pts, eps, JoinConfig(**kw))
        c1, t1 = sj.counts(), sj.table()
        assert st1["tuned"] == 1
        assert np.array_equal(c0, c1) and np.array_equal(t0, t1)
        # an explicit shape at the extremes of the ranges gives the same lists too
        extreme = {"threads": 64, "warps": 1, "ctas_per_sm": 1, "streams": 1}
        sj.tuning(path, pts.shape[1], int(st0["density_log2"]), extreme)
        sj.run(pts, eps, JoinConfig(**kw))
        assert np.array_equal(c0, sj.counts()) and np.array_equal(t0, sj.table())


def test_tuning_rejects_bad_shapes():
    from gpu_self_join_b200._native import GsjError

    with SelfJoin(0) as sj:
        with pytest.raises(GsjError):
            sj.tuning(1, 2, 0, {"threads": 100})
        with pytest.raises(GsjError):
            sj.tuning(0, 6, 0, {"warps": 9})
        assert sj.tuning(1, 2, 5) is None
