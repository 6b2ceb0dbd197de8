"""Results delivered to host memory in batches (gsj_join_host).

The dense low-dimensional path fills the table in batches of point ids whose
lists fit one device segment of GPUBUFFERSIZE entries and copies each batch
to the host while the next is computed.  Whatever the batch size, the number
of segments in flight and the kind of host memory, the host result must equal
the device-resident result of gsj_join exactly (same lists, same order).
"""
import numpy as np
import pytest

from gpu_self_join_b200 import JoinConfig, SelfJoin, synth

pytestmark = pytest.mark.gpu


def _pinned(n):
    import torch

    return torch.empty(max(n, 1), dtype=torch.int32).pin_memory().numpy().view(np.uint32)[:n]


@pytest.fixture(scope="module")
def c2_small():
    pts = synth.generate("c2_gmm2d", 1_000_000)
    with SelfJoin(0) as sj:
        st = sj.run(pts, 0.5, JoinConfig(indexed_dims=2, stamp=True))
        return pts, st, sj.counts(), sj.table()


@pytest.mark.parametrize("buffer_pairs,streams,pinned", [
    (0, 0, False),             # defaults: 100M-entry segments, 3 in flight, at least 3 batches
    (1_000_000, 3, True),      # tens of batches, pinned destinations (direct DMA)
    (700_001, 2, False),       # pageable destinations (pinned staging), odd segment size
    (2_000_000, 1, True),      # one segment: every batch waits for the previous copy
])
def test_host_batches_equal_device_result(c2_small, buffer_pairs, streams, pinned):
    pts, st0, c0, t0 = c2_small
    R = int(st0["total_pairs"])
    counts = _pinned(pts.shape[0]) if pinned else np.empty(pts.shape[0], dtype=np.uint32)
    table = _pinned(R) if pinned else np.empty(R, dtype=np.uint32)
    cfg = JoinConfig(indexed_dims=2, stamp=True, buffer_pairs=buffer_pairs, streams=streams)
    with SelfJoin(0) as sj:
        st, c1, t1 = sj.run_host(pts, 0.5, cfg, counts=counts, table=table)
    assert st["join_path"] == 1 and st["total_pairs"] == R
    if buffer_pairs:
        assert st["batches"] >= R // buffer_pairs
    else:
        assert st["batches"] >= 3
    assert np.array_equal(c1, c0)
    assert np.array_equal(t1, t0)


def test_host_result_too_small_table_reports_size(c2_small):
    pts, st0, c0, t0 = c2_small
    with SelfJoin(0) as sj:
        # run_host retries with the reported size
        st, c1, t1 = sj.run_host(pts, 0.5, JoinConfig(indexed_dims=2), table=np.empty(10, dtype=np.uint32))
        assert np.array_equal(c1, c0) and np.array_equal(t1, t0)
        # the device keeps no table after a batched host join
        with pytest.raises(Exception):
            sj.table()


@pytest.mark.parametrize("case", ["warp_6d", "tile_18d"])
def test_host_result_other_paths(case):
    rng = np.random.default_rng(9)
    if case == "warp_6d":
        pts = rng.uniform(0, 6, size=(20000, 6)).astype(np.float32)
        kw, eps = dict(indexed_dims=6, stamp=True), 1.0
    else:
        base = rng.uniform(0, 10, size=(4, 18))[rng.integers(0, 4, 10000)]
        pts = (base + rng.standard_normal((10000, 18)) * 0.8).astype(np.float32)
        kw, eps = dict(indexed_dims=6), 3.0
    with SelfJoin(0) as sj:
        sj.run(pts, eps, JoinConfig(**kw))
        c0, t0 = sj.counts(), sj.table()
        st, c1, t1 = sj.run_host(pts, eps, JoinConfig(buffer_pairs=100_000, **kw))
    assert np.array_equal(c1, c0) and np.array_equal(t1, t0)
