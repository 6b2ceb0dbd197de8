"""Host-side workload generation: the seeded request stream of the 90-D
workload's second phase, the heavy-tailed generator it draws points from, and
bench.py's eps calibration (sample mean neighbour count at eps = target)."""
import numpy as np
import torch

import bench
from gpu_self_join_b200 import synth


def test_request_stream_is_seeded_and_in_range():
    a = synth.request_stream(64)
    b = synth.request_stream(64)
    assert a == b
    assert [r.index for r in a] == list(range(64))
    assert all(10_000 <= r.N <= 500_000 for r in a)
    assert {r.n for r in a} <= {8, 16, 32, 90}
    assert all(10.0 <= r.target_mean <= 100.0 for r in a)
    # a longer stream starts with the shorter one
    assert synth.request_stream(128)[:64] == a


def test_gen_heavy_shapes_and_tails():
    for n in (8, 16, 32, 90):
        x = synth.gen_heavy(4000, n, seed=3)
        assert x.shape == (4000, n) and x.dtype == np.float32
        assert np.all(np.isfinite(x))
    # the Student-t part (dims past the first 12) has heavier tails than a Gaussian
    x = synth.gen_heavy(20000, 32, seed=4).astype(np.float64)
    t = x[:, 12:]
    kurt = np.mean(((t - t.mean(0)) / t.std(0)) ** 4, axis=0)
    assert np.median(kurt) > 4.0
    assert np.array_equal(synth.gen_heavy(100, 16, seed=5), synth.gen_heavy(100, 16, seed=5))


def test_calibrate_eps_hits_the_target_count():
    x = torch.from_numpy(synth.gen_heavy(6000, 8, seed=6))
    target = 25.0
    eps = bench._calibrate_eps(x, target, seed=11)
    g = torch.Generator(device=x.device)
    g.manual_seed(11)
    q = x[torch.randperm(x.shape[0], generator=g, device=x.device)[:256]].double()
    d2 = torch.cdist(q, x.double()).pow(2)
    k = int(round(256 * target))
    e2 = eps * eps
    assert int((d2 < e2 * (1 - 1e-9)).sum()) < k <= int((d2 <= e2 * (1 + 1e-9)).sum())
