"""Host-side logic of bench.py that needs no GPU: the roofline object per
join path (kernel label, bound, algorithmic bytes or FLOPs, fraction of the
peak) and the traffic figure read back from the committed ncu summaries."""
import math

import pytest

import bench
from gpu_self_join_b200 import synth


def _stats(path, count_ms, fill_ms, candidates=0):
    return [{"dev_ms_fill": fill_ms, "dev_ms_count": count_ms, "dev_ms_index": 1.0, "join_path": path,
             "candidates": candidates}]


def test_rows_path_fill_dominant():
    w = synth.WORKLOADS["c2_gmm2d"]
    N, n, R, C = w.N, w.n, 642_337_374, 1_802_646_654
    roof = bench._roofline(_stats(1, 1.4, 5.2, C), N, n, R, w)
    assert roof["kernel"] == "join_fill" and roof["bound"] == "hbm" and roof["unit"] == "GB/s"
    want = 4.0 * R + 24.0 * N + C / 8.0  # table, per-query metadata, hit masks
    assert roof["algorithmic_bytes"] == want
    assert math.isclose(roof["achieved"], want / 5.2e-3 / 1e9)
    assert math.isclose(roof["frac"], roof["achieved"] / roof["peak"])
    # the whole join against the path's algorithmic bytes 4Nn + 4N + 4R
    b_alg = 4.0 * N * n + 4.0 * N + 4.0 * R
    assert roof["join"]["algorithmic_bytes"] == b_alg
    assert math.isclose(roof["join"]["ms"], 1.0 + 1.4 + 5.2)


def test_rows_path_count_dominant():
    w = synth.WORKLOADS["c2_gmm2d"]
    C = 1_000_000
    roof = bench._roofline(_stats(1, 6.0, 5.0, C), w.N, w.n, 10, w)
    assert roof["kernel"] == "join_count"
    assert roof["algorithmic_bytes"] == 4.0 * w.N * w.n + 4.0 * w.N + 8.0 * w.N + C / 8.0


@pytest.mark.parametrize("path", [0, 2])
def test_emit_paths(path):
    w = synth.WORKLOADS["c3_gmm6d"]
    R = 317_398_440
    roof = bench._roofline(_stats(path, 38.4, 19.9), w.N, w.n, R, w)
    assert roof["kernel"] == "join_emit" and roof["bound"] == "hbm"
    assert roof["algorithmic_bytes"] == 4.0 * w.N * w.n + 4.0 * w.N + 8.0 * R
    place = bench._roofline(_stats(path, 10.0, 19.9), w.N, w.n, R, w)
    assert place["kernel"] == "pair_place"
    assert place["algorithmic_bytes"] == 12.0 * R + 8.0 * w.N


def test_screen_path_is_a_tensor_roofline():
    w = synth.WORKLOADS["c4_derived18d"]
    cand = 765_422_617_530
    roof = bench._roofline(_stats(3, 403.6, 34.6, cand), w.N, w.n, 540_628_642, w)
    assert roof["kernel"] == "tile_screen" and roof["bound"] == "tensor" and roof["unit"] == "TFLOP/s"
    assert roof["algorithmic_flops"] == 2.0 * (w.n + 2) * cand
    assert math.isclose(roof["achieved"], roof["algorithmic_flops"] / 0.4036 / 1e12)
    assert 0.0 < roof["frac"] < 1.0
    assert roof["peak_source"] in ("measured", "fallback (sustained)")


def test_traffic_lookup_missing_profile():
    assert bench._traffic_from_profile("no_such_kernel", "c2_gmm2d") is None


def test_traffic_of_the_committed_fill_profile():
    """The fill capture's DRAM traffic, scaled to the 20M-point launch, lies between the
    algorithmic bytes of that launch and a few times them (a figure left unscaled from the
    8M-point capture, or one of another kernel, would fall outside)."""
    w = synth.WORKLOADS["c2_gmm2d"]
    R, C = 642_337_374, 1_802_646_654
    traffic = bench._traffic_from_profile("join_fill", "c2_gmm2d")
    assert traffic is not None
    alg = 4.0 * R + 24.0 * w.N + C / 8.0
    assert alg < traffic < 6.0 * alg
