"""Parity against the reference's own algorithm 3, built from its sources and
run on a B200 (tests/golden/make_ref_fixtures.py).  Each fixture holds the
seeded input spec, the reference's total and the SHA-256 of its sorted
per-point neighbour lists (DSSJ_out.txt, main.cu:544-565).

* CPU: the oracle restatement reproduces every fixture bit-exactly.
* GPU: the CUDA path (through the C ABI) reproduces every fixture bit-exactly.
"""
import json
import os

import numpy as np
import pytest

from tests.golden.make_ref_fixtures import PIN_CONFIGS, lists_digest, pin_points

GOLD = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLD, "ref_pins.json")) as _f:
    PINS = json.load(_f)


def _input(name):
    if name == "test_dat":
        return np.load(os.path.join(GOLD, "test_dat_f32.npy"))
    spec = PINS[name]
    assert PIN_CONFIGS[name][:7] == (spec["n"], spec["k"], spec["dtype"], spec["reorder"], spec["ilp"],
                                     spec["shortcircuit"], spec["query_reorder"])
    assert PIN_CONFIGS[name][7:] == (spec["N"], spec["eps"]), "pin input spec changed since the reference run"
    return pin_points(name)


def test_fixture_covers_both_precisions_and_models():
    dts = {v["dtype"] for v in PINS.values()}
    assert dts == {"float32", "float64"}
    assert {v["ilp"] for v in PINS.values()} >= {0, 2, 4, 8}
    assert {v["shortcircuit"] for v in PINS.values()} == {False, True}
    assert PINS["test_dat"]["reference_total"] == 27982028
    # SORT=1 builds (params.h:46), both sort-dimension cases, and one input on
    # which the pruned window drops pairs that the full traversal reports
    srt = {k: v for k, v in PINS.items() if v.get("sort")}
    assert {v["n"] == v["k"] for v in srt.values()} == {True, False}
    assert "d3_k2_sort_gap" in srt


def test_sort_gap_pin_differs_from_full_traversal(oracle):
    spec = PINS["d3_k2_sort_gap"]
    pts = _input("d3_k2_sort_gap")
    _, full, _ = oracle.join_counts(pts, spec["eps"], oracle.OracleConfig(k=spec["k"]))
    assert spec["reference_total"] < full


@pytest.mark.parametrize("name", sorted(PINS))
def test_oracle_reproduces_reference(oracle, name):
    spec = PINS[name]
    pts = _input(name)
    cfg = oracle.OracleConfig(k=spec["k"], reorder=spec["reorder"], ilp=spec["ilp"],
                              shortcircuit=spec["shortcircuit"], sort=spec.get("sort", False))
    counts, _, nbrs = oracle.join_lists(pts, spec["eps"], cfg)
    assert int(counts.sum(dtype=np.uint64)) == spec["reference_total"]
    assert lists_digest(counts, nbrs) == spec["reference_lists_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("stamp", [False, True])
@pytest.mark.parametrize("name", sorted(PINS))
def test_gpu_reproduces_reference(name, stamp):
    from gpu_self_join_b200 import JoinConfig, SelfJoin

    spec = PINS[name]
    pts = _input(name)
    cfg = JoinConfig(indexed_dims=spec["k"], reorder=spec["reorder"], ilp=spec["ilp"],
                     shortcircuit=spec["shortcircuit"], query_reorder=spec["query_reorder"], stamp=stamp,
                     sort=spec.get("sort", False))
    with SelfJoin(0) as sj:
        st = sj.run(pts, spec["eps"], cfg)
        counts, table = sj.counts(), sj.table()
    seg = np.repeat(np.arange(counts.size), counts.astype(np.int64))
    canon = table[np.lexsort((table, seg))]
    assert st["total_pairs"] == spec["reference_total"]
    assert lists_digest(counts, canon) == spec["reference_lists_sha256"]
