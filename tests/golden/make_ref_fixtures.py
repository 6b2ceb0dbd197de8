"""Pins the oracle to the reference's own algorithm 3 and writes the fixtures
of tests/golden/ref_pins.json.

Runs on a machine with a CUDA GPU and the reference binaries built from the
reference's sources by oracle/build_ref.sh (oracle/_ref/<config>/main, built
with PRINTNEIGHBORTABLE=1, so each run writes its sorted per-point lists to
DSSJ_out.txt, main.cu:544-565).  For every configuration it

  1. generates a seeded input (pin_points) with many pairs placed at distance
     ~eps, so that different floating-point evaluation orders disagree on
     some of them,
  2. checks ON THE CPU, with the oracle's restatement of the reference's
     batch estimator (GPU.cu:57-268), that no batch of the reference run can
     exceed its result buffer - the reference writes results without a bounds
     check (kernel.cu:367-375) - and skips the configuration otherwise,
  3. runs `main <file> <eps> <dim> 3`, parses DSSJ_out.txt,
  4. compares the per-point lists with the oracle under each candidate
     arithmetic model and records which model reproduces the reference.

    python tests/golden/make_ref_fixtures.py [--out tests/golden/ref_pins.json]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# name -> (n, k, dtype, reorder, ilp, shortcircuit, queryreorder, N, eps)
# must match the builds of oracle/build_ref.sh
PIN_CONFIGS = {
    "d2_plain": (2, 2, "float32", False, 0, False, False, 40000, 1.0),
    "d2_plain_f64": (2, 2, "float64", False, 0, False, False, 36000, 1.0),
    "d6_plain": (6, 6, "float32", False, 0, False, False, 40000, 2.0),
    "d18_k6_ilp8_sc": (18, 6, "float32", True, 8, True, True, 30000, 3.0),
    "d18_k6_ilp8": (18, 6, "float32", True, 8, False, True, 30000, 3.0),
    "d18_k6_ilp4_sc": (18, 6, "float32", True, 4, True, False, 30000, 3.0),
    "d90_k6_ilp8_sc": (90, 6, "float32", True, 8, True, True, 8000, 8.0),
    "d5_k3_f64_ilp2_sc": (5, 3, "float64", True, 2, True, True, 30000, 2.0),
    "d5_k3_f64_plain": (5, 3, "float64", True, 0, False, False, 60000, 1.3),
    "d18_k6_f64_ilp8": (18, 6, "float64", True, 8, False, True, 30000, 3.0),
    "d18_k6_f64_ilp8_sc": (18, 6, "float64", True, 8, True, True, 30000, 3.0),
    "d5_k3_f32_ilp8": (5, 3, "float32", True, 8, False, False, 30000, 2.0),
    "d5_k3_f64_ilp8": (5, 3, "float64", True, 8, False, False, 60000, 1.3),
    "d3_k3_f64_ilp2": (3, 3, "float64", False, 2, False, False, 30000, 2.0),
    "d5_k3_f32_ilp2_sc": (5, 3, "float32", True, 2, True, True, 30000, 2.0),
    "d2_sort": (2, 2, "float32", False, 0, False, False, 40000, 1.0),
    "d3_k2_sort": (3, 2, "float32", False, 0, False, False, 40000, 1.5),
    "d5_k3_f64_sort": (5, 3, "float64", True, 2, True, False, 30000, 2.0),
    "d3_k2_sort_gap": (3, 2, "float32", False, 0, False, False, 40000, 0.5),
}
# configurations built with SORT=1 (params.h:46; oracle/build_ref.sh)
SORTED = {"d2_sort", "d3_k2_sort", "d5_k3_f64_sort", "d3_k2_sort_gap"}
# pins that run another pin's reference build
BUILD_OF = {"d3_k2_sort_gap": "d3_k2_sort"}


def gap_points(name: str) -> np.ndarray:
    """Pairs of points equal in the indexed dimensions and exactly eps apart
    in the sort dimension (values are multiples of eps, exact in binary): the
    pruned window's strict `< eps` (kernel.cu:461) drops the partner above
    the query, while the full scan reports both directions."""
    n, k, dt, _, _, _, _, N, eps = PIN_CONFIGS[name]
    seed = int.from_bytes(hashlib.sha256(name.encode()).digest()[:4], "little")
    rng = np.random.default_rng(seed)
    m = N // 2
    base = rng.uniform(0, 40 * eps, size=(m, n))
    base[:, k] = rng.integers(0, 80, m) * eps
    partner = base.copy()
    partner[:, k] += eps
    pts = np.concatenate([base, partner]).astype(dt)
    return pts[rng.permutation(N)]


def pin_points(name: str) -> np.ndarray:
    """Seeded input of a pin configuration: clustered points plus partners
    placed at distance eps (computed in float64, then rounded)."""
    if name.endswith("_gap"):
        return gap_points(name)
    n, k, dt, _, _, _, _, N, eps = PIN_CONFIGS[name]
    seed = int.from_bytes(hashlib.sha256(name.encode()).digest()[:4], "little")
    rng = np.random.default_rng(seed)
    nb = N // 2
    scales = rng.uniform(0.5, 4.0, size=n)
    centres = rng.uniform(0, 30, size=(6, n))
    base = centres[rng.integers(0, 6, nb)] + rng.standard_normal((nb, n)) * scales * eps
    d = rng.standard_normal((N - nb, n))
    d *= eps / np.linalg.norm(d, axis=1, keepdims=True)
    partner = base[rng.integers(0, nb, N - nb)] + d
    pts = np.concatenate([base, partner]).astype(dt)
    return pts[rng.permutation(N)]


def lists_digest(counts, nbrs) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(counts, dtype=np.uint32).tobytes())
    h.update(np.ascontiguousarray(nbrs, dtype=np.uint32).tobytes())
    return h.hexdigest()


def parse_dssj(path: str, N: int):
    counts = np.zeros(N, dtype=np.uint32)
    vals = []
    with open(path) as f:
        first = f.readline()
        assert first.startswith("#")
        for i in range(N):
            ln = f.readline()
            parts = [p for p in ln.strip().split(",") if p.strip()]
            counts[i] = len(parts)
            vals.append(np.array(parts, dtype=np.int64).astype(np.uint32) if parts else np.zeros(0, np.uint32))
    return counts, (np.concatenate(vals) if vals else np.zeros(0, np.uint32))


def oracle_variants(O, name, pts):
    """Every contraction policy of the device model (see DevNode in
    oracle/gsj_oracle.cpp) plus the host's unfused arithmetic."""
    n, k, dt, reorder, ilp, sc, qr, N, eps = PIN_CONFIGS[name]
    srt = name in SORTED
    out = {}
    for fz in (False, True):
        for fl in (False, True):
            for xl in (False, True):
                out[f"fold{int(fz)}_left{int(fl)}_xleft{int(xl)}"] = O.OracleConfig(
                    k=k, reorder=reorder, ilp=ilp, shortcircuit=sc, fold_zero=fz, fuse_left=fl, cross_left=xl,
                    sort=srt)
    out["pinned"] = O.OracleConfig(k=k, reorder=reorder, ilp=ilp, shortcircuit=sc, sort=srt)
    if srt:
        out["unsorted_traversal"] = O.OracleConfig(k=k, reorder=reorder, ilp=ilp, shortcircuit=sc)
    out["host_unfused"] = O.OracleConfig(k=k, reorder=reorder, ilp=0, model=O.MODEL_HOST)
    return out


def safe_to_run(O, name, pts) -> tuple[bool, str]:
    n, k, dt, reorder, ilp, sc, qr, N, eps = PIN_CONFIGS[name]
    p32 = pts.astype(np.float32)
    if dt != "float32":
        # the plan is computed in float32 only; double runs are small and the
        # float32 plan is only used as a size sanity check
        pass
    ref_c, ref_tot, _ = O.join_counts(pts, eps, O.OracleConfig(k=k, reorder=reorder, ilp=ilp, shortcircuit=sc))
    smp_c, _, _ = O.join_counts(pts, eps, O.OracleConfig(k=k, reorder=reorder, ilp=0))
    est, nb, buf, mx = O.ref_batch_plan(p32, eps, O.OracleConfig(k=k, reorder=reorder), ref_c, smp_c, qr, 0.05)
    ok = est > 0 and buf > 0 and mx <= 0.9 * buf
    return ok, f"estimate={est} batches={nb} buffer={buf} largest_batch={mx} total={ref_tot}"


def main():
    from oracle import pyoracle as O

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_pins.json"))
    ap.add_argument("--only", default="")
    ap.add_argument("--test-dat", default=os.path.join(HERE, "test_dat_f32.npy"))
    a = ap.parse_args()
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    results = {}
    jobs = [x for x in PIN_CONFIGS if not a.only or x in a.only.split(",")]
    if not a.only or "test_dat" in a.only:
        jobs = ["test_dat"] + jobs
    for name in jobs:
        if name == "test_dat":
            cfgname, pts = "d2_plain", np.load(a.test_dat)
            spec = (2, 2, "float32", False, 0, False, False, pts.shape[0], 1.0)
            PIN_CONFIGS["test_dat"] = spec
        else:
            cfgname, pts = BUILD_OF.get(name, name), pin_points(name)
            spec = PIN_CONFIGS[name]
        n, k, dt, reorder, ilp, sc, qr, N, eps = spec
        binary = os.path.join(ROOT, "oracle", "_ref", cfgname, "main")
        rec = {"config": cfgname, "N": int(N), "n": n, "k": k, "dtype": dt, "reorder": reorder, "ilp": ilp,
               "shortcircuit": sc, "query_reorder": qr, "eps": eps, "sort": name in SORTED}
        if not os.path.exists(binary):
            rec["status"] = "reference binary missing"
            results[name] = rec
            continue
        ok, why = safe_to_run(O, name, pts)
        rec["plan"] = why
        if not ok:
            rec["status"] = "skipped: reference result buffer could overflow"
            results[name] = rec
            continue
        with tempfile.TemporaryDirectory() as td:
            f = os.path.join(td, "data.txt")
            fmt = "%.9g" if dt == "float32" else "%.17g"
            np.savetxt(f, pts, fmt=fmt, delimiter=",")
            r = subprocess.run([binary, f, repr(float(eps)), str(n), "3"], cwd=td, capture_output=True, text=True,
                               timeout=600)
            rec["returncode"] = r.returncode
            dssj = os.path.join(td, "DSSJ_out.txt")
            if r.returncode != 0 or not os.path.exists(dssj):
                rec["status"] = "reference run failed"
                rec["stderr"] = r.stderr[-1500:]
                rec["stdout"] = r.stdout[-1500:]
                results[name] = rec
                continue
            with open(os.path.join(td, "gpu_stats.txt")) as g:
                rec["gpu_stats_line"] = g.read().strip()
            rc, rn = parse_dssj(dssj, N)
        rec["reference_total"] = int(rc.sum(dtype=np.uint64))
        rec["reference_lists_sha256"] = lists_digest(rc, rn)
        rec["models"] = {}
        for vname, cfg in oracle_variants(O, name, pts).items():
            oc, _, on = O.join_lists(pts, eps, cfg)
            same = bool(np.array_equal(oc, rc) and np.array_equal(on, rn))
            rec["models"][vname] = {"identical": same, "total": int(oc.sum(dtype=np.uint64)),
                                    "points_differing": int(np.count_nonzero(oc != rc))}
        rec["status"] = "ok"
        results[name] = rec
        print(name, json.dumps(rec["models"]), flush=True)
    with open(a.out, "w") as f:
        json.dump(results, f, indent=1, sort_keys=True)
    print(json.dumps(results, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()


def merge_into_golden(*result_files: str) -> None:
    """Folds reference-run results into tests/golden/ref_pins.json (the
    committed fixture: input spec, the reference's total and the digest of its
    sorted per-point lists)."""
    path = os.path.join(HERE, "ref_pins.json")
    gold = json.load(open(path)) if os.path.exists(path) else {}
    keep = ("config", "N", "n", "k", "dtype", "reorder", "ilp", "shortcircuit", "query_reorder", "eps", "sort",
            "reference_total", "reference_lists_sha256")
    for f in result_files:
        for name, rec in json.load(open(f)).items():
            if rec.get("status") == "ok":
                gold[name] = {k: rec.get(k, False) for k in keep}
                gold[name]["gpu_stats_line"] = ", ".join(rec["gpu_stats_line"].split(", ")[2:])
    with open(path, "w") as fh:
        json.dump(gold, fh, indent=1, sort_keys=True)
