"""Times the reference's own GPU algorithm 3 on the benchmarked synthetic
workloads, on the box this runs on, with the reference's own timer
(main.cu:246-254: distanceTableNDGridBatches plus REORDER, index build
excluded), beside this library's time for the same join.

The reference binaries are built from the reference's sources by
oracle/build_ref.sh (timing builds t_d2, t_d6, t_d18, t_d90: the workloads'
params.h switches, no neighbour-table print; STAMP=0 since the reference's CLI
does not compile with STAMP=1 - same pair set).  Before a reference run, its
batch plan is restated on the CPU (oracle orc_ref_batch_plan, GPU.cu:57-268)
with this library's per-point counts (bit-identical to the reference's on every
pinned input) and the run is skipped unless the largest batch stays below 95 %
of the reference's unguarded result buffer.

    python tests/golden/time_ref_gpu.py [--only c1_uniform2d,...] [--out FILE]

Test infrastructure: needs a GPU; not part of the test suite.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

BUILD_OF = {"c1_uniform2d": "t_d2", "c2_gmm2d": "t_d2", "c3_gmm6d": "t_d6", "c4_derived18d": "t_d18",
            "c5_heavy90d": "t_d90"}


def write_text(path: str, pts: np.ndarray) -> None:
    import pandas as pd

    pd.DataFrame(pts).to_csv(path, header=False, index=False, float_format="%.9g")


def main() -> None:
    from gpu_self_join_b200 import JoinConfig, SelfJoin, synth
    from oracle import pyoracle as O

    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="")
    ap.add_argument("--out", default=os.path.join(HERE, "ref_gpu_times.json"))
    a = ap.parse_args()
    names = [x for x in BUILD_OF if not a.only or x in a.only.split(",")]
    res = {}
    for name in names:
        w = synth.WORKLOADS[name]
        pts = synth.generate(name)
        N, n = pts.shape
        rec = {"workload": name, "N": int(N), "n": n, "eps": w.eps, "build": BUILD_OF[name]}
        binary = os.path.join(ROOT, "oracle", "_ref", BUILD_OF[name], "main")
        cfg = JoinConfig(indexed_dims=w.k, reorder=w.reorder, shortcircuit=w.shortcircuit, ilp=w.ilp, stamp=w.stamp,
                         query_reorder=w.query_reorder)
        with SelfJoin(0) as sj:
            sj.run(pts, w.eps, cfg)  # warm-up
            st = sj.run(pts, w.eps, cfg)
            counts = sj.counts()
            t0 = time.perf_counter()
            sth, c_h, _ = sj.run_host(pts, w.eps, cfg)
            e2e_s = time.perf_counter() - t0
        rec["ours"] = {"total_pairs": int(st["total_pairs"]), "join_path": int(st["join_path"]),
                       "device_join_ms": float(st["dev_ms_index"] + st["dev_ms_count"] + st["dev_ms_fill"]),
                       "host_result_wall_ms": e2e_s * 1e3}
        if not os.path.exists(binary):
            rec["status"] = "reference binary missing"
            res[name] = rec
            continue
        ocfg = O.OracleConfig(k=w.k, reorder=w.reorder)
        est, nb, buf, mx = O.ref_batch_plan(pts.astype(np.float32), w.eps, ocfg, counts, counts,
                                            w.query_reorder, 0.05)
        rec["plan"] = {"estimate": est, "batches": nb, "buffer": buf, "largest_batch": mx}
        if not (est > 0 and buf > 0 and mx <= 0.95 * buf):
            rec["status"] = "skipped: the reference's result buffer could overflow"
            res[name] = rec
            continue
        with tempfile.TemporaryDirectory() as td:
            f = os.path.join(td, "data.txt")
            write_text(f, pts)
            t0 = time.perf_counter()
            r = subprocess.run([binary, f, repr(float(w.eps)), str(n), "3"], cwd=td, capture_output=True,
                               text=True, timeout=1800)
            rec["reference_wall_s"] = time.perf_counter() - t0
            rec["returncode"] = r.returncode
            stats = os.path.join(td, "gpu_stats.txt")
            if r.returncode != 0 or not os.path.exists(stats):
                rec["status"] = "reference run failed"
                rec["stderr"] = r.stderr[-1000:]
                res[name] = rec
                continue
            line = open(stats).read().strip().splitlines()[-1]
            fields = [x.strip() for x in line.split(",")]
            rec["reference"] = {"timer_s": float(fields[0]), "total_pairs": int(fields[3]), "stats_line": line}
        rec["same_total"] = rec["reference"]["total_pairs"] == rec["ours"]["total_pairs"]
        rec["status"] = "ok"
        res[name] = rec
        print(name, json.dumps(rec), flush=True)
    with open(a.out, "w") as fh:
        json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()
