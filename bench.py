#!/usr/bin/env python
"""Benchmark of the B200 epsilon-grid self-join (algorithm 3 drop-in).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workload (default): the 2-D low-dimensional large workload - 20M points, 90%
from 64 isotropic Gaussians + 10% uniform background in [0,1000)^2, eps set
for about 32 neighbours per point, STAMP=1 (synthetic, seeded; see
gpu_self_join_b200/synth.py).  A step is one complete self-join of the
workload: index build, count pass, offsets, fill pass (the full neighbour
table).

Metric: result pairs per second (R / step time), whole job over N GPUs.
  value  - inputs resident in HBM, results left in HBM (device-timed: CUDA
           events on the current stream around K back-to-back steps; the
           input, 160 MB, and the working set exceed the 126 MB L2).
  e2e    - the same metric through the public API with host buffers: H2D of
           the pinned input, the join, D2H of numNeighbors and neighborTable
           into pinned host memory, every step.
Multi-GPU: "replicas only" - every rank joins its own copy (no data-path
collective); value = pairs of all ranks / max-over-ranks time.

--impl reference times the reference's own CPU implementation of the path on
this host's cores, on a bounded query sample of the same workload (see
_reference_arm).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import time
import sys

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def _env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.path = None

    def _lines(self) -> int:
        try:
            with open(self.path) as f:
                return sum(1 for ln in f if ln.strip())
        except OSError:
            return 0

    def start(self):
        """Starts sampling every 50 ms and returns once the first sample is
        written, so that a short timed region is still covered."""
        import tempfile

        self.path = tempfile.mktemp(suffix=".csv")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t_end = time.time() + 3.0
        while time.time() < t_end and self.proc.poll() is None and self._lines() == 0:
            time.sleep(0.01)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        # one more sample taken at or after the end of the timed region
        n0, t_end = self._lines(), time.time() + 0.5
        while time.time() < t_end and self.proc.poll() is None and self._lines() <= n0:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        try:
            with open(self.path) as f:
                self.lines = [ln.strip() for ln in f]
            os.remove(self.path)
        except OSError:
            self.lines = []
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ helpers
def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _tensor_peak():
    """Dense BF16 tensor peak: the sustained (power-capped) figure, since the
    screen runs inside joins of hundreds of milliseconds, back to back."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        v = d.get("bf16_tflops_sustained", d.get("bf16_tflops"))
        if v is not None:
            return float(v), "measured"
    return 1400.0, "fallback (sustained)"


def _traffic_from_profile(kernel: str, workload: str):
    """DRAM bytes per launch recorded from an ncu capture in profiles/."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for ln in f:
            if ln.startswith("traffic_bytes_per_launch:"):
                try:
                    return float(ln.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


def _roofline(stats: list, N: int, n: int, R: int, w) -> dict:
    """Roofline object for the join's dominant stage.  The device clock
    brackets two stages per join: "count" (ROWS: the count pass; the other
    paths: the estimate + the pair-emitting pass) and "fill" (ROWS: the fill
    pass; the other paths: pair placement + list sort).  Algorithmic bytes per
    launch (C = candidate evaluations):
      join_fill   table 4R written, per-query list length, bit-mask offsets,
                  id and list offset 24N, hit masks C/8 read
      join_count  coordinates 4Nn, ids 4N, list lengths 8N (by slot and by id),
                  hit masks C/8 written
      join_emit   coordinates 4Nn + ids 4N + 8-byte pair keys 8R
      pair_place  keys 8R read + table 4R + offsets 8N written
    The screen is a tensor-core kernel: 2(n+2) FLOPs per screened pair (one
    dot product of the n centred coordinates and the two norm columns).
    `join` is the whole join against the algorithmic bytes of the path,
    4Nn + 4N + 4R (coordinates read once, numNeighbors and the table written)."""
    fill_ms = statistics.mean(s["dev_ms_fill"] for s in stats)
    count_ms = statistics.mean(s["dev_ms_count"] for s in stats)
    index_ms = statistics.mean(s["dev_ms_index"] for s in stats)
    C = float(stats[-1]["candidates"])
    path = int(stats[-1].get("join_path", 1))
    peak, peak_kind = _peaks()
    b_coords = 4.0 * N * n
    bound, unit, pk = "hbm", "GB/s", peak
    if path == 1:  # GSJ_PATH_ROWS
        work_fill = 4.0 * R + 24.0 * N + C / 8.0
        work_count = b_coords + 4.0 * N + 8.0 * N + C / 8.0
        names = ("join_fill", "join_count")
    else:
        work_fill = 8.0 * R + 4.0 * R + 8.0 * N
        work_count = b_coords + 4.0 * N + 8.0 * R
        names = ("pair_place", "join_emit")
    if fill_ms >= count_ms:
        kname, kms, kwork = names[0], fill_ms, work_fill
    else:
        kname, kms, kwork = names[1], count_ms, work_count
        if path == 3:  # GSJ_PATH_SCREEN
            kname, bound, unit = "tile_screen", "tensor", "TFLOP/s"
            kwork = 2.0 * (n + 2) * C
            pk, peak_kind = _tensor_peak()
    achieved = kwork / (kms / 1e3) / (1e12 if unit == "TFLOP/s" else 1e9)
    join_ms = index_ms + count_ms + fill_ms
    b_alg = b_coords + 4.0 * N + 4.0 * R
    roof = {"bound": bound, "kernel": kname, "achieved": achieved, "peak": pk, "unit": unit,
            "frac": achieved / pk, "peak_source": peak_kind,
            ("algorithmic_flops" if unit == "TFLOP/s" else "algorithmic_bytes"): kwork,
            "kernel_ms": kms, "traffic": _traffic_from_profile(kname, w.name),
            "stage_ms": {"index": index_ms, "count": count_ms, "fill": fill_ms},
            "join": {"ms": join_ms, "algorithmic_bytes": b_alg, "achieved_gbs": b_alg / (join_ms / 1e3) / 1e9,
                     "frac": b_alg / (join_ms / 1e3) / 1e9 / peak}}
    return roof


def _link_peaks(nbytes: int) -> dict | None:
    """Pinned host<->device copy bandwidth of this box (the host-link
    roofline of the e2e number): best of 5 copies of nbytes each way."""
    import torch

    try:
        dev = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        host = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
        res = {}
        for name, fn in (("h2d_gbs", lambda: dev.copy_(host, non_blocking=True)),
                         ("d2h_gbs", lambda: host.copy_(dev, non_blocking=True))):
            best = None
            for _ in range(5):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fn()
                e1.record()
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1)
                best = t if best is None else min(best, t)
            res[name] = nbytes / (best / 1e3) / 1e9
        res["how"] = f"pinned copy of {nbytes} bytes each way, best of 5 (CUDA events)"
        del dev, host
        return res
    except Exception:
        return None


def _screened_vs_plain(args, local_rank: int) -> dict:
    """The metric's comparison: the tensor-core-screened join against the
    plain exact FP32 join on the 18-D and 90-D workloads, end to end through
    gsj_join_host (pinned host input and outputs), same step counts for both
    arms, and both arms' outputs compared entry by entry."""
    import torch

    from gpu_self_join_b200 import JoinConfig, SelfJoin, synth

    out = {}
    for name in ("c4_derived18d", "c5_heavy90d"):
        w = synth.WORKLOADS[name]
        pts = synth.generate(name)
        N, n = pts.shape
        h_in = torch.from_numpy(pts).pin_memory().numpy()
        res, tables = {}, {}
        with SelfJoin(local_rank) as sj:
            for arm, plain in (("screened", False), ("plain", True)):
                cfg = JoinConfig(indexed_dims=w.k, reorder=w.reorder, shortcircuit=w.shortcircuit, ilp=w.ilp,
                                 stamp=w.stamp, query_reorder=w.query_reorder, plain=plain)
                st, _, _ = sj.run_host(h_in, w.eps, cfg)  # warm-up, gives the result size
                R = int(st["total_pairs"])
                hc = torch.empty(N, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
                ht = torch.empty(max(R, 1), dtype=torch.int32).pin_memory().numpy().view(np.uint32)[:R]
                sampler = ClockSampler(local_rank)
                sampler.start()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                stats = []
                e0.record()
                for _ in range(args.sv_steps):
                    stats.append(sj.run_host(h_in, w.eps, cfg, counts=hc, table=ht)[0])
                e1.record()
                torch.cuda.synchronize()
                clocks = sampler.stop()
                ms = e0.elapsed_time(e1) / args.sv_steps
                s = stats[-1]
                res[arm] = {"e2e_ms": ms, "pairs_per_s": R / (ms / 1e3), "result_pairs": R,
                            "join_path": int(s["join_path"]), "stage_ms": {"index": s["dev_ms_index"],
                            "count": s["dev_ms_count"], "fill": s["dev_ms_fill"]},
                            "screen_rechecks": int(s["screen_rechecks"]), "candidates": int(s["candidates"]),
                            "clocks": clocks}
                if plain:
                    # FP32 work of the reference's traversal: 3n FLOPs per candidate
                    flops = 3.0 * n * s["candidates"]
                    res[arm]["fp32_tflops"] = flops / (s["dev_ms_count"] / 1e3) / 1e12
                else:
                    tpk, kind = _tensor_peak()
                    tf = 2.0 * (n + 2) * s["candidates"] / (s["dev_ms_count"] / 1e3) / 1e12
                    res[arm]["tensor"] = {"tflops": tf, "peak": tpk, "frac": tf / tpk, "peak_source": kind}
                tables[arm] = (hc.copy(), ht.copy())
        same = (np.array_equal(tables["screened"][0], tables["plain"][0])
                and np.array_equal(tables["screened"][1], tables["plain"][1]))
        res["same_pairs"] = bool(same)
        res["speedup_e2e"] = res["plain"]["e2e_ms"] / res["screened"]["e2e_ms"]
        res["points"], res["dim"], res["eps"], res["steps"] = N, n, w.eps, args.sv_steps
        out[name] = res
        del tables
    return out


def _learned_vs_sampled(args, local_rank: int) -> dict:
    """The 6-D workload's estimator comparison: the result-count model is
    trained on the device on the exact per-cell counts of a join of the same
    distribution at half size, then the full 5M-point join runs with the
    sampled estimator and with the learned one (device-resident input, same
    step counts); reported: each estimate, its error, its device time, the
    join time, re-runs, and whether both joins gave the same lists."""
    import torch

    from gpu_self_join_b200 import JoinConfig, SelfJoin, synth

    name = "c3_gmm6d"
    w = synth.WORKLOADS[name]
    cfg_s = JoinConfig(indexed_dims=w.k, reorder=w.reorder, shortcircuit=w.shortcircuit, ilp=w.ilp, stamp=w.stamp,
                       query_reorder=w.query_reorder)
    cfg_l = JoinConfig(indexed_dims=w.k, reorder=w.reorder, shortcircuit=w.shortcircuit, ilp=w.ilp, stamp=w.stamp,
                       query_reorder=w.query_reorder, learned=True)
    out = {"workload": name, "train_points": 2_500_000}
    with SelfJoin(local_rank) as sj:
        sj.run(torch.from_numpy(synth.generate(name, 2_500_000)).cuda(), w.eps, cfg_s)
        t0 = time.perf_counter()
        loss = sj.model_train(400)
        out["train"] = {"steps": 400, "wall_ms": (time.perf_counter() - t0) * 1e3, "last_loss": loss}
        x = torch.from_numpy(synth.generate(name)).cuda()
        lists = {}
        for arm, cfg in (("sampled", cfg_s), ("learned", cfg_l)):
            sj.run(x, w.eps, cfg)  # warm-up
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            stats = [sj.run(x, w.eps, cfg) for _ in range(args.sv_steps)]
            e1.record()
            torch.cuda.synchronize()
            s = stats[-1]
            R = int(s["total_pairs"])
            out[arm] = {"join_ms": e0.elapsed_time(e1) / args.sv_steps, "estimate": int(s["estimate"]),
                        "estimate_error": (int(s["estimate"]) - R) / R, "estimate_dev_ms": s["dev_ms_estimate"],
                        "reruns": int(s["reruns"]), "result_pairs": R}
            lists[arm] = (sj.counts(), sj.table())
    out["same_pairs"] = bool(np.array_equal(lists["sampled"][0], lists["learned"][0])
                             and np.array_equal(lists["sampled"][1], lists["learned"][1]))
    return out


HARNESS = os.path.join(ROOT, "oracle", "_ref", "rtree_harness")


def _rtree_runs(pts: np.ndarray, w, steps: int, sample: int, threads: int, seed: int = 1) -> dict:
    """Runs the reference's R-tree self-join code (oracle/_ref/rtree_harness,
    built from the reference's sources) once: tree over all points, then
    `steps` rounds of `sample` seeded queries."""
    import tempfile

    with tempfile.TemporaryDirectory() as td:
        f = os.path.join(td, "pts.bin")
        np.ascontiguousarray(pts, dtype=np.float32).tofile(f)
        out = subprocess.run([HARNESS, f, str(pts.shape[0]), str(pts.shape[1]), repr(float(w.eps)), str(threads),
                              str(steps), str(sample), str(seed)], capture_output=True, text=True, check=True)
    return json.loads(out.stdout.strip().splitlines()[-1])


def _rtree_step_values(r: dict) -> list[float]:
    N, smp, tb = r["N"], r["sample"], r["build_s"]
    return [(st["pairs"] * N / smp) / (tb + st["query_s"] * N / smp) for st in r["steps"]]


def _rtree_sample_text(r: dict, nsteps: int) -> str:
    return (f"reference R-tree (RTree.h + tree_index.cpp:191-233, built from the reference's sources): tree over all "
            f"{r['N']} points built once in {r['build_s']:.2f} s on 1 thread as the reference does; {nsteps} rounds of "
            f"{r['sample']} seeded queries on {r['threads']} threads; pairs/s extrapolated to the full join "
            f"(build + all {r['N']} queries)")


def _cpu_baseline(pts: np.ndarray, w, budget_s: float = 15.0) -> dict:
    """The reference's own CPU self-join (its R-tree search and filter) on a
    bounded query sample of the same workload, all host threads; the oracle's
    grid join (a CPU port of algorithm 3) where the harness is not built."""
    cores = os.cpu_count() or 1
    N = pts.shape[0]
    if os.path.exists(HARNESS) and pts.shape[1] == 2:
        r = _rtree_runs(pts, w, steps=3, sample=min(N, 200_000), threads=cores)
        v = _rtree_step_values(r)
        return {"value": statistics.mean(v), "unit": "pairs/s", "cores": cores, "kind": "reference",
                "sample": _rtree_sample_text(r, 3)}
    from oracle import pyoracle as O

    O.lib()
    rng = np.random.default_rng(12345)
    cfg = O.OracleConfig(k=w.k, reorder=w.reorder, ilp=w.ilp, shortcircuit=w.shortcircuit, nthreads=cores)
    nq = min(N, 20000)
    q = np.sort(rng.choice(N, size=nq, replace=False)).astype(np.uint32)
    tot, si, sq = O.join_sample(pts, w.eps, cfg, q)
    per_q = sq / nq
    nq2 = int(min(N, max(nq, (budget_s - si) / max(per_q, 1e-9))))
    if nq2 > nq * 2:
        q = np.sort(rng.choice(N, size=nq2, replace=False)).astype(np.uint32)
        tot, si, sq = O.join_sample(pts, w.eps, cfg, q)
        nq = nq2
    est_R = tot * (N / nq)
    est_t = si + sq * (N / nq)
    return {"value": est_R / est_t, "unit": "pairs/s", "cores": cores, "kind": "port",
            "sample": f"oracle grid join: index over all {N} points ({si:.2f} s) + {nq} seeded queries "
                      f"({sq:.2f} s); pairs/s extrapolated to all {N} queries"}


# ------------------------------------------------------------------ request stream
def _calibrate_eps(x, target: float, seed: int) -> float:
    """eps with `target` mean neighbours per point (self included) on 256
    seeded queries: the (256 * target)-th smallest of their squared distances
    to all points (float64 on the device), i.e. the sample mean count at eps
    is the target."""
    import torch

    N = x.shape[0]
    g = torch.Generator(device=x.device)
    g.manual_seed(seed)
    q = x[torch.randperm(N, generator=g, device=x.device)[:256]].double()
    qn = (q * q).sum(1, keepdim=True)
    k = max(1, int(round(q.shape[0] * target)))
    best = None
    for c0 in range(0, N, 65536):
        p = x[c0:c0 + 65536].double()
        d2 = (qn + (p * p).sum(1)[None, :] - 2.0 * (q @ p.T)).clamp_min(0.0).reshape(-1)
        cand = d2 if best is None else torch.cat([best, d2])
        best = torch.topk(cand, min(k, cand.numel()), largest=False).values
    return float(best.max().sqrt().item())


def _requests(args) -> None:
    """The 90-D workload's second phase: a seeded stream of independent joins
    (N log-uniform in [10k, 500k], n from {8, 16, 32, 90}, eps for 10-100 mean
    neighbours, the 90-D workload's switches), each through gsj_join on
    device-resident points.  Reports the per-request latency (host wall clock
    around the call, which returns when the join is done) and the stream's
    result pairs per second."""
    import time

    import torch

    from gpu_self_join_b200 import JoinConfig, SelfJoin, synth

    rank, local_rank, world = _env_rank()
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    reqs = synth.request_stream(args.requests)
    prepared = []
    for r in reqs:
        x = torch.from_numpy(synth.gen_heavy(r.N, r.n, r.seed)).cuda()
        prepared.append((r, x, _calibrate_eps(x, r.target_mean, r.seed)))
    torch.cuda.synchronize()
    sj = SelfJoin(local_rank)

    def cfg_of(r):
        return JoinConfig(indexed_dims=min(6, r.n), reorder=True, shortcircuit=True, ilp=8, stamp=False,
                          query_reorder=True, plain=args.plain)

    # Workers: long-lived contexts (own stream and memory pool each), one host
    # thread per context pulling the next request; the library releases the
    # interpreter lock inside every call, so the joins of different workers
    # overlap on the GPU.
    import queue
    import threading

    workers = [sj] + [SelfJoin(local_rank) for _ in range(max(1, args.workers) - 1)]
    for wj in workers:
        for r, x, eps in prepared[:max(3, args.warmup)]:
            wj.run(x, eps, cfg_of(r))
    torch.cuda.synchronize()
    lat, stats_all = [0.0] * len(prepared), [None] * len(prepared)
    todo = queue.Queue()
    for i in range(len(prepared)):
        todo.put(i)

    def serve(wj):
        while True:
            try:
                i = todo.get_nowait()
            except queue.Empty:
                return
            r, x, eps = prepared[i]
            t0 = time.perf_counter()
            stats_all[i] = wj.run(x, eps, cfg_of(r))
            lat[i] = (time.perf_counter() - t0) * 1e3

    t_all = time.perf_counter()
    threads = [threading.Thread(target=serve, args=(wj,)) for wj in workers]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    t_all = time.perf_counter() - t_all
    pairs = sum(int(st["total_pairs"]) for st in stats_all)
    paths = {}
    for st in stats_all:
        paths[int(st["join_path"])] = paths.get(int(st["join_path"]), 0) + 1
    for wj in workers:
        wj.close()
    lat_sorted = sorted(lat)

    def pct(p):
        return lat_sorted[min(len(lat_sorted) - 1, int(round(p / 100.0 * (len(lat_sorted) - 1))))]

    def mean_of(key):
        return statistics.mean(float(st[key]) for st in stats_all)

    line = {
        "metric": "request stream: result pairs/s (256 joins, 90-D workload phase 2)", "value": pairs / t_all,
        "unit": "pairs/s", "n_gpus": 1, "steps": len(prepared), "warmup": max(3, args.warmup),
        "ms_per_step": t_all * 1e3 / len(prepared), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded request stream)",
        "config": {"workload": "c5_requests", "requests": len(prepared), "plain": bool(args.plain),
                   "N_range": [min(r.N for r, _, _ in prepared), max(r.N for r, _, _ in prepared)],
                   "dims": sorted({r.n for r, _, _ in prepared}), "result_pairs": pairs,
                   "join_paths": {str(k): v for k, v in sorted(paths.items())}},
        "latency_ms": {"p50": pct(50), "p90": pct(90), "p99": pct(99), "max": lat_sorted[-1]},
        "workers": len(workers),
        "mean_ms": {"host_index": mean_of("ms_index"), "host_join": mean_of("ms_join"),
                    "dev_index": mean_of("dev_ms_index"), "dev_count": mean_of("dev_ms_count"),
                    "dev_fill": mean_of("dev_ms_fill"), "launches": mean_of("kernel_launches")},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def _ours(args) -> None:
    import torch
    import torch.distributed as dist

    from gpu_self_join_b200 import JoinConfig, SelfJoin, synth
    from gpu_self_join_b200.replicas import reduce_step

    rank, local_rank, world = _env_rank()
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    w = synth.WORKLOADS[args.workload]
    pts = synth.generate(args.workload, args.points)
    N, n = pts.shape
    cfg = JoinConfig(indexed_dims=w.k, reorder=w.reorder, shortcircuit=w.shortcircuit, ilp=w.ilp, stamp=w.stamp,
                     query_reorder=w.query_reorder, plain=args.plain)
    sj = SelfJoin(local_rank)
    x_dev = torch.from_numpy(pts).cuda()
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- value: device-resident input and result
    for _ in range(args.warmup):
        sj.run(x_dev, w.eps, cfg)
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    stats = []
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        stats.append(sj.run(x_dev, w.eps, cfg))
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    R = stats[-1]["total_pairs"]
    pairs_local = R * args.steps
    ms_max, pairs_all = reduce_step(ms, pairs_local, device="cuda")
    value = pairs_all / (ms_max / 1e3)

    # ---- roofline of the dominant kernel
    roof = _roofline(stats, N, n, R, w)

    # ---- e2e: host buffers through the public API (gsj_join_host: pinned
    # input, the table produced in batches that are copied to pinned host
    # memory while the next batch is computed)
    e2e = None
    if not args.no_e2e:
        h_in = torch.from_numpy(pts).pin_memory().numpy()
        h_counts = torch.empty(N, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
        h_table = torch.empty(max(R, 1), dtype=torch.int32).pin_memory().numpy().view(np.uint32)[:R]
        for _ in range(max(1, min(args.warmup, 2))):
            sj.run_host(h_in, w.eps, cfg, counts=h_counts, table=h_table)
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        est = []
        for _ in range(args.steps):
            est.append(sj.run_host(h_in, w.eps, cfg, counts=h_counts, table=h_table)[0])
        f1.record()
        torch.cuda.synchronize()
        barrier()
        ems, _ = reduce_step(f0.elapsed_time(f1), 0.0, device="cuda")
        d2h = int(4 * N + 4 * R)
        e2e = {"value": pairs_all / (ems / 1e3), "unit": "pairs/s", "ms_per_step": ems / args.steps,
               "h2d_bytes_per_step": int(N * n * 4), "d2h_bytes_per_step": d2h,
               "batches": int(est[-1]["batches"]), "api": "gsj_join_host (pinned host buffers)",
               "host_ms": {k: float(np.mean([e[k] for e in est]))
                           for k in ("ms_h2d", "ms_index", "ms_join", "ms_d2h", "ms_total")}}
        link = _link_peaks(max(d2h, 1 << 26))
        if link:
            t_link = (N * n * 4) / (link["h2d_gbs"] * 1e9) + d2h / (link["d2h_gbs"] * 1e9)
            e2e["roofline"] = {"bound": "host link", "h2d_gbs": link["h2d_gbs"], "d2h_gbs": link["d2h_gbs"],
                               "link_ms": t_link * 1e3, "frac": t_link * 1e3 / (ems / args.steps),
                               "how": link["how"]}

    launches = int(sum(s.get("kernel_launches", 0) for s in stats))
    line = {
        "metric": "self-join result pairs/s (2-D, 20M points, STAMP=1)" if args.workload == "c2_gmm2d"
        else f"self-join result pairs/s ({args.workload})",
        "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded, shapes/distributions of the benchmark workload)",
        "config": {"workload": args.workload, "points": N, "dim": n, "eps": w.eps, "indexed_dims": w.k,
                   "plain": bool(args.plain),
                   "stamp": w.stamp, "reorder": w.reorder, "ilp": w.ilp, "shortcircuit": w.shortcircuit,
                   "query_reorder": w.query_reorder, "result_pairs_per_step": R,
                   "candidates_per_step": stats[-1]["candidates"], "join_path": int(stats[-1]["join_path"]),
                   "screen_rechecks_per_step": int(stats[-1]["screen_rechecks"]), "parallelism": f"replicas x{world}",
                   "l2": "inputs (160 MB) and working set larger than L2"},
        "roofline": roof, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
    }
    if rank == 0 and world == 1 and args.workload == "c2_gmm2d" and not args.no_screened_vs_plain:
        sj.close()
        try:
            line["screened_vs_plain"] = _screened_vs_plain(args, local_rank)
        except Exception as ex:  # reported, never required for the headline line
            line["screened_vs_plain"] = {"error": str(ex)}
        try:
            line["learned_vs_sampled"] = _learned_vs_sampled(args, local_rank)
        except Exception as ex:  # reported, never fatal for the headline line
            line["learned_vs_sampled"] = {"error": str(ex)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = _cpu_baseline(pts, w)
        except Exception as ex:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(ex)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sj.close()
    if world > 1:
        dist.destroy_process_group()


# ------------------------------------------------------------------ reference arm
def _reference_arm(args) -> None:
    """The reference's CPU implementation of the self-join (its R-tree search
    and filter, tree_index.cpp:191-233, built from its sources into
    oracle/_ref/rtree_harness) on the same workload with all host threads:
    the tree is built once over all points, then W + K rounds of seeded
    queries; each round's value is the pairs/s of the full join extrapolated
    from it.  Without the harness, the oracle port of algorithm 3 is timed."""
    rank, _, world = _env_rank()
    if rank != 0:
        return
    from gpu_self_join_b200 import synth

    w = synth.WORKLOADS[args.workload]
    pts = synth.generate(args.workload, args.points)
    N, n = pts.shape
    cores = os.cpu_count() or 1
    if os.path.exists(HARNESS) and n == 2:
        r = _rtree_runs(pts, w, steps=args.warmup + args.steps, sample=min(N, 200_000), threads=cores)
        vals = _rtree_step_values(r)[args.warmup:]
        kind, desc = "reference", _rtree_sample_text(r, args.steps)
    else:
        vals = []
        for _ in range(args.warmup + args.steps):
            vals.append(_cpu_baseline(pts, w, budget_s=5.0)["value"])
        vals = vals[args.warmup:]
        kind, desc = "port", "oracle grid join (CPU port of algorithm 3) on seeded query samples"
    value = statistics.mean(vals)
    metric = ("self-join result pairs/s (2-D, 20M points, STAMP=1)" if args.workload == "c2_gmm2d"
              else f"self-join result pairs/s ({args.workload})")
    line = {"impl": "reference", "metric": metric, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "points": N, "dim": n, "eps": w.eps},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": kind, "sample": desc},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2_gmm2d")
    ap.add_argument("--points", type=int, default=None,
                    help="generate a smaller instance of the workload (profiling captures only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--requests", type=int, default=256, help="joins in the c5_requests stream")
    ap.add_argument("--workers", type=int, default=1,
                    help="c5_requests: concurrent worker contexts (one stream and host thread each)")
    ap.add_argument("--no-screened-vs-plain", action="store_true",
                    help="skip the 18-D / 90-D screened-versus-plain block of the default line")
    ap.add_argument("--sv-steps", type=int, default=3, help="timed joins per arm of the screened-vs-plain block")
    ap.add_argument("--plain", action="store_true",
                    help="no tensor-core screen on high-dimensional workloads (exact FP32 for every pair)")
    args = ap.parse_args()
    if args.impl == "reference":
        _reference_arm(args)
    elif args.workload == "c5_requests":
        _requests(args)
    else:
        _ours(args)


if __name__ == "__main__":
    main()
