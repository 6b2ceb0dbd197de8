"""Context-based Python API over the C ABI (include/gpuselfjoin.h).

    with SelfJoin(device=0) as sj:
        stats = sj.run(points, eps, indexed_dims=2, stamp=True)
        counts, table = sj.counts(), sj.table()

``points`` is an N x n float32/float64 numpy array (host) or a CUDA torch
tensor (device-resident input, no host copy).  Results stay on the device
until fetched; ``counts_offsets_table_device`` returns them as CUDA torch
tensors without a host round trip.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class JoinConfig:
    """The reference's params.h switches that shape a join (params.h:17-93)."""

    indexed_dims: int = 6     # NUMINDEXEDDIM (clamped to n)
    reorder: bool = False     # REORDER
    shortcircuit: bool = False  # SHORTCIRCUIT
    ilp: int = 0              # ILP
    stamp: bool = False       # STAMP
    query_reorder: bool = False  # QUERYREORDER
    sort_lists: bool = False  # sort each neighbour list ascending
    no_unicomp: bool = False  # full-neighbourhood traversal even with stamp (same pair set)
    plain: bool = False       # no tensor-core screen (every pair in exact FP32; same pair set)
    exact_size: bool = False  # pair buffers sized by a counting pass, not an estimate (same pair set)
    buffer_pairs: int = 0     # GPUBUFFERSIZE: entries per device result segment of run_host (0: 100M)
    streams: int = 0          # GPUSTREAMS: result segments in flight in run_host (0: 3)
    min_batches: int = 0      # MINBATCHES: fewest result batches of run_host (0: 3)
    learned: bool = False     # size pair buffers with the context's learned result-count model
    sort: bool = False        # SORT: cells sorted by one dimension, neighbour scans pruned (the reference's pairs)


class SelfJoin:
    def __init__(self, device: int = 0):
        self._L = N.lib()
        self._ctx = ctypes.c_void_p()
        N.check(self._L.gsj_create(ctypes.byref(self._ctx), int(device)))
        self.device = int(device)
        self.n = 0
        self.N = 0

    def close(self) -> None:
        if self._ctx:
            self._L.gsj_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _cfg(self, n: int, dtype, cfg: JoinConfig) -> N.GsjConfig:
        c = N.GsjConfig()
        c.dim = n
        c.indexed_dims = min(int(cfg.indexed_dims), n)
        c.dtype = N.GSJ_FLOAT64 if dtype == np.float64 else N.GSJ_FLOAT32
        c.reorder = int(cfg.reorder)
        c.shortcircuit = int(cfg.shortcircuit)
        c.ilp = int(cfg.ilp)
        c.stamp = int(cfg.stamp)
        c.query_reorder = int(cfg.query_reorder)
        c.device = self.device
        c.flags = (N.GSJ_FLAG_QUIET | (N.GSJ_FLAG_SORT_LISTS if cfg.sort_lists else 0)
                   | (N.GSJ_FLAG_NO_UNICOMP if cfg.no_unicomp else 0) | (N.GSJ_FLAG_PLAIN if cfg.plain else 0)
                   | (N.GSJ_FLAG_EXACT_SIZE if cfg.exact_size else 0))
        c.buffer_pairs = int(cfg.buffer_pairs)
        c.streams = int(cfg.streams)
        c.min_batches = int(cfg.min_batches)
        c.estimator = N.GSJ_EST_LEARNED if cfg.learned else N.GSJ_EST_SAMPLED
        c.sort = int(cfg.sort)
        return c

    def run(self, points, eps: float, config: JoinConfig | None = None, **kw) -> dict:
        """Runs the join; returns the native statistics as a dict."""
        cfg = config or JoinConfig(**kw)
        st = N.GsjStats()
        if hasattr(points, "is_cuda") and points.is_cuda:  # torch tensor on the device
            import torch

            if points.dim() != 2 or not points.is_contiguous():
                raise ValueError("points must be a contiguous N x n tensor")
            dt = np.float64 if points.dtype == torch.float64 else np.float32
            if points.dtype not in (torch.float32, torch.float64):
                raise TypeError("points must be float32 or float64")
            Np, n = points.shape
            c = self._cfg(n, dt, cfg)
            N.check(self._L.gsj_join(self._ctx, ctypes.c_void_p(points.data_ptr()), Np, float(eps), ctypes.byref(c), 1,
                                     ctypes.byref(st)), self._ctx)
        else:
            p = np.ascontiguousarray(points)
            if p.dtype not in (np.float32, np.float64):
                p = p.astype(np.float32)
            if p.ndim != 2:
                raise ValueError("points must be N x n")
            Np, n = p.shape
            c = self._cfg(n, p.dtype, cfg)
            N.check(self._L.gsj_join(self._ctx, p.ctypes.data, Np, float(eps), ctypes.byref(c), 0, ctypes.byref(st)),
                    self._ctx)
        self.N, self.n = Np, n
        return st.as_dict()

    def run_host(self, points, eps: float, config: JoinConfig | None = None, counts: np.ndarray | None = None,
                 table: np.ndarray | None = None, **kw) -> tuple[dict, np.ndarray, np.ndarray]:
        """Runs the join with the result delivered to host memory
        (gsj_join_host): the table is produced in batches that are copied to
        the host while the next batch is computed.  ``counts``/``table`` may
        be given (pinned buffers are written by DMA directly); a table that is
        too small is replaced by one of the exact size and the join repeated.
        Returns (stats, numNeighbors, neighborTable)."""
        cfg = config or JoinConfig(**kw)
        st = N.GsjStats()
        on_dev = hasattr(points, "is_cuda") and points.is_cuda
        if on_dev:
            Np, n = points.shape
            import torch

            dt = np.float64 if points.dtype == torch.float64 else np.float32
            ptr = ctypes.c_void_p(points.data_ptr())
        else:
            p = np.ascontiguousarray(points)
            if p.dtype not in (np.float32, np.float64):
                p = p.astype(np.float32)
            Np, n = p.shape
            dt = p.dtype
            ptr = ctypes.c_void_p(p.ctypes.data)
        c = self._cfg(n, dt, cfg)
        counts = np.empty(Np, dtype=np.uint32) if counts is None else counts
        table = np.empty(0, dtype=np.uint32) if table is None else table
        total = ctypes.c_uint64()
        for _ in range(2):
            rc = self._L.gsj_join_host(self._ctx, ptr, Np, float(eps), ctypes.byref(c), int(on_dev),
                                       counts.ctypes.data, table.ctypes.data if table.size else None, table.size,
                                       ctypes.byref(total), ctypes.byref(st))
            if rc == N.GSJ_ERR_OVERFLOW:
                table = np.empty(int(total.value), dtype=np.uint32)
                continue
            N.check(rc, self._ctx)
            break
        self.N, self.n = Np, n
        return st.as_dict(), counts, table[: int(total.value)]

    # ---- launch-shape tuning
    def _points_arg(self, points):
        if hasattr(points, "is_cuda") and points.is_cuda:
            import torch

            dt = np.float64 if points.dtype == torch.float64 else np.float32
            return ctypes.c_void_p(points.data_ptr()), points.shape, dt, 1, points
        p = np.ascontiguousarray(points)
        if p.dtype not in (np.float32, np.float64):
            p = p.astype(np.float32)
        return ctypes.c_void_p(p.ctypes.data), p.shape, p.dtype, 0, p

    def autotune(self, points, eps: float, config: JoinConfig | None = None, repeats: int = 2, **kw) -> dict:
        """Times the join of `points` under candidate launch shapes of the path
        it takes and keeps the fastest in this context's tuning table;
        returns the chosen shape."""
        cfg = config or JoinConfig(**kw)
        ptr, shape, dt, on_dev, keep = self._points_arg(points)
        c = self._cfg(shape[1], dt, cfg)
        t = N.GsjTuning()
        N.check(self._L.gsj_autotune(self._ctx, ptr, shape[0], float(eps), ctypes.byref(c), on_dev, int(repeats),
                                     ctypes.byref(t)), self._ctx)
        del keep
        return t.as_dict()

    def tuning(self, path: int, dim: int, density_log2: int, shape: dict | None = None) -> dict | None:
        """The tuning-table entry of (path, dim, density_log2); with `shape`,
        sets it first.  None when there is no entry."""
        t = N.GsjTuning()
        if shape is not None:
            for k, v in shape.items():
                setattr(t, k, int(v))
            N.check(self._L.gsj_tuning_set(self._ctx, path, dim, density_log2, ctypes.byref(t)), self._ctx)
        if self._L.gsj_tuning_get(self._ctx, path, dim, density_log2, ctypes.byref(t)) != N.GSJ_OK:
            return None
        return t.as_dict()

    # ---- learned result-count model (GSJ_EST_LEARNED)
    def model_train(self, steps: int = 400) -> float:
        """Trains the context's model on the exact counts of the last join;
        returns the last minibatch loss."""
        loss = ctypes.c_float()
        N.check(self._L.gsj_model_train(self._ctx, int(steps), ctypes.byref(loss)), self._ctx)
        return float(loss.value)

    def model_reset(self) -> None:
        N.check(self._L.gsj_model_reset(self._ctx), self._ctx)

    def model_weights(self, weights: np.ndarray | None = None) -> np.ndarray:
        """The model's weights; with `weights`, sets them first."""
        if weights is not None:
            w = np.ascontiguousarray(weights, dtype=np.float32)
            N.check(self._L.gsj_model_weights(self._ctx, w.ctypes.data, w.size, 1), self._ctx)
        out = np.empty(N.MODEL_WEIGHTS, dtype=np.float32)
        N.check(self._L.gsj_model_weights(self._ctx, out.ctypes.data, out.size, 0), self._ctx)
        return out

    def model_features(self) -> tuple[np.ndarray, np.ndarray]:
        """The last join's per-cell features and targets (log2(1 + mean count))."""
        m = ctypes.c_uint32()
        N.check(self._L.gsj_model_features(self._ctx, None, None, 0, ctypes.byref(m)), self._ctx)
        X = np.empty((m.value, N.MODEL_FEATURES), dtype=np.float32)
        y = np.empty(m.value, dtype=np.float32)
        N.check(self._L.gsj_model_features(self._ctx, X.ctypes.data, y.ctypes.data, m.value, ctypes.byref(m)),
                self._ctx)
        return X, y

    def model_predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.empty(X.shape[0], dtype=np.float32)
        N.check(self._L.gsj_model_predict(self._ctx, X.ctypes.data, X.shape[0], out.ctypes.data), self._ctx)
        return out

    def model_loss_grad(self, X: np.ndarray, y: np.ndarray) -> tuple[float, np.ndarray]:
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        grad = np.empty(N.MODEL_WEIGHTS, dtype=np.float32)
        N.check(self._L.gsj_model_loss_grad(self._ctx, X.ctypes.data, y.ctypes.data, X.shape[0], loss.ctypes.data,
                                            grad.ctypes.data), self._ctx)
        return float(loss[0]), grad

    def bruteforce(self, points, eps: float) -> tuple[np.ndarray, int]:
        """Brute-force neighbour counts over all N^2 pairs (the reference's GPU
        algorithm 1, kernel.cu:486-515): (counts per point, total).  Replaces
        any join result held by this object."""
        p = np.ascontiguousarray(points)
        if p.dtype not in (np.float32, np.float64):
            p = p.astype(np.float32)
        if p.ndim != 2:
            raise ValueError("points must be N x n")
        Np, n = p.shape
        c = self._cfg(n, p.dtype, JoinConfig(indexed_dims=min(6, n)))
        counts = np.empty(Np, dtype=np.uint32)
        total = ctypes.c_uint64()
        N.check(self._L.gsj_bruteforce_count(self._ctx, p.ctypes.data, Np, float(eps), ctypes.byref(c), 0,
                                             counts.ctypes.data, ctypes.byref(total)), self._ctx)
        self.N = 0
        return counts, int(total.value)

    def total_pairs(self) -> int:
        r = ctypes.c_uint64()
        N.check(self._L.gsj_result_size(self._ctx, ctypes.byref(r)), self._ctx)
        return int(r.value)

    def counts(self, out: np.ndarray | None = None) -> np.ndarray:
        out = np.empty(self.N, dtype=np.uint32) if out is None else out
        N.check(self._L.gsj_result_counts(self._ctx, out.ctypes.data, 0), self._ctx)
        return out

    def table(self, out: np.ndarray | None = None) -> np.ndarray:
        R = self.total_pairs()
        out = np.empty(R, dtype=np.uint32) if out is None else out
        N.check(self._L.gsj_result_table(self._ctx, out.ctypes.data, out.size, 0), self._ctx)
        return out

    def counts_offsets_table_device(self):
        """(counts int32[N], offsets int64[N+1], table int32[R]) as CUDA torch
        tensors (copies of the context's result, device to device)."""
        import torch

        R = self.total_pairs()
        dev = torch.device("cuda", self.device)
        counts = torch.empty(self.N, dtype=torch.int32, device=dev)
        table = torch.empty(max(R, 1), dtype=torch.int32, device=dev)[:R]
        offsets = torch.empty(self.N + 1, dtype=torch.int64, device=dev)
        cp, op, tp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        N.check(self._L.gsj_result_device(self._ctx, ctypes.byref(cp), ctypes.byref(op), ctypes.byref(tp)), self._ctx)
        N.check(self._L.gsj_result_counts(self._ctx, ctypes.c_void_p(counts.data_ptr()), 1), self._ctx)
        if R:
            N.check(self._L.gsj_result_table(self._ctx, ctypes.c_void_p(table.data_ptr()), R, 1), self._ctx)
        torch.cuda.synchronize(dev)
        # offsets: a device copy through a tensor view of the native buffer
        offsets.copy_(torch.cumsum(torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), counts.to(torch.int64)]),
                                   0))
        return counts, offsets, table


def threshold(eps: float, dtype=np.float32) -> float:
    """Largest s with sqrt(s) <= eps in dtype (the distance test's threshold)."""
    L = N.lib()
    if np.dtype(dtype) == np.float64:
        return L.gsj_threshold_f64(float(eps))
    return L.gsj_threshold_f32(float(eps))
