"""ctypes binding of the CPU oracle (oracle/gsj_oracle.cpp).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` as the checker; the product path never
imports it.  The oracle restates the reference's algorithm 3 on the CPU
(main.cu:690-1075, kernel.cu:132-480, GPU.cu:57-268 and GPU.cu:1491-1525 of
mgowanlock/gpu_self_join).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

MODEL_DEVICE = 0  # reference GPU arithmetic (fused multiply-add chain)
MODEL_HOST = 1    # reference host arithmetic (no contraction)
MODEL_FP64 = 2    # double-precision decision


class _Cfg(ctypes.Structure):
    _fields_ = [
        ("k", ctypes.c_uint32),
        ("reorder", ctypes.c_uint32),
        ("ilp", ctypes.c_uint32),
        ("shortcircuit", ctypes.c_uint32),
        ("model", ctypes.c_uint32),
        ("sc_contract", ctypes.c_uint32),
        ("stamp_ref", ctypes.c_uint32),
        ("nthreads", ctypes.c_uint32),
        ("fold_zero", ctypes.c_uint32),
        ("fuse_left", ctypes.c_uint32),
        ("cross_left", ctypes.c_uint32),
        ("sort", ctypes.c_uint32),
    ]


@dataclass
class OracleConfig:
    """Mirror of the reference's params.h switches that affect results."""

    k: int                    # NUMINDEXEDDIM
    reorder: bool = False     # REORDER
    ilp: int = 0              # ILP
    shortcircuit: bool = False  # SHORTCIRCUIT
    model: int = MODEL_DEVICE
    sc_contract: bool = False
    stamp_ref: bool = False   # reproduce the reference's STAMP=1 duplicated output
    nthreads: int = 0
    fold_zero: bool | None = None  # None: the pinned policy of the dtype
    fuse_left: bool | None = None
    cross_left: bool | None = None
    sort: bool = False        # SORT: per-cell sorted points, pruned scans (params.h:46)

    def c(self, dtype=np.float32) -> _Cfg:
        fz, fl, xl = pinned_policy(dtype)
        fz = fz if self.fold_zero is None else self.fold_zero
        fl = fl if self.fuse_left is None else self.fuse_left
        xl = xl if self.cross_left is None else self.cross_left
        return _Cfg(self.k, int(self.reorder), self.ilp, int(self.shortcircuit), self.model,
                    int(self.sc_contract), int(self.stamp_ref), self.nthreads, int(fz), int(fl), int(xl),
                    int(self.sort))


def pinned_policy(dtype) -> tuple[bool, bool, bool]:
    """(fold_zero, fuse_left, cross_left) of the reference's device arithmetic,
    as pinned against the reference's own builds (tests/golden/ref_pins.json):
    float32 keeps fma(d, d, 0); float64 folds 0 + d*d to a pending product and,
    when both operands of an addition are pending products, fuses the
    accumulator's in `acc += d*d` and the added register's in
    `runningDist[0] += runningDist[j]`."""
    if np.dtype(dtype) == np.float64:
        return True, True, False
    return False, False, False


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        u64, u32, i64 = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int64
        for sfx, fl in (("f32", ctypes.c_float), ("f64", ctypes.c_double)):
            getattr(_lib, f"orc_join_counts_{sfx}").argtypes = [P, u64, u32, fl, P, P, P, P]
            getattr(_lib, f"orc_join_lists_{sfx}").argtypes = [P, u64, u32, fl, P, P, P]
            getattr(_lib, f"orc_bruteforce_counts_{sfx}").argtypes = [P, u64, u32, fl, P, P, P]
            getattr(_lib, f"orc_reorder_perm_{sfx}").argtypes = [P, u64, u32, P, P]
            getattr(_lib, f"orc_grid_dims_{sfx}").argtypes = [P, u64, u32, u32, fl, P, P, P, P]
            getattr(_lib, f"orc_within_{sfx}").argtypes = [P, P, u32, fl, P]
            getattr(_lib, f"orc_import_text_{sfx}").argtypes = [ctypes.c_char_p, u32, P, u64]
            getattr(_lib, f"orc_import_text_{sfx}").restype = i64
        _lib.orc_join_sample_f32.argtypes = [P, u64, u32, ctypes.c_float, P, P, u64, P, P, P]
        _lib.orc_sample_lists_f32.argtypes = [P, u64, u32, ctypes.c_float, P, P, u64, P, P, u64, P]
        _lib.orc_sample_lists_f64.argtypes = [P, u64, u32, ctypes.c_double, P, P, u64, P, P, u64, P]
        _lib.orc_ref_batch_plan_f32.argtypes = [P, u64, u32, ctypes.c_float, P, P, P, u32,
                                                ctypes.c_double, P, P, P, P]
    return _lib


def _sfx(a: np.ndarray) -> str:
    if a.dtype == np.float32:
        return "f32"
    if a.dtype == np.float64:
        return "f64"
    raise TypeError(f"unsupported dtype {a.dtype}")


def _prep(points: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(points)
    if p.ndim != 2:
        raise ValueError("points must be N x n")
    return p


def join_counts(points: np.ndarray, eps: float, cfg: OracleConfig):
    """Per-point neighbour counts, total pairs and candidate evaluations."""
    p = _prep(points)
    N, n = p.shape
    s = _sfx(p)
    counts = np.zeros(N, dtype=np.uint32)
    total = ctypes.c_uint64()
    cand = ctypes.c_uint64()
    c = cfg.c(p.dtype)
    rc = getattr(lib(), f"orc_join_counts_{s}")(p.ctypes.data, N, n, eps, ctypes.byref(c),
                                                counts.ctypes.data, ctypes.byref(total),
                                                ctypes.byref(cand))
    if rc != 0:
        raise ValueError(f"oracle rejected the configuration (rc={rc})")
    return counts, int(total.value), int(cand.value)


def join_lists(points: np.ndarray, eps: float, cfg: OracleConfig):
    """(counts uint32[N], offsets uint64[N+1], neighbours uint32[R]) with each
    point's neighbour ids sorted ascending."""
    p = _prep(points)
    N, n = p.shape
    counts, total, _ = join_counts(p, eps, cfg)
    offsets = np.zeros(N + 1, dtype=np.uint64)
    np.cumsum(counts, out=offsets[1:])
    nbrs = np.zeros(total, dtype=np.uint32)
    c = cfg.c(p.dtype)
    rc = getattr(lib(), f"orc_join_lists_{_sfx(p)}")(p.ctypes.data, N, n, eps, ctypes.byref(c),
                                                     offsets.ctypes.data, nbrs.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle rejected the configuration (rc={rc})")
    return counts, offsets, nbrs


def bruteforce_counts(points: np.ndarray, eps: float, cfg: OracleConfig):
    p = _prep(points)
    N, n = p.shape
    counts = np.zeros(N, dtype=np.uint32)
    total = ctypes.c_uint64()
    c = cfg.c(p.dtype)
    getattr(lib(), f"orc_bruteforce_counts_{_sfx(p)}")(p.ctypes.data, N, n, eps, ctypes.byref(c),
                                                       counts.ctypes.data, ctypes.byref(total))
    return counts, int(total.value)


def reorder_perm(points: np.ndarray):
    p = _prep(points)
    N, n = p.shape
    perm = np.zeros(n, dtype=np.uint32)
    var = np.zeros(n, dtype=p.dtype)
    getattr(lib(), f"orc_reorder_perm_{_sfx(p)}")(p.ctypes.data, N, n, perm.ctypes.data,
                                                  var.ctypes.data)
    return perm, var


def grid_dims(points: np.ndarray, k: int, eps: float):
    p = _prep(points)
    N, n = p.shape
    mn = np.zeros(k, dtype=p.dtype)
    mx = np.zeros(k, dtype=p.dtype)
    nc = np.zeros(k, dtype=np.uint32)
    tot = ctypes.c_uint64()
    getattr(lib(), f"orc_grid_dims_{_sfx(p)}")(p.ctypes.data, N, n, k, eps, mn.ctypes.data,
                                               mx.ctypes.data, nc.ctypes.data, ctypes.byref(tot))
    return mn, mx, nc, int(tot.value)


def within(p: np.ndarray, c: np.ndarray, eps: float, cfg: OracleConfig) -> bool:
    p = np.ascontiguousarray(p)
    c = np.ascontiguousarray(c, dtype=p.dtype)
    cc = cfg.c(p.dtype)
    return bool(getattr(lib(), f"orc_within_{_sfx(p)}")(p.ctypes.data, c.ctypes.data, p.shape[0],
                                                        eps, ctypes.byref(cc)))


def import_text(path: str, n: int, dtype=np.float32) -> np.ndarray:
    """importNDDataset restated (import_dataset.cpp:49-95)."""
    s = "f32" if np.dtype(dtype) == np.float32 else "f64"
    f = getattr(lib(), f"orc_import_text_{s}")
    npts = f(path.encode(), n, None, 0)
    if npts < 0:
        raise OSError(f"cannot read {path}")
    out = np.zeros((npts, n), dtype=dtype)
    f(path.encode(), n, out.ctypes.data, out.size)
    return out


def ref_batch_plan(points: np.ndarray, eps: float, cfg: OracleConfig, ref_counts: np.ndarray,
                   sample_counts: np.ndarray, query_reorder: bool, alpha: float = 0.05):
    """The reference's sampled batch plan (GPU.cu:57-268): returns
    (estimate, numBatches, GPUBufferSize, largest per-batch result count)."""
    p = _prep(points).astype(np.float32, copy=False)
    N, n = p.shape
    rc = np.ascontiguousarray(ref_counts, dtype=np.uint32)
    sc = np.ascontiguousarray(sample_counts, dtype=np.uint32)
    est = ctypes.c_uint64()
    nb = ctypes.c_uint32()
    bs = ctypes.c_uint32()
    mx = ctypes.c_uint64()
    c = cfg.c(np.float32)
    lib().orc_ref_batch_plan_f32(p.ctypes.data, N, n, eps, ctypes.byref(c), rc.ctypes.data,
                                 sc.ctypes.data, int(query_reorder), alpha, ctypes.byref(est),
                                 ctypes.byref(nb), ctypes.byref(bs), ctypes.byref(mx))
    return int(est.value), int(nb.value), int(bs.value), int(mx.value)


def join_sample(points: np.ndarray, eps: float, cfg: OracleConfig, queries: np.ndarray):
    """Oracle grid join of a query sample: (pairs, index seconds, query seconds)."""
    p = _prep(points).astype(np.float32, copy=False)
    N, n = p.shape
    q = np.ascontiguousarray(queries, dtype=np.uint32)
    tot = ctypes.c_uint64()
    si = ctypes.c_double()
    sq = ctypes.c_double()
    c = cfg.c(np.float32)
    lib().orc_join_sample_f32(p.ctypes.data, N, n, eps, ctypes.byref(c), q.ctypes.data, q.size, ctypes.byref(tot),
                              ctypes.byref(si), ctypes.byref(sq))
    return int(tot.value), float(si.value), float(sq.value)


def sample_lists(points: np.ndarray, eps: float, cfg: OracleConfig, queries: np.ndarray):
    """Sorted neighbour lists of the listed queries (full enumeration, the
    configured decision model): (counts uint32[nq], lists uint32[sum]), the
    lists concatenated in the order of `queries`."""
    p = _prep(points)
    N, n = p.shape
    q = np.ascontiguousarray(queries, dtype=np.uint32)
    counts = np.zeros(q.size, dtype=np.uint32)
    tot = ctypes.c_uint64()
    c = cfg.c(p.dtype)
    f = getattr(lib(), f"orc_sample_lists_{_sfx(p)}")
    cap = max(1, 64 * q.size)
    lists = np.zeros(cap, dtype=np.uint32)
    rc = f(p.ctypes.data, N, n, eps, ctypes.byref(c), q.ctypes.data, q.size, counts.ctypes.data, lists.ctypes.data,
           cap, ctypes.byref(tot))
    if rc != 0:
        raise ValueError(f"oracle rejected the configuration (rc={rc})")
    if tot.value > cap:
        cap = int(tot.value)
        lists = np.zeros(cap, dtype=np.uint32)
        f(p.ctypes.data, N, n, eps, ctypes.byref(c), q.ctypes.data, q.size, counts.ctypes.data, lists.ctypes.data,
          cap, ctypes.byref(tot))
    return counts, lists[: int(tot.value)]
