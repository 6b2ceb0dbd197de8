"""ctypes binding of libgpuselfjoin.so (include/gpuselfjoin.h).

The library is built in-tree (``python -m gpu_self_join_b200.build``).  There
is no fallback: when the shared library is missing or cannot be loaded, every
entry point raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpuselfjoin.so")

GSJ_OK = 0
GSJ_FLOAT32 = 0
GSJ_FLOAT64 = 1
GSJ_FLAG_SORT_LISTS = 0x1
GSJ_FLAG_QUIET = 0x2
GSJ_FLAG_NO_UNICOMP = 0x4
GSJ_FLAG_PLAIN = 0x8
GSJ_FLAG_EXACT_SIZE = 0x10
GSJ_EST_SAMPLED = 0
GSJ_EST_LEARNED = 1
GSJ_ERR_OVERFLOW = -5

# Every symbol declared in include/gpuselfjoin.h.
EXPORTED_SYMBOLS = (
    "gsj_default_config", "gsj_set_default_config", "gsj_create", "gsj_destroy", "gsj_join",
    "gsj_result_size", "gsj_result_counts", "gsj_result_table", "gsj_result_device", "gsj_last_error",
    "gsj_threshold_f32", "gsj_threshold_f64", "GDSJoinPy", "copyResultIntoPythonArray", "GDSJoinPy_f32",
    "GDSJoinPy_f64", "copyResultIntoPythonArray64", "gsj_list_offsets_noalloc", "gsj_bruteforce_count",
    "gsj_join_host", "gsj_model_train", "gsj_model_reset", "gsj_model_weights", "gsj_model_features",
    "gsj_model_predict", "gsj_model_loss_grad", "gsj_autotune", "gsj_tuning_get", "gsj_tuning_set",
)
MODEL_WEIGHTS = 3201
MODEL_FEATURES = 16


class GsjConfig(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_uint32),
        ("indexed_dims", ctypes.c_uint32),
        ("dtype", ctypes.c_uint32),
        ("reorder", ctypes.c_uint32),
        ("shortcircuit", ctypes.c_uint32),
        ("ilp", ctypes.c_uint32),
        ("stamp", ctypes.c_uint32),
        ("query_reorder", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
        ("buffer_pairs", ctypes.c_uint64),
        ("streams", ctypes.c_uint32),
        ("min_batches", ctypes.c_uint32),
        ("estimator", ctypes.c_uint32),
        ("sort", ctypes.c_uint32),
    ]


class GsjStats(ctypes.Structure):
    _fields_ = [
        ("num_points", ctypes.c_uint64),
        ("total_pairs", ctypes.c_uint64),
        ("candidates", ctypes.c_uint64),
        ("total_cells", ctypes.c_uint64),
        ("nonempty_cells", ctypes.c_uint64),
        ("work_items", ctypes.c_uint64),
        ("ms_h2d", ctypes.c_double),
        ("ms_index", ctypes.c_double),
        ("ms_join", ctypes.c_double),
        ("ms_d2h", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("dev_ms_index", ctypes.c_double),
        ("dev_ms_count", ctypes.c_double),
        ("dev_ms_fill", ctypes.c_double),
        ("kernel_launches", ctypes.c_uint64),
        ("join_path", ctypes.c_uint64),
        ("screen_rechecks", ctypes.c_uint64),
        ("reruns", ctypes.c_uint64),
        ("batches", ctypes.c_uint64),
        ("tuned", ctypes.c_uint64),
        ("density_log2", ctypes.c_uint64),
        ("estimate", ctypes.c_uint64),
        ("dev_ms_estimate", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class GsjTuning(ctypes.Structure):
    _fields_ = [
        ("threads", ctypes.c_uint32),
        ("warps", ctypes.c_uint32),
        ("ctas_per_sm", ctypes.c_uint32),
        ("streams", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class GsjError(RuntimeError):
    pass


_lib = None


def lib() -> ctypes.CDLL:
    """Loads the in-tree native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GsjError(f"{LIB_PATH} not found: build it with `python -m gpu_self_join_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P, u32, u64, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
    L.gsj_default_config.argtypes = [ctypes.POINTER(GsjConfig)]
    L.gsj_default_config.restype = None
    L.gsj_set_default_config.argtypes = [ctypes.POINTER(GsjConfig)]
    L.gsj_create.argtypes = [ctypes.POINTER(P), i32]
    L.gsj_destroy.argtypes = [P]
    L.gsj_join.argtypes = [P, P, u64, ctypes.c_double, ctypes.POINTER(GsjConfig), i32, ctypes.POINTER(GsjStats)]
    L.gsj_join_host.argtypes = [P, P, u64, ctypes.c_double, ctypes.POINTER(GsjConfig), i32, P, P, u64,
                                ctypes.POINTER(u64), ctypes.POINTER(GsjStats)]
    L.gsj_result_size.argtypes = [P, ctypes.POINTER(u64)]
    L.gsj_result_counts.argtypes = [P, P, i32]
    L.gsj_result_table.argtypes = [P, P, u64, i32]
    L.gsj_result_device.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P)]
    L.gsj_last_error.argtypes = [P]
    L.gsj_last_error.restype = ctypes.c_char_p
    L.gsj_threshold_f32.argtypes = [ctypes.c_float]
    L.gsj_threshold_f32.restype = ctypes.c_float
    L.gsj_threshold_f64.argtypes = [ctypes.c_double]
    L.gsj_threshold_f64.restype = ctypes.c_double
    L.GDSJoinPy_f32.argtypes = [P, ctypes.c_uint, ctypes.c_float, ctypes.c_uint, i32, P]
    L.GDSJoinPy_f64.argtypes = [P, ctypes.c_uint, ctypes.c_double, ctypes.c_uint, i32, P]
    L.copyResultIntoPythonArray64.argtypes = [P, u64]
    L.gsj_list_offsets_noalloc.argtypes = [P, u64, P, P]
    L.gsj_bruteforce_count.argtypes = [P, P, u64, ctypes.c_double, ctypes.POINTER(GsjConfig), i32, P,
                                       ctypes.POINTER(u64)]
    L.gsj_autotune.argtypes = [P, P, u64, ctypes.c_double, ctypes.POINTER(GsjConfig), i32, u32,
                               ctypes.POINTER(GsjTuning)]
    L.gsj_tuning_get.argtypes = [P, u32, u32, u32, ctypes.POINTER(GsjTuning)]
    L.gsj_tuning_set.argtypes = [P, u32, u32, u32, ctypes.POINTER(GsjTuning)]
    L.gsj_model_train.argtypes = [P, u32, P]
    L.gsj_model_reset.argtypes = [P]
    L.gsj_model_weights.argtypes = [P, P, u32, i32]
    L.gsj_model_features.argtypes = [P, P, P, u32, ctypes.POINTER(u32)]
    L.gsj_model_predict.argtypes = [P, P, u32, P]
    L.gsj_model_loss_grad.argtypes = [P, P, P, u32, P, P]
    L.copyResultIntoPythonArray.argtypes = [P, ctypes.c_uint]
    L.copyResultIntoPythonArray.restype = None
    L.GDSJoinPy.restype = None
    _lib = L
    return L


def check(rc: int, ctx=None) -> None:
    if rc != GSJ_OK:
        msg = lib().gsj_last_error(ctx)
        raise GsjError(f"gpuselfjoin error {rc}: {msg.decode() if msg else ''}")


def default_config() -> GsjConfig:
    c = GsjConfig()
    lib().gsj_default_config(ctypes.byref(c))
    return c
