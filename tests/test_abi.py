"""CPU tests of the C ABI: the in-tree library loads, exports every symbol
declared in include/gpuselfjoin.h, and its host-side logic (distance
threshold, defaults, error reporting) behaves; no compute calls are made."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpuselfjoin.h")


def _declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^GSJ_API\s+[\w\s\*]*?\b(\w+)\s*\(", txt, re.M)))


def test_header_declares_reference_abi():
    syms = _declared_symbols()
    # the reference's shared-library exports (main.cu:360, main.cu:507)
    assert "GDSJoinPy" in syms and "copyResultIntoPythonArray" in syms
    assert len(syms) >= 17


def test_library_exports_every_declared_symbol():
    from gpu_self_join_b200 import _native

    lib = _native.lib()
    for s in _declared_symbols():
        assert hasattr(lib, s), f"{s} not exported"
    assert set(_native.EXPORTED_SYMBOLS) <= set(_declared_symbols())


def test_no_oracle_in_product():
    # the product path never references the oracle
    for dp, _, fs in os.walk(os.path.join(ROOT, "gpu_self_join_b200")):
        for f in fs:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                assert "oracle" not in open(os.path.join(dp, f)).read().lower().replace("oracle-free", ""), f


@pytest.mark.parametrize("eps", [1.0, 0.5, 0.1, 3.7, 1e-3, 2.5e-38, 1e19, 3e38, 0.0])
def test_threshold_f32_equivalent_to_sqrt_test(eps):
    from gpu_self_join_b200 import _native

    L = _native.lib()
    e = np.float32(eps)
    T = np.float32(L.gsj_threshold_f32(float(e)))
    assert np.sqrt(T) <= e
    nxt = np.nextafter(T, np.float32(np.inf))
    assert not (np.sqrt(nxt) <= e)
    # every float within 2^16 ulps of T, and random floats over the whole range
    bits = T.view(np.uint32).astype(np.int64)
    win = np.arange(max(0, bits - 65536), bits + 65536, dtype=np.int64)
    win = win[win < 0x7F800000].astype(np.uint32).view(np.float32)
    rnd = np.random.default_rng(1).integers(0, 0x7F800000, 200000, dtype=np.uint32).view(np.float32)
    for s in (win, rnd):
        assert np.array_equal(s <= T, np.sqrt(s) <= e)


@pytest.mark.parametrize("eps", [1.0, 0.3, 7.25, 1e-200, 1e200])
def test_threshold_f64(eps):
    from gpu_self_join_b200 import _native

    L = _native.lib()
    T = L.gsj_threshold_f64(eps)
    assert np.sqrt(T) <= eps
    assert not (np.sqrt(np.nextafter(T, np.inf)) <= eps)


def test_threshold_negative_and_nan():
    from gpu_self_join_b200 import _native

    L = _native.lib()
    assert L.gsj_threshold_f32(-1.0) == -np.inf
    assert L.gsj_threshold_f32(float("nan")) == -np.inf
    assert L.gsj_threshold_f32(float("inf")) == np.inf


def test_default_config_and_setter():
    from gpu_self_join_b200 import _native

    c = _native.default_config()
    assert c.indexed_dims >= 1 and c.dtype in (0, 1)
    c2 = _native.GsjConfig()
    ctypes.memmove(ctypes.byref(c2), ctypes.byref(c), ctypes.sizeof(c))
    c2.stamp = 1
    _native.check(_native.lib().gsj_set_default_config(ctypes.byref(c2)))
    assert _native.default_config().stamp == 1
    _native.check(_native.lib().gsj_set_default_config(ctypes.byref(c)))


def test_errors_are_returned_not_fatal():
    from conftest import HAVE_GPU
    from gpu_self_join_b200 import _native

    L = _native.lib()
    ctx = ctypes.c_void_p()
    rc = L.gsj_create(ctypes.byref(ctx), 10_000)
    assert rc != 0
    assert L.gsj_last_error(None)
    if not HAVE_GPU:
        with pytest.raises(_native.GsjError):
            from gpu_self_join_b200 import SelfJoin

            SelfJoin(0)
    # copy without a pending result is a state error, not a crash
    assert L.copyResultIntoPythonArray64(None, 0) == -4
