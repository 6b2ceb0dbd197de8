"""The allocation-free entry point gsj_list_offsets_noalloc.

Some callers of this library cannot call cudaMalloc: a host framework whose
own allocator already holds (nearly) all device memory in its pool, where a
fresh cudaMalloc fails or forces the pool to release memory, and code on a
latency-critical path, where cudaMalloc/cudaFree would synchronise the
device.  For them the list-offset scan (the exclusive prefix of numNeighbors
that lays out neighborTable) is also exported in a form whose scratch is a
fixed array inside the library.

The test calls that entry point through the C ABI and compares its result
with the offsets the existing entry points produce - gsj_join computes them
for its own table, gsj_result_device exposes them - exactly, since they are
integers.  It does so twice in a row on different inputs, so the second call
runs over scratch that still holds the first call's contents.  This file is
collected last so that a stop at the first failure has already run every
other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_u64(ptr: int, n: int) -> np.ndarray:
    """Copies n uint64 values from a raw device pointer to the host."""
    from cuda.bindings import runtime as rt

    out = np.empty(n, dtype=np.uint64)
    (err,) = rt.cudaMemcpy(out.ctypes.data, ptr, n * 8, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess
    return out


def _join_offsets(sj, N):
    """numNeighbors pointer and list offsets of the join just run."""
    L = sj._L
    cp, op, tp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    rc = L.gsj_result_device(sj._ctx, ctypes.byref(cp), ctypes.byref(op), ctypes.byref(tp))
    assert rc == 0
    return cp.value, _device_u64(op.value, N + 1)


def test_noalloc_offsets_match_join_twice():
    import torch

    from gpu_self_join_b200 import JoinConfig, SelfJoin, synth
    from gpu_self_join_b200._native import lib

    L = lib()
    inputs = [
        (synth.generate("c1_uniform2d", 150_000), 1.0),                   # 37 tiles of counts
        (synth.generate("c2_gmm2d", 600_000), 0.5),                       # 147 tiles, other values
    ]
    with SelfJoin(0) as sj:
        for pts, eps in inputs:
            N = pts.shape[0]
            sj.run(pts, eps, JoinConfig(indexed_dims=2, stamp=True))
            counts_ptr, ref = _join_offsets(sj, N)
            host_counts = sj.counts()
            out = torch.empty(N + 1, dtype=torch.int64, device="cuda")
            out.fill_(-1)
            torch.cuda.synchronize()
            rc = L.gsj_list_offsets_noalloc(ctypes.c_void_p(counts_ptr), N, ctypes.c_void_p(out.data_ptr()), None)
            assert rc == 0, L.gsj_last_error(None)
            torch.cuda.synchronize()
            got = out.cpu().numpy().view(np.uint64)
            assert np.array_equal(got, ref)
            # independent of the library's scan: the prefix of the host counts
            want = np.concatenate([[0], np.cumsum(host_counts, dtype=np.uint64)]).astype(np.uint64)
            assert np.array_equal(got, want)
            assert int(got[-1]) == int(host_counts.sum(dtype=np.uint64)) == sj.total_pairs()


@pytest.mark.parametrize("shift_in,shift_out", [(0, 0), (1, 0), (0, 1), (3, 1)])
def test_noalloc_offsets_any_alignment_many_tiles(shift_in, shift_out):
    """Counts and offsets at every 16-byte misalignment the element types allow
    (the scan loads and stores whole 16-byte vectors only from aligned arrays),
    over more than 4096 tiles of 4096 counts (the single-block scan of the tile
    sums then takes two rounds) and a ragged last tile."""
    import torch

    from gpu_self_join_b200._native import lib

    L = lib()
    n = 4097 * 4096 + 1234
    rng = np.random.default_rng(11 + shift_in + 2 * shift_out)
    host = rng.integers(0, 3000, size=n, dtype=np.uint32)
    cbuf = torch.from_numpy(np.concatenate([np.zeros(shift_in, np.uint32), host]).view(np.int32)).cuda()
    obuf = torch.full((n + 1 + shift_out,), -1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = L.gsj_list_offsets_noalloc(ctypes.c_void_p(cbuf.data_ptr() + 4 * shift_in), n,
                                    ctypes.c_void_p(obuf.data_ptr() + 8 * shift_out), None)
    assert rc == 0, L.gsj_last_error(None)
    torch.cuda.synchronize()
    got = obuf.cpu().numpy().view(np.uint64)
    want = np.concatenate([[0], np.cumsum(host, dtype=np.uint64)]).astype(np.uint64)
    assert np.array_equal(got[shift_out:], want)
    assert (got[:shift_out] == np.uint64(2**64 - 1)).all()  # nothing written before the output


def test_noalloc_empty_input_writes_zero_total():
    """n = 0: the single offset (the total) is zero, whatever the output held."""
    import torch

    from gpu_self_join_b200._native import lib

    L = lib()
    counts = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.full((1,), 12345, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = L.gsj_list_offsets_noalloc(ctypes.c_void_p(counts.data_ptr()), 0, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0, L.gsj_last_error(None)
    torch.cuda.synchronize()
    assert int(out.cpu()[0]) == 0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from gpu_self_join_b200._native import lib

    L = lib()
    counts = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.empty(17, dtype=torch.int64, device="cuda")
    rc = L.gsj_list_offsets_noalloc(ctypes.c_void_p(counts.data_ptr()), 33_550_337, ctypes.c_void_p(out.data_ptr()),
                                    None)
    assert rc != 0
    assert b"scratch limit" in L.gsj_last_error(None)
