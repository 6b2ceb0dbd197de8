"""Python interface of the self-join, call-compatible with the reference's
gdsjoingpu.py (gdsjoingpu.py:146-232 of mgowanlock/gpu_self_join).

    numNeighbors, neighborTable = gdsjoin(dataset, epsilon, numdim, dtype, verbose)

``dataset`` is the flattened row-major data (a list or any array, length
N * numdim), ``dtype`` is "float" or "double" (the reference's DTYPE).  The
result is ``numNeighbors`` (uint32[N]) and ``neighborTable`` (uint32[R]), the
neighbour lists concatenated in point-id order - exactly the reference's
output format.  The two-phase native protocol is the reference's as well:
GDSJoinPy fills numNeighbors, then copyResultIntoPythonArray copies the table
into the array allocated here (main.cu:360-511).  Differences from the shipped
wrapper: the device ordinal is passed (the reference's wrapper passes 5 of
GDSJoinPy's 6 arguments, gdsjoingpu.py:205-214 vs main.cu:360), numpy 2 is
supported (np.asfarray is gone), failures raise instead of exiting.
"""

from __future__ import annotations

import os
import sys
from contextlib import contextmanager

import numpy as np

from . import _native as N


@contextmanager
def _hide_stdout():
    """Silences C-level stdout (the reference's HideOutput, gdsjoingpu.py:95-119)."""
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    try:
        os.dup2(devnull, 1)
        yield
    finally:
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)


def gdsjoin(DATASET, EPSILON, NDIM, DTYPE, verbose=False, device=0):
    """Self-join of DATASET (flattened N x NDIM) with distance EPSILON.

    Returns (numNeighbors uint32[N], neighborTable uint32[sum(numNeighbors)]).
    """
    if verbose:
        return gdsjoinmain(DATASET, EPSILON, NDIM, DTYPE, device)
    with _hide_stdout():
        return gdsjoinmain(DATASET, EPSILON, NDIM, DTYPE, device)


def gdsjoinmain(DATASET, EPSILON, NDIM, DTYPE, device=0):
    L = N.lib()
    if DTYPE == "float":
        np_t, fn = np.float32, L.GDSJoinPy_f32
    elif DTYPE == "double":
        np_t, fn = np.float64, L.GDSJoinPy_f64
    else:
        raise ValueError('DTYPE must be "float" or "double"')
    NDIM = int(NDIM)
    data = np.ascontiguousarray(np.asarray(DATASET, dtype=np_t).reshape(-1))
    numPoints = data.size // NDIM
    data = data[: numPoints * NDIM]
    numNeighbors = np.zeros(numPoints, dtype=np.uint32)
    N.check(fn(data.ctypes.data, numPoints, EPSILON, NDIM, int(device), numNeighbors.ctypes.data))
    resultSetSize = int(numNeighbors.sum(dtype=np.uint64))
    neighborTable = np.zeros(resultSetSize, dtype=np.uint32)
    N.check(L.copyResultIntoPythonArray64(neighborTable.ctypes.data, resultSetSize))
    return numNeighbors, neighborTable
