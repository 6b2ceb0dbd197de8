"""Seeded synthetic stand-ins for the five benchmark workloads.

The reference ships one test input (test_dat.txt) and no benchmark data; the
workloads below follow the published shapes, sizes and value distributions of
the benchmark configurations and are generated from a fixed seed
(20261203 + workload index) with numpy's PCG64, so every machine produces the
same float arrays.

    c1_uniform2d     N=100,000   n=2   uniform [0,100)^2, eps=1.0
    c2_gmm2d         N=20M       n=2   64 isotropic Gaussians + 10% uniform background in [0,1000)^2
    c3_gmm6d         N=5M        n=6   32 Gaussians, centres U[0,100)^6, per-dim sigma U[1,6]
    c4_derived18d    N=5M        n=18  8 GMM base features + 10 smooth derived features, standardised
    c5_heavy90d      N=515,345   n=90  12 Gaussian dims (variance log-U[1,100]) + 78 Student-t(3)
                                       dims with a rank-8 factor correlation

eps of workloads 2-5 is chosen so that the mean number of neighbours per
point (self included) is about the target; it was calibrated once on a seeded
0.1% query sample against the full data set (``calibrate_eps``) and is stored
in WORKLOADS.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BASE_SEED = 20261203


@dataclass(frozen=True)
class Workload:
    name: str
    index: int
    N: int
    n: int
    eps: float
    target_mean: float  # mean neighbours per point the eps was calibrated for
    k: int              # NUMINDEXEDDIM
    stamp: bool
    reorder: bool
    ilp: int
    shortcircuit: bool
    query_reorder: bool


WORKLOADS = {
    "c1_uniform2d": Workload("c1_uniform2d", 0, 100_000, 2, 1.0, 32.4, 2, True, False, 0, False, False),
    "c2_gmm2d": Workload("c2_gmm2d", 1, 20_000_000, 2, 0.24630223214626312, 32.0, 2, True, False, 0, False, False),
    "c3_gmm6d": Workload("c3_gmm6d", 2, 5_000_000, 6, 2.0983946323394775, 64.0, 6, True, False, 0, False, False),
    "c4_derived18d": Workload("c4_derived18d", 3, 5_000_000, 18, 0.4803199768066406, 100.0, 6, False, True, 8, True, True),
    "c5_heavy90d": Workload("c5_heavy90d", 4, 515_345, 90, 13.249305725097656, 50.0, 6, False, True, 8, True, True),
}


def _rng(index: int) -> np.random.Generator:
    return np.random.default_rng(BASE_SEED + index)


def gen_c1(N: int = 100_000) -> np.ndarray:
    return _rng(0).uniform(0.0, 100.0, size=(N, 2)).astype(np.float32)


def gen_c2(N: int = 20_000_000) -> np.ndarray:
    rng = _rng(1)
    K = 64
    centres = rng.uniform(0.0, 1000.0, size=(K, 2))
    sigma = rng.uniform(5.0, 40.0, size=K)
    w = rng.dirichlet(np.ones(K))
    n_bg = N // 10
    n_g = N - n_bg
    comp = rng.choice(K, size=n_g, p=w)
    pts = np.empty((N, 2), dtype=np.float32)
    pts[:n_g] = centres[comp] + rng.standard_normal((n_g, 2)) * sigma[comp, None]
    pts[n_g:] = rng.uniform(0.0, 1000.0, size=(n_bg, 2))
    return pts[rng.permutation(N)]


def gen_c3(N: int = 5_000_000) -> np.ndarray:
    rng = _rng(2)
    K, n = 32, 6
    centres = rng.uniform(0.0, 100.0, size=(K, n))
    sigma = rng.uniform(1.0, 6.0, size=(K, n))
    comp = rng.integers(0, K, size=N)
    pts = centres[comp] + rng.standard_normal((N, n)) * sigma[comp]
    return pts.astype(np.float32)


def gen_c4(N: int = 5_000_000) -> np.ndarray:
    rng = _rng(3)
    K, nb = 16, 8
    centres = rng.uniform(-4.0, 4.0, size=(K, nb))
    scales = np.exp(rng.standard_normal((K, nb)))  # log-normal per-dim scales, sigma_log = 1
    comp = rng.integers(0, K, size=N)
    b = centres[comp] + rng.standard_normal((N, nb)) * scales[comp]
    d = np.empty((N, 10))
    d[:, 0] = b[:, 0] * b[:, 1]
    d[:, 1] = b[:, 2] * b[:, 3]
    d[:, 2] = b[:, 4] / (1.0 + np.abs(b[:, 5]))
    d[:, 3] = b[:, 6] / (1.0 + np.abs(b[:, 7]))
    d[:, 4] = np.sqrt(b[:, 0] ** 2 + b[:, 2] ** 2)
    d[:, 5] = np.sqrt(b[:, 1] ** 2 + b[:, 3] ** 2 + b[:, 5] ** 2)
    d[:, 6] = np.sqrt((b[:, 4:8] ** 2).sum(1))
    d[:, 7] = b[:, 0] * b[:, 7]
    d[:, 8] = np.tanh(b[:, 2]) * b[:, 6]
    d[:, 9] = b[:, 1] / (1.0 + b[:, 3] ** 2)
    d += rng.normal(0.0, 0.05, size=d.shape)
    x = np.concatenate([b, d], axis=1)
    x = (x - x.mean(0)) / x.std(0)
    return x.astype(np.float32)


def gen_c5(N: int = 515_345) -> np.ndarray:
    rng = _rng(4)
    var = np.exp(rng.uniform(np.log(1.0), np.log(100.0), size=12))
    g = rng.standard_normal((N, 12)) * np.sqrt(var)
    m = 78
    F = rng.standard_normal((m, 8)) * 0.6
    diag = rng.uniform(0.3, 1.0, size=m)
    z = rng.standard_normal((N, 8)) @ F.T + rng.standard_normal((N, m)) * np.sqrt(diag)
    chi = rng.chisquare(3.0, size=(N, 1))
    t = z / np.sqrt(chi / 3.0)  # multivariate Student-t, nu = 3
    return np.concatenate([g, t], axis=1).astype(np.float32)


def gen_heavy(N: int, n: int, seed: int) -> np.ndarray:
    """The 90-D workload's distribution at another dimensionality: the first
    min(12, n) dims Gaussian with variances log-U[1,100], the rest
    multivariate Student-t (nu = 3) with a low-rank (<= 8) factor correlation
    plus diagonal."""
    rng = np.random.default_rng(seed)
    ng = min(12, n)
    var = np.exp(rng.uniform(np.log(1.0), np.log(100.0), size=ng))
    g = rng.standard_normal((N, ng)) * np.sqrt(var)
    m = n - ng
    if m == 0:
        return g.astype(np.float32)
    r = min(8, m)
    F = rng.standard_normal((m, r)) * 0.6
    diag = rng.uniform(0.3, 1.0, size=m)
    z = rng.standard_normal((N, r)) @ F.T + rng.standard_normal((N, m)) * np.sqrt(diag)
    chi = rng.chisquare(3.0, size=(N, 1))
    return np.concatenate([g, z / np.sqrt(chi / 3.0)], axis=1).astype(np.float32)


@dataclass(frozen=True)
class Request:
    index: int
    N: int
    n: int
    target_mean: float  # mean neighbours per point the request's eps is chosen for
    seed: int


def request_stream(count: int = 256) -> list[Request]:
    """The 90-D workload's second phase: `count` independent self-joins, N
    log-uniform in [10k, 500k], n from {8, 16, 32, 90}, a target of 10-100
    mean neighbours each (seed BASE_SEED + 5)."""
    rng = np.random.default_rng(BASE_SEED + 5)
    out = []
    for i in range(count):
        N = int(round(np.exp(rng.uniform(np.log(10_000), np.log(500_000)))))
        n = int(rng.choice([8, 16, 32, 90]))
        target = float(rng.uniform(10.0, 100.0))
        out.append(Request(i, N, n, target, int(rng.integers(0, 2**31 - 1))))
    return out


GENERATORS = {"c1_uniform2d": gen_c1, "c2_gmm2d": gen_c2, "c3_gmm6d": gen_c3, "c4_derived18d": gen_c4,
              "c5_heavy90d": gen_c5}


def generate(name: str, N: int | None = None) -> np.ndarray:
    gen = GENERATORS[name]
    return gen() if N is None else gen(N)


def mean_neighbours(points: np.ndarray, eps: float, sample: int, seed: int) -> float:
    """Mean neighbours (self included) of a seeded query sample, by brute
    force in float64 chunks (used only to calibrate eps)."""
    rng = np.random.default_rng(seed)
    q = points[rng.choice(points.shape[0], size=sample, replace=False)].astype(np.float64)
    P = points.astype(np.float32)
    tot = 0
    e2 = eps * eps
    for i in range(0, sample, 64):
        qq = q[i:i + 64].astype(np.float32)
        d2 = (P * P).sum(1)[None, :] - 2.0 * (qq @ P.T) + (qq * qq).sum(1)[:, None]
        tot += int((d2 <= e2).sum())
    return tot / sample


def calibrate_eps(name: str, points: np.ndarray | None = None, frac: float = 0.001, iters: int = 30) -> float:
    """Bisects eps so that the sampled mean neighbour count hits the target."""
    w = WORKLOADS[name]
    pts = generate(name) if points is None else points
    sample = max(64, int(round(pts.shape[0] * frac)))
    try:
        from scipy.spatial import cKDTree

        rng = np.random.default_rng(BASE_SEED + 100 + w.index)
        q = pts[rng.choice(pts.shape[0], size=sample, replace=False)]
        tree = cKDTree(pts)

        def mean_at(e: float) -> float:
            return float(np.mean(tree.query_ball_point(q, e, return_length=True)))
    except ImportError:  # pragma: no cover
        def mean_at(e: float) -> float:
            return mean_neighbours(pts, e, sample, BASE_SEED + 100 + w.index)

    lo, hi = 0.0, 1.0
    while mean_at(hi) < w.target_mean:
        hi *= 2.0
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        if mean_at(mid) < w.target_mean:
            lo = mid
        else:
            hi = mid
    return float(np.float32(hi))
