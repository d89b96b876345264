"""FP64 finite differences and dense-operator columns of the cage-fitting loss.

TEST INFRASTRUCTURE ONLY: the checker of the CUDA adjoint on the fitting
workload at its full depth (2000-face mixed cage, depth 5; about 580 FP64
forwards).  Every forward is the FP64 oracle's scatter rule
(``oracle.refine_points`` with ``real=float64``: CatmullClark.h:1437-1991 and
:2032-2615 in double) on the cage's refined topology.  The forwards run in a
pool of worker processes started with the ``spawn`` method (no process is
forked from one that has used a GPU); each worker builds the workload, the
topology, the fitting target and the FP64 residual once.

The loss is L(x) = mean ||P_D(x) - T||^2 over the finest level's points, with
T = P_D(x0 + N(0, sigma^2)) in FP64.  It is quadratic in x, so a central
difference is exact up to rounding; the dense-operator gradient of entry
(v, k) is (2 / N) <S e_(v,k), P_D(x0) - T>, with the column S e_(v,k) of the
linear refinement operator streamed as one FP64 forward of a basis vector.
"""
from __future__ import annotations

import concurrent.futures as cf
import multiprocessing as mp
import os

import numpy as np

_W = {}


def _setup(depth: int, seed: int, sigma: float):
    from halfedgecatmullclark_b200 import configs
    from oracle import oracle
    w = configs.fitting_cage(depth=depth)
    he, cr = oracle.refine_topology(w.cage, w.depth)
    sl = oracle.level_slice(w.cage, w.depth, w.depth, "V")
    x0 = w.cage.vertex_points.astype(np.float64)
    rng = np.random.default_rng(seed)

    def fwd(x):
        return oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float64, cage_points=x)[sl]
    target = fwd(x0 + rng.normal(0.0, sigma, x0.shape))
    _W.update(w=w, fwd=fwd, x0=x0, target=target, resid=fwd(x0) - target, n=target.size)


def _init(depth, seed, sigma):
    _setup(depth, seed, sigma)


def _loss(x) -> float:
    return float(np.mean((_W["fwd"](x) - _W["target"]) ** 2))


def _task(job):
    kind, v, k, h = job
    x = _W["x0"]
    if kind == "fd":
        xp, xm = x.copy(), x.copy()
        xp[v, k] += h
        xm[v, k] -= h
        return (_loss(xp) - _loss(xm)) / (2.0 * h)
    e = np.zeros_like(x)
    e[v, k] = 1.0
    col = _W["fwd"](e)
    return 2.0 / _W["n"] * float(np.sum(col * _W["resid"]))


def target(depth: int = 5, seed: int = 0, sigma: float = 0.05) -> np.ndarray:
    """The FP64 fitting target T (finest level) the workers use."""
    _setup(depth, seed, sigma)
    return _W["target"]


def check_gradient(verts, depth: int = 5, seed: int = 0, sigma: float = 0.05, h: float = 1e-6,
                   processes: int | None = None):
    """FP64 central differences (step h) and dense-operator gradients of the
    fitting loss at cage vertices `verts` (all three coordinates each).
    Returns (fd, dense), both of shape (len(verts), 3)."""
    verts = [int(v) for v in verts]
    jobs = [("fd", v, k, h) for v in verts for k in range(3)] + [("dense", v, k, 0.0) for v in verts for k in range(3)]
    n = processes or max(1, min(len(jobs), os.cpu_count() or 1))
    # a worker that fails to start ends the map with BrokenProcessPool (a
    # multiprocessing.Pool would start new workers for ever)
    with cf.ProcessPoolExecutor(n, mp_context=mp.get_context("spawn"), initializer=_init,
                                initargs=(depth, seed, sigma)) as pool:
        out = list(pool.map(_task, jobs, chunksize=max(1, len(jobs) // (4 * n))))
    m = 3 * len(verts)
    return np.array(out[:m]).reshape(-1, 3), np.array(out[m:]).reshape(-1, 3)
