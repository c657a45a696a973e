"""ctypes front end of the FP64 C restatement (oracle/esp_oracle.c).

Test infrastructure only: the timed CPU baseline of bench.py and a second,
compiled oracle checked against the numpy one (oracle/esp_ref.py). Systems
run in parallel on OpenMP threads, one system per thread; each runs a
neighbour list, one evaluation and `nsteps` NVE steps.
"""
from __future__ import annotations

import ctypes
import math
import os
from typing import List, Sequence

import numpy as np

from esp_hoomd_b200 import tables
from oracle import esp_ref as R

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "libesp_oracle.so")
_lib = None

# kappa_N = pi r_c / h needed for a 1e-5 relative RMS force error (the
# library's planning table at that target)
KAPPA_1E5 = 18.5


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise ImportError("oracle/libesp_oracle.so not built: run `make -C oracle port`")
        L = ctypes.CDLL(LIB)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.esp_oracle_run_batch.argtypes = [I, P, P, P, P, P, P, P, P, P, P, P, I, I, P, I, P, D, D, D, D, I, D, P, I]
        L.esp_oracle_run_batch.restype = I
        L.esp_oracle_max_threads.restype = I
        _lib = L
    return _lib


def max_threads() -> int:
    return int(lib().esp_oracle_max_threads())


def plan(systems: Sequence, rcut: float, P: int = 8, kappa: float = KAPPA_1E5) -> List[tables.ESPParams]:
    """Per-system parameters of the library's rule: mesh = smallest
    2/3/5-smooth n >= L / h with h = pi r_c / kappa_N, one split
    c = 0.93 kappa_N (rounded to 0.5) for all, window c_w = 2.2 P."""
    h = math.pi * rcut / kappa
    c = round(2 * 0.93 * kappa) * 0.5
    split = tables.split_cached(c)
    window = tables.window_cached(P, 2.2 * P, max(P + 2, 9))
    out = []
    for s in systems:
        mesh = tuple(tables.smooth235(max(P, int(math.ceil(L / h)))) for L in s.box)
        out.append(tables.ESPParams(mesh=mesh, box=s.box, rcut=rcut, split=split, window=window))
    return out


def _gkey(p: tables.ESPParams):
    return (tuple(p.box), tuple(p.mesh), id(p.split), id(p.window), p.rcut)


def influence_tables(params: Sequence[tables.ESPParams], cache=None) -> dict:
    """Influence tables (numpy FP64) of every distinct (box, mesh), keyed as
    run_batch's cache."""
    cache = {} if cache is None else cache
    for p in params:
        if _gkey(p) not in cache:
            cache[_gkey(p)] = np.ascontiguousarray(R.influence(p), dtype=np.float64)
    return cache


def run_batch(systems: Sequence, params: Sequence[tables.ESPParams], rlist: float, nsteps: int, dt: float,
              threads: int = 0, influence_cache=None):
    """Runs every system (neighbour list + evaluation + nsteps NVE steps) in
    FP64 and returns (positions [list], velocities, forces, energies). The
    influence tables are built first (numpy) and are not part of the run."""
    split, window, rcut = params[0].split, params[0].window, params[0].rcut
    for p in params:
        if p.split is not split or p.window is not window or p.rcut != rcut:
            raise ValueError("systems of one batch share split, window and cutoff")
    cache = {} if influence_cache is None else influence_cache
    Ns = np.array([s.N for s in systems], dtype=np.int32)
    p_off = np.concatenate([[0], np.cumsum(Ns)[:-1]]).astype(np.int64)
    pos = np.ascontiguousarray(np.concatenate([s.pos for s in systems]), dtype=np.float64)
    vel = np.ascontiguousarray(np.concatenate([s.vel for s in systems]), dtype=np.float64)
    mass = np.ascontiguousarray(np.concatenate([s.mass for s in systems]), dtype=np.float64)
    q = np.ascontiguousarray(np.concatenate([s.q for s in systems]), dtype=np.float64)
    F = np.zeros_like(pos)
    boxes = np.ascontiguousarray([p.box for p in params], dtype=np.float64)
    meshes = np.ascontiguousarray([p.mesh for p in params], dtype=np.int32)
    Gs, g_off, o = [], [], 0
    influence_tables(params, cache)
    for p in params:
        key = _gkey(p)
        Gs.append(cache[key])
        g_off.append(o)
        o += cache[key].size
    G = np.ascontiguousarray(np.concatenate([g.ravel() for g in Gs]))
    g_off = np.array(g_off, dtype=np.int64)
    wcoef = np.ascontiguousarray(window.coef, dtype=np.float64)
    qv = np.ascontiguousarray(split.qv, dtype=np.float64)
    energy = np.zeros(len(systems))
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = lib().esp_oracle_run_batch(len(systems), ptr(Ns), ptr(p_off), ptr(pos), ptr(vel), ptr(mass), ptr(q), ptr(F),
                                    ptr(boxes), ptr(meshes), ptr(g_off), ptr(G), window.P, wcoef.shape[1] - 1,
                                    ptr(wcoef), qv.size, ptr(qv), float(split.lambda0), float(split.m2), float(rcut),
                                    float(rlist), int(nsteps), float(dt), ptr(energy), int(threads))
    if rc != 0:
        raise RuntimeError("esp_oracle_run_batch failed")
    split_at = np.cumsum(Ns)[:-1]
    return np.split(pos, split_at), np.split(vel, split_at), np.split(F, split_at), energy
