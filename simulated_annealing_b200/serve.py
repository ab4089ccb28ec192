"""Serving engine (sa_serve_* in include/sa_b200_batch.h) from Python.

A ``Server`` runs anneal requests with continuous batching: requests are
admitted while the device pools (sized from a memory budget) have room, every
``step(nsweeps)`` advances all admitted requests in one set of kernel launches,
and finished requests are collected with ``poll()`` / ``result()``. Each
request's result depends only on its own parameters (lattice, L, seeds,
schedule), so it is the same whether it ran alone or beside others.

The per-request computation is the reference's annealing<gpu_sys>
(src/annealing.hpp:20-60): one temperature per step of ``sweeps_per_step``
sweeps, -H measured after every sweep and its running maximum kept.
"""
from __future__ import annotations

import ctypes
import heapq
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check
from .batch import LATTICE

_c = ctypes
_vp = _c.c_void_p
_i64p = _c.POINTER(_c.c_int64)
_u64p = _c.POINTER(_c.c_uint64)
_f64p = _c.POINTER(_c.c_double)

for _name, _res, _args in [
    ("sa_serve_create", _c.c_int, [_c.c_size_t, _c.c_int, _c.POINTER(_vp)]),
    ("sa_serve_destroy", _c.c_int, [_vp]),
    ("sa_serve_set_stream", _c.c_int, [_vp, _vp]),
    ("sa_serve_submit", _c.c_int, [_vp, _c.c_int, _c.c_int, _c.c_uint64, _c.c_uint64, _f64p, _c.c_int,
                                   _c.c_int, _i64p]),
    ("sa_serve_run", _c.c_int, [_vp, _c.c_long]),
    ("sa_serve_sync", _c.c_int, [_vp]),
    ("sa_serve_poll", _c.c_int, [_vp, _i64p, _c.c_int, _c.POINTER(_c.c_int)]),
    ("sa_serve_result", _c.c_int, [_vp, _c.c_int64, _i64p, _i64p, _u64p]),
    ("sa_serve_active", _c.c_int, [_vp, _c.POINTER(_c.c_int), _c.POINTER(_c.c_longlong)]),
]:
    _lib.register(_name, _res, _args)


@dataclass
class Result:
    emax: np.ndarray   # int64[64]: running max of -H per replica
    elast: np.ndarray  # int64[64]: -H after the last sweep
    spins: np.ndarray | None = None  # uint64[N], row-major


class Server:
    def __init__(self, budget_bytes: int = 1 << 30, max_requests: int = 4096):
        self._lib = _lib.load()
        h = _vp()
        check(self._lib.sa_serve_create(int(budget_bytes), int(max_requests), _c.byref(h)))
        self._h = h
        self._n = {}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.sa_serve_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, lattice, L: int, seed_J: int, seed: int, T, sweeps_per_step: int) -> int | None:
        """Admit a request; None when the pools are full right now."""
        if isinstance(lattice, str):
            lattice = LATTICE[lattice]
        T = np.ascontiguousarray(T, dtype=np.float64)
        rid = _c.c_int64()
        st = self._lib.sa_serve_submit(self._h, int(lattice), int(L), int(seed_J) & (2**64 - 1),
                                       int(seed) & (2**64 - 1), T.ctypes.data_as(_f64p), len(T),
                                       int(sweeps_per_step), _c.byref(rid))
        if st == _lib.SA_ERR_BUDGET:
            return None
        check(st)
        dim = 3 if lattice == _lib.SA_LATTICE_3D else 2
        self._n[rid.value] = L ** dim
        return rid.value

    def step(self, nsweeps: int) -> None:
        check(self._lib.sa_serve_run(self._h, int(nsweeps)))

    def sync(self) -> None:
        check(self._lib.sa_serve_sync(self._h))

    def poll(self, cap: int = 4096) -> list[int]:
        ids = np.zeros(cap, dtype=np.int64)
        n = _c.c_int()
        check(self._lib.sa_serve_poll(self._h, ids.ctypes.data_as(_i64p), cap, _c.byref(n)))
        return ids[: n.value].tolist()

    def result(self, rid: int, spins: bool = False) -> Result:
        emax = np.zeros(64, dtype=np.int64)
        elast = np.zeros(64, dtype=np.int64)
        s = np.zeros(self._n[rid], dtype=np.uint64) if spins else None
        check(self._lib.sa_serve_result(self._h, int(rid), emax.ctypes.data_as(_i64p),
                                        elast.ctypes.data_as(_i64p),
                                        s.ctypes.data_as(_u64p) if spins else None))
        del self._n[rid]
        return Result(emax, elast, s)

    def active(self) -> tuple[int, int]:
        n = _c.c_int()
        f = _c.c_longlong()
        check(self._lib.sa_serve_active(self._h, _c.byref(n), _c.byref(f)))
        return n.value, f.value


@dataclass(order=True)
class Request:
    arrival: float
    lattice: str = field(compare=False)
    L: int = field(compare=False)
    seed_J: int = field(compare=False)
    seed: int = field(compare=False)
    T: np.ndarray = field(compare=False)
    sweeps_per_step: int = field(compare=False)


def poisson_requests(n: int, rate: float, seed: int = 0, lattice: str = "3d", L_range=(8, 32),
                     sweeps_range=(1_000, 100_000), T0: float = 3.0, T1: float = 0.2,
                     sweeps_per_step: int = 100) -> list[Request]:
    """Seeded open-loop arrivals: exponential gaps at `rate` per second, L
    log-uniform (rounded to even), total sweeps log-uniform; each request a
    linear T0 -> T1 schedule in steps of `sweeps_per_step` sweeps."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for k in range(n):
        L = int(round(np.exp(rng.uniform(np.log(L_range[0]), np.log(L_range[1]))) / 2)) * 2
        L = max(L_range[0], min(L_range[1], L))
        sweeps = float(np.exp(rng.uniform(np.log(sweeps_range[0]), np.log(sweeps_range[1]))))
        steps = max(1, int(round(sweeps / sweeps_per_step)))
        T = np.linspace(T0, T1, steps)
        out.append(Request(float(t[k]), lattice, L, 10_000 + k, 20_000 + k, T, sweeps_per_step))
    return out


def run_open_loop(server: Server, requests: list[Request], chunk: int = 100, clock=time.perf_counter):
    """Serves `requests` (sorted by arrival, seconds from start) in real time:
    admits what has arrived and fits, advances everything by `chunk` sweeps,
    collects what finished. Returns per-request latency (seconds from arrival
    to result), the results by index, and the wall time."""
    pending = list(requests)
    heapq.heapify(pending)
    waiting: list[tuple[int, Request]] = []
    index = {id(r): k for k, r in enumerate(requests)}
    live: dict[int, int] = {}
    latency = np.zeros(len(requests))
    results: dict[int, Result] = {}
    t0 = clock()
    while pending or waiting or live:
        now = clock() - t0
        while pending and pending[0].arrival <= now:
            r = heapq.heappop(pending)
            waiting.append((index[id(r)], r))
        while waiting:
            k, r = waiting[0]
            rid = server.submit(r.lattice, r.L, r.seed_J, r.seed, r.T, r.sweeps_per_step)
            if rid is None:
                break
            live[rid] = k
            waiting.pop(0)
        if not live:
            if pending:
                time.sleep(max(0.0, min(pending[0].arrival - (clock() - t0), 0.001)))
            continue
        server.step(chunk)
        done = server.poll()
        if done:
            server.sync()
            t = clock() - t0
            for rid in done:
                k = live.pop(rid)
                results[k] = server.result(rid)
                latency[k] = t - requests[k].arrival
    return latency, results, clock() - t0
