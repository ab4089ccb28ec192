"""The reference's drivers over GpuSystem, as Python classes.

ParallelTempering mirrors parallel_tempering<system> (src/parallel_tempering.hpp)
and Annealing mirrors annealing<system> (src/annealing.hpp): same constructor
arguments, step() semantics, exchange generator (std::mt19937(123), drawn by
the library's sa_pt_sequence) and exchange test (sa_pt_mask). With GpuSystem
slots this is the plain one-system-per-launch form: every sweep of every slot
is two kernel launches and every measurement is a device->host copy; the
batched engine (simulated_annealing_b200.batch) runs the same schedule in one
persistent launch.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check

PRINT_E, PRINT_MIN = 0, 1


class ParallelTempering:
    def __init__(self, systems, T, steps: int = 1):
        if len(systems) != len(T):
            raise ValueError("one temperature per system")
        self.sys = list(systems)
        self.T = sorted(float(t) for t in T)
        self.steps = int(steps)
        self.E = [None] * len(self.T)
        self.E_min = None
        self.acc_sum = np.zeros(len(self.T) - 1)
        self.acc_n = np.zeros(len(self.T) - 1, dtype=np.int64)
        self._k = 0  # exchange attempts so far (position in the generator's sequence)
        self._lib = _lib.load()
        for s, t in zip(self.sys, self.T):
            s.set_T(t)

    def _next_pair(self):
        pair = np.zeros(1, dtype=np.int32)
        r = np.zeros(1, dtype=np.float64)
        check(self._lib.sa_pt_sequence(len(self.T), self._k, 1, pair.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                       r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        self._k += 1
        return int(pair[0]), float(r[0])

    def step(self, stride: int = 0):
        """`steps` sweeps of every slot, measurement, then one exchange attempt.
        Returns (pair, mask)."""
        n = len(self.T)
        for i in range(self.steps):
            for j in range(n):
                self.sys[j].sweep()
                if (stride != 0 and i % stride == 0) or i == self.steps - 1:
                    self.E[j] = np.asarray(self.sys[j].measure(), dtype=np.float32)
            if stride == 0:
                e0 = self.E[0]
                self.E_min = e0.copy() if self.E_min is None else np.maximum(self.E_min, e0)
        i, r = self._next_pair()
        Ei = np.ascontiguousarray(self.E[i], dtype=np.float32)
        Ej = np.ascontiguousarray(self.E[i + 1], dtype=np.float32)
        mask = int(self._lib.sa_pt_mask(Ei.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                        Ej.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                        self.T[i], self.T[i + 1], r))
        self.acc_sum[i] += bin(mask).count("1") / 64.0
        self.acc_n[i] += 1
        self.sys[i].swap(self.sys[i + 1], mask)
        return i, mask

    def acceptance(self) -> np.ndarray:
        return np.where(self.acc_n > 0, self.acc_sum / np.maximum(self.acc_n, 1), 0.0)


class Annealing:
    """annealing<system>: step(stride) = `steps` sweeps with a measurement every
    `stride`, running max of -H (min_E), then T *= alfa (or the next entry of an
    explicit schedule)."""

    def __init__(self, T_s: float, steps: int, alfa: float, system, schedule=None):
        self.T = float(T_s)
        self.steps = int(steps)
        self.alfa = float(alfa)
        self.sys = system
        self.schedule = list(schedule) if schedule is not None else None
        self._k = 0
        self.min_E = None
        self.result = None
        self.sys.set_T(self.T)

    def step(self, stride: int = 1):
        for i in range(self.steps):
            self.sys.sweep()
            if stride != 0 and i % stride == 0:
                self.result = np.asarray(self.sys.measure(), dtype=np.float32)
                self.min_E = self.result.copy() if self.min_E is None else np.maximum(self.min_E, self.result)
        self._k += 1
        if self.schedule is not None:
            self.T = self.schedule[min(self._k, len(self.schedule) - 1)]
        else:
            self.T = self.T * self.alfa
        self.sys.set_T(self.T)
