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
import struct

import numpy as np

from . import _lib
from ._lib import check

PRINT_E, PRINT_MIN = 0, 1


for _name, _res, _args in [
    ("sa_pt_gen_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("sa_pt_gen_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("sa_pt_gen_next", ctypes.c_int, [ctypes.c_void_p, ctypes.c_long, ctypes.POINTER(ctypes.c_int32),
                                      ctypes.POINTER(ctypes.c_double)]),
    ("sa_pt_gen_widen", ctypes.c_int, [ctypes.c_void_p]),
    ("sa_pt_gen_save", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.POINTER(ctypes.c_size_t)]),
    ("sa_pt_gen_load", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
]:
    _lib.register(_name, _res, _args)


def _cpp_float(x: float) -> str:
    """A float as std::ostream writes it by default (6 significant digits)."""
    return "%g" % x


def _cpp_to_string(x: float) -> str:
    """std::to_string(double): %f."""
    return "%f" % x


class ParallelTempering:
    """parallel_tempering<system> (src/parallel_tempering.hpp:17-52) over
    GpuSystem slots: the same constructor (systems, temperatures -- sorted --,
    sweeps per step, output file name with a '%' placeholder), step(),
    print(), print_swap(), set_info(), reset(), get_E_min(), save(), load()
    and update_T().

    save() returns the template's checkpoint stream, the ".tempsys" files of
    the reference's CLI (src/parallel_tempering.hpp:280-318): steps, the two
    print flags, the exchange generator (std::mt19937 and its two
    distributions, raw), the file name, T, E_min, the acceptance
    accumulators (double sum, long long count), then per slot its last
    energies and its system record. In mt19937_64 mode a slot's record is
    the reference CPU classes' own (cpu_2dp::save / cpu_3d::save), so the
    stream is the one parallel_tempering<cpu_sys> writes and loads; in the
    default Philox mode it is this engine's record with an 8-byte length in
    front (as the C++ gpu_sys shim writes it). load() reads either.

    Two reference defects are kept where they decide results: reset() does
    not clear the acceptance accumulators (accumulator::reset is a no-op,
    src/accumulator.hpp:36-38), and update_T clones the upper system of a
    pair for the inserted temperature (src/parallel_tempering.hpp:394). One
    is not: the reference's load() drops the file name
    (binary_read_string returns before assigning, src/bin_io.cpp:3-8); here
    the name read is kept."""

    def __init__(self, systems, T, steps: int = 1, filename: str = "%"):
        if len(systems) != len(T):
            raise ValueError("one temperature per system")
        self.sys = list(systems)
        self.T = sorted(float(t) for t in T)
        self.steps = int(steps)
        self.fname = str(filename)
        self.E = [np.zeros(0, dtype=np.float32) for _ in self.T]
        self.E_min = np.zeros(0, dtype=np.float32)
        self.acc_sum = [0.0] * (len(self.T) - 1)
        self.acc_n = [0] * (len(self.T) - 1)
        self.print_E = False
        self.print_min = False
        self._files = []
        self._file_min = None
        self._lib = _lib.load()
        g = ctypes.c_void_p()
        check(self._lib.sa_pt_gen_create(len(self.T), ctypes.byref(g)))
        self._gen = g
        for s, t in zip(self.sys, self.T):
            s.set_T(t)

    def __del__(self):
        try:
            if getattr(self, "_gen", None) is not None and self._gen.value:
                self._lib.sa_pt_gen_destroy(self._gen)
                self._gen = ctypes.c_void_p()
            self._close_files()
        except Exception:
            pass

    def _next_pair(self):
        pair = np.zeros(1, dtype=np.int32)
        r = np.zeros(1, dtype=np.float64)
        check(self._lib.sa_pt_gen_next(self._gen, 1, pair.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                       r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return int(pair[0]), float(r[0])

    def step(self, stride: int = 0):
        """`steps` sweeps of every slot with measurements, then one exchange
        attempt (src/parallel_tempering.hpp:81-115). Returns (pair, mask)."""
        n = len(self.T)
        for i in range(self.steps):
            for j in range(n):
                self.sys[j].sweep()
                if (stride != 0 and i % stride == 0) or i == self.steps - 1:
                    self.E[j] = np.asarray(self.sys[j].measure(), dtype=np.float32)
            if stride != 0 and i % stride == 0:
                self.print(PRINT_E)
            elif stride == 0:
                e0 = self.E[0]
                self.E_min = e0.copy() if self.E_min.size == 0 else np.maximum(self.E_min, e0)
        i, r = self._next_pair()
        # one mask word per 64 replicas (src/parallel_tempering.hpp:143-160)
        masks = []
        for w in range(len(self.E[i]) // 64):
            Ei = np.ascontiguousarray(self.E[i][64 * w:64 * w + 64], dtype=np.float32)
            Ej = np.ascontiguousarray(self.E[i + 1][64 * w:64 * w + 64], dtype=np.float32)
            masks.append(int(self._lib.sa_pt_mask(Ei.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                  Ej.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                  self.T[i], self.T[i + 1], r)))
        self.acc_sum[i] += sum(bin(m).count("1") for m in masks) / 64.0
        self.acc_n[i] += 1
        self.sys[i].swap(self.sys[i + 1], masks if len(masks) > 1 else masks[0])
        return i, (masks if len(masks) > 1 else masks[0])

    def acceptance(self) -> np.ndarray:
        """accumulator<double>::get() per pair: the mean accepted fraction."""
        return np.array([s / n if s != 0 else 0.0 for s, n in zip(self.acc_sum, self.acc_n)])

    def get_E_min(self) -> np.ndarray:
        return self.E_min.copy()

    # -- file output (src/parallel_tempering.hpp:118-139, 164-210) -------------
    def _open(self, select, append=False):
        mode = "a" if append else "w"
        if select == PRINT_E and not self.print_E:
            self._files = [open(self.fname.replace("%", "T" + _cpp_to_string(t)), mode) for t in self.T]
            self.print_E = True
        elif select == PRINT_MIN and not self.print_min:
            self._file_min = open(self.fname.replace("%", "E_min"), mode)
            self.print_min = True

    def _close_files(self):
        for f in self._files:
            f.close()
        self._files = []
        if self._file_min is not None:
            self._file_min.close()
            self._file_min = None

    def print(self, select: int) -> None:
        self._open(select)
        if select == PRINT_E:
            for f, e in zip(self._files, self.E):
                f.write("".join(_cpp_float(float(v)) + "\t" for v in e) + "\n")
                f.flush()
        else:
            self._file_min.write("".join(_cpp_float(float(v)) + "\t" for v in self.E_min) + "\n")
            self._file_min.flush()

    def set_info(self, info: str, select: int) -> None:
        self._open(select)
        if select == PRINT_E:
            for f in self._files:
                f.write(info)
        else:
            self._file_min.write(info)

    def print_swap(self) -> str:
        acc = self.acceptance()
        return "".join(f"{_cpp_float(self.T[i])} -> {_cpp_float(self.T[i + 1])}\t: {_cpp_float(acc[i])}\n"
                       for i in range(len(self.T) - 1))

    def reset(self) -> None:
        """E_min to 0, new random spins in every slot; the acceptance
        accumulators stay (the reference's reset of them is a no-op)."""
        self.E_min = np.zeros_like(self.E_min)
        for s in self.sys:
            s.init_rand()

    # -- checkpoints (src/parallel_tempering.hpp:280-377) ----------------------
    def _gen_bytes(self) -> bytes:
        n = ctypes.c_size_t()
        check(self._lib.sa_pt_gen_save(self._gen, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        check(self._lib.sa_pt_gen_save(self._gen, buf, n.value, ctypes.byref(n)))
        return buf.raw[: n.value]

    @staticmethod
    def _record(s) -> bytes:
        return s.checkpoint_record()

    @staticmethod
    def _read_record(s, data: bytes, off: int) -> int:
        return s.read_checkpoint_record(data, off)

    def save(self) -> bytes:
        out = [struct.pack("<q??", self.steps, self.print_E, self.print_min), self._gen_bytes()]
        name = self.fname.encode()
        out.append(struct.pack("<Q", len(name)) + name)
        out.append(struct.pack("<Q", len(self.T)) + np.asarray(self.T, dtype="<f8").tobytes())
        out.append(struct.pack("<Q", self.E_min.size) + np.asarray(self.E_min, dtype="<f4").tobytes())
        out.append(struct.pack("<Q", len(self.acc_sum)))
        out += [struct.pack("<dq", s, n) for s, n in zip(self.acc_sum, self.acc_n)]
        out.append(struct.pack("<Q", len(self.E)))
        for e, s in zip(self.E, self.sys):
            out.append(struct.pack("<Q", e.size) + np.asarray(e, dtype="<f4").tobytes())
            out.append(self._record(s))
        return b"".join(out)

    def load(self, data: bytes) -> None:
        """Reads save()'s stream (or one the reference's template wrote over
        systems of the same kinds) into this driver and its systems; the
        systems must already be in the record's random mode."""
        self._close_files()
        off = 0
        self.steps, pe, pm = struct.unpack_from("<q??", data, off)
        off += 10
        glen = len(self._gen_bytes())
        check(self._lib.sa_pt_gen_load(self._gen, ctypes.create_string_buffer(data[off:off + glen], glen), glen))
        off += glen
        (n,) = struct.unpack_from("<Q", data, off)
        self.fname = data[off + 8:off + 8 + n].decode(errors="replace")
        off += 8 + n
        (n,) = struct.unpack_from("<Q", data, off)
        self.T = np.frombuffer(data, dtype="<f8", count=n, offset=off + 8).tolist()
        off += 8 + 8 * n
        self.print_E = self.print_min = False
        if pe:
            self._open(PRINT_E, append=True)
        if pm:
            self._open(PRINT_MIN, append=True)
        (n,) = struct.unpack_from("<Q", data, off)
        self.E_min = np.frombuffer(data, dtype="<f4", count=n, offset=off + 8).astype(np.float32)
        off += 8 + 4 * n
        (n,) = struct.unpack_from("<Q", data, off)
        off += 8
        self.acc_sum, self.acc_n = [], []
        for _ in range(n):
            a, c = struct.unpack_from("<dq", data, off)
            self.acc_sum.append(a)
            self.acc_n.append(c)
            off += 16
        (n,) = struct.unpack_from("<Q", data, off)
        off += 8
        if n != len(self.sys):
            raise ValueError(f"checkpoint holds {n} systems, the driver has {len(self.sys)}")
        self.E = []
        for s in self.sys:
            (m,) = struct.unpack_from("<Q", data, off)
            self.E.append(np.frombuffer(data, dtype="<f4", count=m, offset=off + 8).astype(np.float32))
            off += 8 + 4 * m
            off = self._read_record(s, data, off)
        if off != len(data):
            raise ValueError("trailing bytes after the checkpoint")

    def update_T(self) -> None:
        """Adaptive temperatures (src/parallel_tempering.hpp:384-413): after
        every pair whose acceptance is below 0.3, insert the mean of its two
        temperatures, carried by a copy of the pair's upper system."""
        i = 0
        while i < len(self.acc_sum):
            acc = self.acc_sum[i] / self.acc_n[i] if self.acc_sum[i] != 0 else 0.0
            if acc < 0.3:
                i += 1
                self.acc_sum.insert(i, 0.0)
                self.acc_n.insert(i, 0)
                self.T.insert(i, (self.T[i] + self.T[i - 1]) / 2.0)
                self.E.insert(i, np.zeros(0, dtype=np.float32))
                self.sys.insert(i, self.sys[i].clone())
                self.sys[i].set_T(self.T[i])
                if self.print_E:
                    self._files.insert(i, open(self.fname.replace("%", "T" + _cpp_to_string(self.T[i])), "w"))
                check(self._lib.sa_pt_gen_widen(self._gen))
            i += 1


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
