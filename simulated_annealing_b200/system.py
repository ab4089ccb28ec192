"""GpuSystem: the reference's gpu_sys interface (src/gpu_sys.cuh:12-29) over the C ABI.

Method names, argument meaning and results follow gpu_sys; the work runs in
libsa_b200.so on the GPU. ``measure()`` returns the reference's float vector
(index j = replica bit j); ``measure_exact()`` returns the exact integer parts.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _lib
from ._lib import check

LATTICES = {"2d": _lib.SA_LATTICE_2D, "2p": _lib.SA_LATTICE_2D_OPEN_X, "3d": _lib.SA_LATTICE_3D}


def _p(a: np.ndarray, ct=ctypes.c_uint64):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def read_J_file(fname: str, dim: int, N: int):
    """The reference's J file (load_J_2d / load_J_3d, src/sys_file.cpp:10-35,
    :60-88): int dim; long N; then Jx[2N], Jy[2N] (and Jz[2N]) as raw
    little-endian words, no padding. Raises ValueError where the reference
    returns -1 (cannot open), -2 (other dimension) or -3 (other N)."""
    try:
        f = open(fname, "rb")
    except OSError as e:
        raise ValueError(f"cannot open J file {fname}") from e
    with f:
        head = f.read(12)
        if len(head) < 12:
            raise ValueError(f"J file {fname} is truncated")
        d, n = struct.unpack("<iq", head)
        if d != dim:
            raise ValueError(f"J file is {d}D, system is {dim}D")
        if n != N:
            raise ValueError(f"J file has N={n}, system has N={N}")
        arrs = []
        for _ in range(dim):
            b = f.read(16 * N)
            if len(b) != 16 * N:
                raise ValueError(f"J file {fname} is truncated")
            arrs.append(np.frombuffer(b, dtype="<u8").astype(np.uint64))
    return tuple(arrs)


def write_J_file(fname: str, arrays) -> None:
    """Writes the reference's J file (save_J_2d / save_J_3d,
    src/sys_file.cpp:37-58, :90-110) from the reference-layout couplings."""
    arrays = [np.ascontiguousarray(a, dtype="<u8") for a in arrays]
    N = arrays[0].size // 2
    with open(fname, "wb") as f:
        f.write(struct.pack("<iq", len(arrays), N))
        for a in arrays:
            f.write(a.tobytes())


class GpuSystem:
    """One lattice x 64 replicas on the GPU (gpu_2d / gpu_3d replacement)."""

    def __init__(self, lattice, L: int, T: float = 1.0, h: float = 0.0):
        if isinstance(lattice, str):
            lattice = LATTICES[lattice]
        self._lib = _lib.load()
        self.lattice = int(lattice)
        self.L = int(L)
        self.h = float(h)
        handle = ctypes.c_void_p()
        check(self._lib.sa_sys_create(self.lattice, self.L, float(T), float(h), ctypes.byref(handle)))
        self._h = handle
        n = ctypes.c_long()
        check(self._lib.sa_sys_get_N(self._h, ctypes.byref(n)))
        self.N = int(n.value)
        self.dim = 3 if self.lattice == _lib.SA_LATTICE_3D else 2

    # -- gpu_sys -------------------------------------------------------------
    def sweep(self, n: int = 1) -> None:
        check(self._lib.sa_sys_sweep(self._h, int(n)))

    def set_T(self, T: float) -> None:
        check(self._lib.sa_sys_set_T(self._h, float(T)))

    def get_T(self) -> float:
        t = ctypes.c_double()
        check(self._lib.sa_sys_get_T(self._h, ctypes.byref(t)))
        return t.value

    def set_h(self, h: float) -> None:
        check(self._lib.sa_sys_set_h(self._h, float(h)))
        self.h = float(h)

    def set_seed(self, seed: int) -> None:
        check(self._lib.sa_sys_set_seed(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF))

    def set_rng_mode(self, mode) -> None:
        """'philox' (default: the GPU reference's cuRAND schedule) or 'mt19937_64'
        (the CPU reference's stream, bit-exact with cpu_2d/cpu_2dp/cpu_3d).
        Switching reseeds the generator with the current seed."""
        if isinstance(mode, str):
            mode = {"philox": _lib.SA_RNG_PHILOX, "mt19937_64": _lib.SA_RNG_MT19937_64}[mode]
        check(self._lib.sa_sys_set_rng_mode(self._h, int(mode)))

    def set_first_colour(self, colour: int) -> None:
        """Colour of each sweep's first half-sweep (sa_sys_set_first_colour):
        1 is the second configuration of the reference GPU systems'
        two-lattice pair. Philox mode only."""
        check(self._lib.sa_sys_set_first_colour(self._h, int(colour)))

    def set_split_field(self, on: bool) -> None:
        """The reference's SPLIT_H update: bond and field parts of a flip
        accepted with two draws (sa_sys_set_split_field). Philox mode only."""
        check(self._lib.sa_sys_set_split_field(self._h, int(bool(on))))

    def split_field(self) -> bool:
        c = ctypes.c_int()
        check(self._lib.sa_sys_get_split_field(self._h, ctypes.byref(c)))
        return bool(c.value)

    def first_colour(self) -> int:
        c = ctypes.c_int()
        check(self._lib.sa_sys_get_first_colour(self._h, ctypes.byref(c)))
        return c.value

    def rng_mode(self) -> int:
        m = ctypes.c_int()
        check(self._lib.sa_sys_get_rng_mode(self._h, ctypes.byref(m)))
        return m.value

    def measure(self) -> list[float]:
        out = np.zeros(64, dtype=np.float32)
        check(self._lib.sa_sys_measure_float(self._h, _p(out, ctypes.c_float)))
        return out.tolist()

    def measure_exact(self):
        E = np.zeros(64, dtype=np.int64)
        M = np.zeros(64, dtype=np.int64)
        check(self._lib.sa_sys_measure(self._h, _p(E, ctypes.c_int64), _p(M, ctypes.c_int64)))
        return E, M

    def gpu_free(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.sa_sys_destroy(self._h)
            self._h = ctypes.c_void_p()

    def init_J(self) -> None:
        check(self._lib.sa_sys_init_J(self._h))

    def init_rand(self) -> None:
        check(self._lib.sa_sys_init_rand(self._h))

    def init_order(self) -> None:
        check(self._lib.sa_sys_init_order(self._h))

    def get_N(self) -> int:
        return self.N

    def swap(self, other: "GpuSystem", mask) -> None:
        m = int(mask[0]) if hasattr(mask, "__len__") else int(mask)
        check(self._lib.sa_sys_swap(self._h, other._h, m & 0xFFFFFFFFFFFFFFFF))

    # J files (src/sys_file.cpp:10-110): see read_J_file / write_J_file
    def load_J(self, fname: str) -> None:
        self.set_J(*read_J_file(fname, self.dim, self.N))

    def save_J(self, fname: str) -> None:
        write_J_file(fname, self.get_J())

    def save_sys(self, prefix: str) -> None:
        """PBM image per replica bit (src/gpu_2d.cu:275-299)."""
        s = self.get_spins()
        rows = self.L if self.dim == 2 else self.L * self.L
        for i in range(64):
            bits = ((s >> np.uint64(i)) & np.uint64(1)).astype(np.uint8).reshape(rows, self.L)
            with open(f"{prefix}{i}.pbm", "w") as f:
                f.write(f"P1\n{self.L} {rows}\n")
                for row in bits:
                    f.write("".join("1 " if b else "0 " for b in row) + "\n")

    def save(self) -> bytes:
        n = ctypes.c_size_t()
        check(self._lib.sa_sys_save(self._h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        check(self._lib.sa_sys_save(self._h, buf, n.value, ctypes.byref(n)))
        return buf.raw[: n.value]

    def load(self, data: bytes) -> None:
        buf = ctypes.create_string_buffer(data, len(data))
        check(self._lib.sa_sys_load(self._h, buf, len(data)))

    def clone(self) -> "GpuSystem":
        """A copy of this system (cpu_sys::clone, src/cpu_sys.hpp:30) in a new
        device allocation: same lattice, temperature, field, spins and
        couplings. In mt19937_64 mode the copy's generator is reseeded with
        1234, as the reference's copy constructors do (src/cpu_3d.cpp:47-78,
        src/cpu_2dp.cpp:53-84); in Philox mode it keeps the seed and position.
        (The reference's cpu_2d inherits cpu_2dp::clone and so copies a
        periodic lattice into an open-x one; here the lattice is kept.)"""
        c = GpuSystem(self.lattice, self.L, self.get_T(), self.h)
        if self.rng_mode() == _lib.SA_RNG_MT19937_64:
            c.load_reference(self.save_reference())
            c.set_seed(1234)
        else:
            c.load(self.save())
        return c

    def checkpoint_record(self) -> bytes:
        """The system's part of a parallel-tempering checkpoint: in
        mt19937_64 mode the reference CPU classes' own record (cpu_2dp::save /
        cpu_3d::save), else this engine's record with an 8-byte length in
        front (what the C++ gpu_sys shim writes)."""
        if self.rng_mode() == _lib.SA_RNG_MT19937_64:
            return self.save_reference()
        blob = self.save()
        return struct.pack("<Q", len(blob)) + blob

    def read_checkpoint_record(self, data: bytes, off: int) -> int:
        """Loads checkpoint_record()'s bytes at data[off:]; returns the end."""
        if self.rng_mode() == _lib.SA_RNG_MT19937_64:
            n = len(self.save_reference())
            self.load_reference(data[off:off + n])
            return off + n
        (n,) = struct.unpack_from("<Q", data, off)
        self.load(data[off + 8:off + 8 + n])
        return off + 8 + n

    def save_reference(self) -> bytes:
        """The record cpu_2dp::save / cpu_3d::save write (mt19937_64 mode)."""
        n = ctypes.c_size_t()
        check(self._lib.sa_sys_save_reference(self._h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        check(self._lib.sa_sys_save_reference(self._h, buf, n.value, ctypes.byref(n)))
        return buf.raw[: n.value]

    def load_reference(self, data: bytes) -> None:
        """Load a cpu_2dp / cpu_3d record; switches to mt19937_64 mode."""
        buf = ctypes.create_string_buffer(data, len(data))
        check(self._lib.sa_sys_load_reference(self._h, buf, len(data)))

    def anneal(self, T, sweeps: int, stride: int = 1):
        """annealing<gpu_sys> on the device over the schedule T (one entry per
        step of `sweeps` sweeps). Returns (min_E float[64], step_E int64[nsteps, 64])."""
        T = np.ascontiguousarray(T, dtype=np.float64)
        mn = np.zeros(64, dtype=np.float32)
        stepE = np.zeros((len(T), 64), dtype=np.int64)
        check(self._lib.sa_sys_anneal(self._h, _p(T, ctypes.c_double), len(T), int(sweeps), int(stride),
                                      _p(mn, ctypes.c_float), _p(stepE, ctypes.c_int64)))
        return mn, stepE

    # -- data access -----------------------------------------------------------
    def set_J(self, jx, jy, jz=None) -> None:
        jx = np.ascontiguousarray(jx, dtype=np.uint64)
        jy = np.ascontiguousarray(jy, dtype=np.uint64)
        if self.dim == 3:
            jz = np.ascontiguousarray(jz, dtype=np.uint64)
            check(self._lib.sa_sys_set_J(self._h, _p(jx), _p(jy), _p(jz)))
        else:
            check(self._lib.sa_sys_set_J(self._h, _p(jx), _p(jy), None))

    def get_J(self):
        arrs = [np.zeros(2 * self.N, dtype=np.uint64) for _ in range(self.dim)]
        jz = _p(arrs[2]) if self.dim == 3 else None
        check(self._lib.sa_sys_get_J(self._h, _p(arrs[0]), _p(arrs[1]), jz))
        return tuple(arrs)

    def set_spins(self, s) -> None:
        s = np.ascontiguousarray(s, dtype=np.uint64)
        if s.size != self.N:
            raise ValueError("spin array must have N words")
        check(self._lib.sa_sys_set_spins(self._h, _p(s)))

    def get_spins(self) -> np.ndarray:
        s = np.zeros(self.N, dtype=np.uint64)
        check(self._lib.sa_sys_get_spins(self._h, _p(s)))
        return s

    def rng_state(self):
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        check(self._lib.sa_sys_get_rng(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def set_rng_state(self, seed: int, draw: int, epoch: int) -> None:
        check(self._lib.sa_sys_set_rng(self._h, seed, draw, epoch))

    def sync(self) -> None:
        check(self._lib.sa_sys_sync(self._h))

    def __del__(self):
        try:
            self.gpu_free()
        except Exception:
            pass


class TwoLatticeSystem:
    """The reference GPU systems' own shape (gpu_2d, gpu_3d): 128 replicas per
    system. Their two lattices s1, s2, each updated from the other
    (src/gpu_2d.cu:109-120), carry two configurations: A (s1 on colour-0
    sites, s2 on colour-1 sites), whose sweep updates colour 0 first, and B,
    which updates colour 1 first. Here they are two GpuSystem objects with the
    same couplings, B with first colour 1. measure() returns A's 64 values
    then B's (src/gpu_2d.cu:196-205); swap() takes two mask words
    (src/parallel_tempering.hpp:143-149). Philox mode only."""

    def __init__(self, lattice, L: int, T: float = 1.0, h: float = 0.0):
        self.a = GpuSystem(lattice, L, T, h)
        self.b = GpuSystem(lattice, L, T, h)
        self.b.set_first_colour(1)
        self.lattice, self.L, self.N, self.h = self.a.lattice, self.a.L, self.a.N, self.a.h

    def _both(self, name, *args):
        for s in (self.a, self.b):
            getattr(s, name)(*args)

    def sweep(self, n: int = 1) -> None:
        self._both("sweep", n)

    def set_T(self, T: float) -> None:
        self._both("set_T", T)

    def get_T(self) -> float:
        return self.a.get_T()

    def set_h(self, h: float) -> None:
        self._both("set_h", h)
        self.h = float(h)

    def set_seed(self, seed: int) -> None:
        self._both("set_seed", seed)

    def init_J(self) -> None:
        self._both("init_J")

    def init_rand(self) -> None:
        self._both("init_rand")

    def rng_mode(self) -> int:
        return _lib.SA_RNG_PHILOX

    def measure(self) -> list[float]:
        return self.a.measure() + self.b.measure()

    def get_N(self) -> int:
        return self.N

    def swap(self, other: "TwoLatticeSystem", mask) -> None:
        m = list(mask) if hasattr(mask, "__len__") else [int(mask), 0]
        self.a.swap(other.a, int(m[0]))
        self.b.swap(other.b, int(m[1]))

    def load_J(self, fname: str) -> None:
        self._both("load_J", fname)

    def save_J(self, fname: str) -> None:
        self.a.save_J(fname)

    def get_J(self):
        return self.a.get_J()

    def save(self) -> bytes:
        ra, rb = self.a.save(), self.b.save()
        return struct.pack("<Q", len(ra)) + ra + struct.pack("<Q", len(rb)) + rb

    def load(self, data: bytes) -> None:
        (n,) = struct.unpack_from("<Q", data, 0)
        self.a.load(data[8:8 + n])
        (m,) = struct.unpack_from("<Q", data, 8 + n)
        self.b.load(data[16 + n:16 + n + m])

    def checkpoint_record(self) -> bytes:
        """A's record then B's, each with its length (the C++ shim's layout)."""
        return self.a.checkpoint_record() + self.b.checkpoint_record()

    def read_checkpoint_record(self, data: bytes, off: int) -> int:
        off = self.a.read_checkpoint_record(data, off)
        return self.b.read_checkpoint_record(data, off)

    def clone(self) -> "TwoLatticeSystem":
        c = TwoLatticeSystem(self.lattice, self.L, self.get_T(), self.h)
        c.load(self.save())
        return c

    def gpu_free(self) -> None:
        self._both("gpu_free")
