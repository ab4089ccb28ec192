"""ctypes access to the oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker. It loads

* ``oracle/libsa_oracle.so`` -- the CPU restatement (sa_oracle.cpp), and
* ``oracle/_ref/libsa_ref.so`` -- the reference's own CPU classes
  (cpu_2d / cpu_2dp / cpu_3d, annealing<>, parallel_tempering<>) compiled from
  their sources by oracle/Makefile, when it was built.

Lattice kinds follow the reference classes: 0 = cpu_2d (2D periodic),
1 = cpu_2dp (2D, open in x), 2 = cpu_3d (3D periodic).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libsa_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsa_ref.so")

LAT_2D, LAT_2D_OPEN_X, LAT_3D = 0, 1, 2
MODE_PHILOX, MODE_MT = 0, 1

_u64 = ctypes.c_uint64
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


def build() -> None:
    """Compile the oracle, and the reference library when SA_REFERENCE_SRC names
    the reference's src/ directory."""
    ref = os.environ.get("SA_REFERENCE_SRC")
    extra = [f"REF_SRC={ref}"] if ref else []
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile"), *extra], check=True)


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(ct)


def lattice_N(lattice: int, L: int) -> int:
    return L ** 3 if lattice == LAT_3D else L * L


def _load_oracle():
    if not os.path.exists(ORACLE_SO):
        build()
    lib = ctypes.CDLL(ORACLE_SO)
    lib.sao_philox4x32_10.argtypes = [ctypes.POINTER(ctypes.c_uint32)] * 3
    lib.sao_philox_draw.restype = ctypes.c_uint32
    lib.sao_philox_draw.argtypes = [_u64, _u64, _u64]
    lib.sao_uniform_from_u32.restype = ctypes.c_float
    lib.sao_uniform_from_u32.argtypes = [ctypes.c_uint32]
    lib.sao_threshold.restype = _u64
    lib.sao_threshold.argtypes = [ctypes.c_float]
    lib.sao_check_uniform_monotone.restype = ctypes.c_int
    lib.sao_boltz_table.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _f64p]
    lib.sao_sys_new.restype = _vp
    lib.sao_sys_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    lib.sao_sys_free.argtypes = [_vp]
    lib.sao_sys_N.restype = ctypes.c_long
    lib.sao_sys_N.argtypes = [_vp]
    lib.sao_sys_set_seed.argtypes = [_vp, _u64]
    lib.sao_sys_set_T.argtypes = [_vp, ctypes.c_double]
    lib.sao_sys_set_h.argtypes = [_vp, ctypes.c_double]
    lib.sao_sys_get_T.restype = ctypes.c_double
    lib.sao_sys_get_T.argtypes = [_vp]
    lib.sao_sys_get_draw.restype = _u64
    lib.sao_sys_get_draw.argtypes = [_vp]
    lib.sao_sys_set_draw.argtypes = [_vp, _u64]
    lib.sao_sys_set_first_colour.argtypes = [_vp, ctypes.c_int]
    lib.sao_sys_set_split.argtypes = [_vp, ctypes.c_int]
    for f in ("sao_sys_init_J", "sao_sys_init_rand", "sao_sys_init_order"):
        getattr(lib, f).argtypes = [_vp]
    lib.sao_sys_sweep.argtypes = [_vp, ctypes.c_long]
    lib.sao_sys_measure.argtypes = [_vp, _i64p, _i64p]
    lib.sao_sys_measure_float.argtypes = [_vp, _f32p]
    lib.sao_sys_get_spins.argtypes = [_vp, _u64p]
    lib.sao_sys_set_spins.argtypes = [_vp, _u64p]
    lib.sao_sys_get_J.argtypes = [_vp, _u64p, _u64p, _u64p]
    lib.sao_sys_set_J.argtypes = [_vp, _u64p, _u64p, _u64p]
    lib.sao_sys_swap.argtypes = [_vp, _vp, _u64]
    lib.sao_pt_new.restype = _vp
    lib.sao_pt_new.argtypes = [ctypes.POINTER(_vp), _f64p, ctypes.c_int, ctypes.c_long]
    lib.sao_pt_free.argtypes = [_vp]
    lib.sao_pt_step.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _u64p, _f64p]
    lib.sao_pt_energies.argtypes = [_vp, _f32p]
    lib.sao_pt_acceptance.argtypes = [_vp, _f64p]
    lib.sao_pt_sorted_T.argtypes = [_vp, _f64p]
    lib.sao_anneal_run.argtypes = [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, _f32p, _f32p]
    return lib


_ORACLE = None
_REF = None


def oracle_lib():
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = _load_oracle()
    return _ORACLE


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _REF
    if _REF is None:
        lib = ctypes.CDLL(REF_SO)
        lib.ref_omp_threads.argtypes = [ctypes.c_int]
        lib.ref_sys_new.restype = _vp
        lib.ref_sys_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        lib.ref_sys_free.argtypes = [_vp]
        lib.ref_set_seed.argtypes = [_vp, ctypes.c_long]
        for f in ("ref_init_J", "ref_init_rand", "ref_init_order"):
            getattr(lib, f).argtypes = [_vp]
        lib.ref_set_T.argtypes = [_vp, ctypes.c_double]
        lib.ref_sweep.argtypes = [_vp, ctypes.c_long]
        lib.ref_measure.argtypes = [_vp, _f32p]
        lib.ref_get_N.restype = ctypes.c_long
        lib.ref_get_N.argtypes = [_vp]
        lib.ref_get_state.argtypes = [_vp, _u64p, _u64p, _u64p, _u64p]
        lib.ref_swap.argtypes = [_vp, _vp, _u64]
        lib.ref_pt_new.restype = _vp
        lib.ref_pt_new.argtypes = [ctypes.POINTER(_vp), _f64p, ctypes.c_int, ctypes.c_long]
        lib.ref_pt_step.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _u64p]
        lib.ref_pt_last_T.restype = ctypes.c_double
        lib.ref_pt_last_T.argtypes = [_vp]
        lib.ref_pt_update_T.argtypes = [_vp]
        lib.ref_pt_save.restype = ctypes.c_long
        lib.ref_pt_save.argtypes = [_vp, ctypes.c_char_p, ctypes.c_long]
        lib.ref_pt_load.argtypes = [_vp, ctypes.c_char_p, ctypes.c_long]
        lib.ref_pt_print_swap.restype = ctypes.c_int
        lib.ref_pt_print_swap.argtypes = [_vp, ctypes.c_char_p, ctypes.c_int]
        lib.ref_pt_free.argtypes = [_vp]
        lib.ref_anneal_run.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, _f32p]
        lib.ref_save_J.argtypes = [_vp, ctypes.c_char_p]
        lib.ref_load_J.argtypes = [_vp, ctypes.c_char_p]
        lib.ref_save.restype = ctypes.c_long
        lib.ref_save.argtypes = [_vp, ctypes.c_char_p, ctypes.c_long]
        lib.ref_load.argtypes = [_vp, ctypes.c_char_p, ctypes.c_long]
        _REF = lib
    return _REF


# ----------------------------------------------------------------------------- RNG
def philox_draw(seed: int, subsequence: int, index: int) -> int:
    return int(oracle_lib().sao_philox_draw(seed, subsequence, index))


def uniform_from_u32(u: int) -> float:
    return float(oracle_lib().sao_uniform_from_u32(u))


def threshold(b: float) -> int:
    return int(oracle_lib().sao_threshold(b))


def boltz_table(lattice: int, T: float, h: float) -> np.ndarray:
    out = np.zeros(20, dtype=np.float64)
    oracle_lib().sao_boltz_table(lattice, T, h, _ptr(out, _f64p))
    return out[: (14 if lattice == LAT_3D else 20)]


# ----------------------------------------------------------------------------- systems
class OracleSystem:
    """One 64-replica system of the restatement (PHILOX or MT random numbers)."""

    def __init__(self, lattice: int, L: int, T: float = 1.0, h: float = 0.0, mode: int = MODE_PHILOX):
        self.lib = oracle_lib()
        self.lattice, self.L, self.mode = lattice, L, mode
        self.h = self.lib.sao_sys_new(lattice, L, T, h, mode)
        if not self.h:
            raise ValueError("bad oracle system parameters")
        self.N = int(self.lib.sao_sys_N(self.h))
        self.hfield = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.sao_sys_free(self.h)
            self.h = None

    def set_seed(self, seed: int):
        self.lib.sao_sys_set_seed(self.h, seed)

    def set_T(self, T: float):
        self.lib.sao_sys_set_T(self.h, T)

    def set_h(self, hf: float):
        self.hfield = hf
        self.lib.sao_sys_set_h(self.h, hf)

    @property
    def draw(self) -> int:
        return int(self.lib.sao_sys_get_draw(self.h))

    @draw.setter
    def draw(self, d: int):
        self.lib.sao_sys_set_draw(self.h, d)

    def init_J(self):
        self.lib.sao_sys_init_J(self.h)

    def init_rand(self):
        self.lib.sao_sys_init_rand(self.h)

    def init_order(self):
        self.lib.sao_sys_init_order(self.h)

    def set_first_colour(self, c: int):
        self.lib.sao_sys_set_first_colour(self.h, c)

    def set_split(self, on: bool):
        self.lib.sao_sys_set_split(self.h, int(bool(on)))

    def sweep(self, n: int = 1):
        self.lib.sao_sys_sweep(self.h, n)

    def measure(self):
        E = np.zeros(64, dtype=np.int64)
        M = np.zeros(64, dtype=np.int64)
        self.lib.sao_sys_measure(self.h, _ptr(E, _i64p), _ptr(M, _i64p))
        return E, M

    def measure_float(self) -> np.ndarray:
        out = np.zeros(64, dtype=np.float32)
        self.lib.sao_sys_measure_float(self.h, _ptr(out, _f32p))
        return out

    def spins(self) -> np.ndarray:
        s = np.zeros(self.N, dtype=np.uint64)
        self.lib.sao_sys_get_spins(self.h, _ptr(s, _u64p))
        return s

    def set_spins(self, s: np.ndarray):
        s = np.ascontiguousarray(s, dtype=np.uint64)
        self.lib.sao_sys_set_spins(self.h, _ptr(s, _u64p))

    def J(self):
        jx = np.zeros(2 * self.N, dtype=np.uint64)
        jy = np.zeros(2 * self.N, dtype=np.uint64)
        jz = np.zeros(2 * self.N, dtype=np.uint64)
        self.lib.sao_sys_get_J(self.h, _ptr(jx, _u64p), _ptr(jy, _u64p), _ptr(jz, _u64p))
        return (jx, jy, jz) if self.lattice == LAT_3D else (jx, jy)

    def set_J(self, jx, jy, jz=None):
        jx = np.ascontiguousarray(jx, dtype=np.uint64)
        jy = np.ascontiguousarray(jy, dtype=np.uint64)
        jz = np.ascontiguousarray(jz if jz is not None else np.zeros(2 * self.N), dtype=np.uint64)
        self.lib.sao_sys_set_J(self.h, _ptr(jx, _u64p), _ptr(jy, _u64p), _ptr(jz, _u64p))

    def swap(self, other: "OracleSystem", mask: int):
        self.lib.sao_sys_swap(self.h, other.h, mask)

    def anneal(self, T0, schedule, alfa_or_T1, nsteps, sweeps, stride=1):
        mn = np.zeros(64, dtype=np.float32)
        last = np.zeros((nsteps, 64), dtype=np.float32)
        self.lib.sao_anneal_run(self.h, T0, schedule, alfa_or_T1, nsteps, sweeps, stride,
                                _ptr(mn, _f32p), _ptr(last, _f32p))
        return mn, last


class OraclePT:
    """parallel_tempering<> restated over OracleSystem slots."""

    def __init__(self, systems, T, steps: int = 1):
        self.lib = oracle_lib()
        self.systems = list(systems)
        self.n = len(self.systems)
        arr = (_vp * self.n)(*[s.h for s in self.systems])
        Tv = np.ascontiguousarray(T, dtype=np.float64)
        self.h = self.lib.sao_pt_new(arr, _ptr(Tv, _f64p), self.n, steps)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.sao_pt_free(self.h)
            self.h = None

    def step(self, stride: int = 0):
        pair = ctypes.c_int(0)
        mask = np.zeros(1, dtype=np.uint64)
        r = np.zeros(1, dtype=np.float64)
        self.lib.sao_pt_step(self.h, stride, ctypes.byref(pair), _ptr(mask, _u64p), _ptr(r, _f64p))
        return int(pair.value), int(mask[0]), float(r[0])

    def energies(self) -> np.ndarray:
        out = np.zeros((self.n, 64), dtype=np.float32)
        self.lib.sao_pt_energies(self.h, _ptr(out, _f32p))
        return out

    def acceptance(self) -> np.ndarray:
        out = np.zeros(self.n - 1, dtype=np.float64)
        self.lib.sao_pt_acceptance(self.h, _ptr(out, _f64p))
        return out

    def sorted_T(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.float64)
        self.lib.sao_pt_sorted_T(self.h, _ptr(out, _f64p))
        return out


class RefSystem:
    """The reference's own cpu_2d / cpu_2dp / cpu_3d object (oracle/_ref)."""

    def __init__(self, lattice: int, L: int, T: float = 1.0, h: float = 0.0):
        self.lib = ref_lib()
        self.lattice, self.L = lattice, L
        self.h = self.lib.ref_sys_new(lattice, L, T, h)
        self.N = int(self.lib.ref_get_N(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_sys_free(self.h)
            self.h = None

    def set_seed(self, seed):
        self.lib.ref_set_seed(self.h, seed)

    def init_J(self):
        self.lib.ref_init_J(self.h)

    def init_rand(self):
        self.lib.ref_init_rand(self.h)

    def init_order(self):
        self.lib.ref_init_order(self.h)

    def set_T(self, T):
        self.lib.ref_set_T(self.h, T)

    def sweep(self, n=1):
        self.lib.ref_sweep(self.h, n)

    def measure_float(self) -> np.ndarray:
        out = np.zeros(64, dtype=np.float32)
        self.lib.ref_measure(self.h, _ptr(out, _f32p))
        return out

    def state(self):
        s = np.zeros(self.N, dtype=np.uint64)
        jx = np.zeros(2 * self.N, dtype=np.uint64)
        jy = np.zeros(2 * self.N, dtype=np.uint64)
        jz = np.zeros(2 * self.N, dtype=np.uint64)
        self.lib.ref_get_state(self.h, _ptr(s, _u64p), _ptr(jx, _u64p), _ptr(jy, _u64p), _ptr(jz, _u64p))
        return s, jx, jy, jz

    def swap(self, other, mask):
        self.lib.ref_swap(self.h, other.h, mask)

    def save_J(self, fname: str) -> None:
        self.lib.ref_save_J(self.h, fname.encode())

    def load_J(self, fname: str) -> None:
        self.lib.ref_load_J(self.h, fname.encode())

    def save(self) -> bytes:
        n = self.lib.ref_save(self.h, None, 0)
        buf = ctypes.create_string_buffer(n)
        self.lib.ref_save(self.h, buf, n)
        return buf.raw[:n]

    def load(self, data: bytes) -> None:
        self.lib.ref_load(self.h, data, len(data))

    def anneal(self, T0, alfa, nsteps, sweeps, stride=1):
        mn = np.zeros(64, dtype=np.float32)
        self.lib.ref_anneal_run(self.h, T0, alfa, nsteps, sweeps, stride, _ptr(mn, _f32p))
        return mn


class RefPT:
    """The reference's parallel_tempering<cpu_sys> over RefSystem slots."""

    def __init__(self, systems, T, steps=1):
        self.lib = ref_lib()
        self.systems = list(systems)
        arr = (_vp * len(self.systems))(*[s.h for s in self.systems])
        Tv = np.ascontiguousarray(T, dtype=np.float64)
        self.h = self.lib.ref_pt_new(arr, _ptr(Tv, _f64p), len(self.systems), steps)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_pt_free(self.h)
            self.h = None

    def step(self, stride=0):
        pair = ctypes.c_int(0)
        mask = np.zeros(1, dtype=np.uint64)
        self.lib.ref_pt_step(self.h, stride, ctypes.byref(pair), _ptr(mask, _u64p))
        return int(pair.value), int(mask[0])

    def last_T(self) -> float:
        return float(self.lib.ref_pt_last_T(self.h))

    def update_T(self) -> None:
        self.lib.ref_pt_update_T(self.h)

    def save(self) -> bytes:
        n = self.lib.ref_pt_save(self.h, None, 0)
        buf = ctypes.create_string_buffer(n)
        self.lib.ref_pt_save(self.h, buf, n)
        return buf.raw[:n]

    def load(self, data: bytes) -> None:
        self.lib.ref_pt_load(self.h, data, len(data))

    def print_swap(self) -> str:
        buf = ctypes.create_string_buffer(1 << 16)
        self.lib.ref_pt_print_swap(self.h, buf, 1 << 16)
        return buf.value.decode()
