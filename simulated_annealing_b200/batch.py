"""Batched persistent engine (include/sa_b200_batch.h) from Python.

``Batch`` holds many disorder instances of mixed shape; each is either a
parallel-tempering ensemble over a temperature ladder (the reference's
parallel_tempering<gpu_sys>, src/parallel_tempering.hpp) or an anneal over a
temperature schedule (annealing<gpu_sys>, src/annealing.hpp). One call to
``run(nsweeps)`` is one persistent kernel launch that advances all of them.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check

_c = ctypes
_vp = _c.c_void_p
_i64p = _c.POINTER(_c.c_int64)
_u64p = _c.POINTER(_c.c_uint64)
_f64p = _c.POINTER(_c.c_double)
_ip = _c.POINTER(_c.c_int)
_lp = _c.POINTER(_c.c_long)

for _name, _res, _args in [
    ("sa_batch_create", _c.c_int, [_c.POINTER(_vp)]),
    ("sa_batch_destroy", _c.c_int, [_vp]),
    ("sa_batch_add_ladder", _c.c_int, [_vp, _f64p, _c.c_int, _ip]),
    ("sa_batch_add_schedule", _c.c_int, [_vp, _f64p, _c.c_int, _c.c_int, _ip]),
    ("sa_batch_add_instance", _c.c_int, [_vp, _c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_uint64,
                                         _c.c_uint64, _ip]),
    ("sa_batch_finalize", _c.c_int, [_vp]),
    ("sa_batch_set_exchange_interval", _c.c_int, [_vp, _c.c_int]),
    ("sa_batch_set_measure_stride", _c.c_int, [_vp, _c.c_int]),
    ("sa_batch_set_kernel", _c.c_int, [_vp, _c.c_int]),
    ("sa_batch_set_histograms", _c.c_int, [_vp, _c.c_int]),
    ("sa_batch_histogram", _c.c_int, [_vp, _c.c_int, _c.c_int, _c.POINTER(_c.c_int32), _c.c_long, _lp]),
    ("sa_batch_launches_per_run", _c.c_int, [_vp, _ip]),
    ("sa_batch_record_exchanges", _c.c_int, [_vp, _c.c_long]),
    ("sa_batch_run", _c.c_int, [_vp, _c.c_long]),
    ("sa_batch_sync", _c.c_int, [_vp]),
    ("sa_batch_set_stream", _c.c_int, [_vp, _vp]),
    ("sa_batch_site_slots", _c.c_int, [_vp, _c.POINTER(_c.c_longlong)]),
    ("sa_batch_num_instances", _c.c_int, [_vp, _ip]),
    ("sa_batch_get_spins", _c.c_int, [_vp, _c.c_int, _c.c_int, _u64p]),
    ("sa_batch_get_J", _c.c_int, [_vp, _c.c_int, _u64p, _u64p, _u64p]),
    ("sa_batch_measure", _c.c_int, [_vp, _c.c_int, _c.c_int, _i64p]),
    ("sa_batch_acceptance", _c.c_int, [_vp, _c.c_int, _i64p, _i64p]),
    ("sa_batch_exchanges", _c.c_int, [_vp, _c.c_int, _ip, _u64p, _c.c_long, _lp]),
    ("sa_batch_energies", _c.c_int, [_vp, _vp]),
    ("sa_batch_energy_count", _c.c_int, [_vp, _c.POINTER(_c.c_longlong)]),
    ("sa_batch_acceptance_all", _c.c_int, [_vp, _vp, _vp]),
    ("sa_batch_num_pairs", _c.c_int, [_vp, _c.POINTER(_c.c_longlong)]),
    ("sa_batch_last_h2d_bytes", _c.c_int, [_vp, _c.POINTER(_c.c_longlong)]),
    ("sa_batch_anneal_result", _c.c_int, [_vp, _c.c_int, _i64p, _lp]),
    ("sa_batch_sweeps_done", _c.c_int, [_vp, _c.c_int, _lp]),
    ("sa_tuning_table", _c.c_int, [_c.POINTER(_c.c_int32), _c.c_int, _ip]),
    ("sa_batch_set_tuning", _c.c_int, [_vp, _c.POINTER(_c.c_int32), _c.c_int]),
    ("sa_batch_set_spread", _c.c_int, [_vp, _c.c_int]),
    ("sa_batch_instance_shape", _c.c_int, [_vp, _c.c_int, _c.POINTER(_c.c_int32)]),
    ("sa_batch_set_group_timing", _c.c_int, [_vp, _c.c_int]),
    ("sa_batch_group_times", _c.c_int, [_vp, _c.POINTER(_c.c_int32), _c.POINTER(_c.c_float), _c.c_int, _ip]),
]:
    _lib.register(_name, _res, _args)

LATTICE = {"2d": _lib.SA_LATTICE_2D, "2p": _lib.SA_LATTICE_2D_OPEN_X, "3d": _lib.SA_LATTICE_3D}


def _p(a, ct):
    return a.ctypes.data_as(_c.POINTER(ct))


KERNEL_AUTO, KERNEL_GLOBAL, KERNEL_NO_WIDE = 0, 1, 2


class Batch:
    """kernel: KERNEL_AUTO keeps instances resident in cluster shared memory
    where they fit (a lone single-slot 3D anneal of L >= 40 runs wide, over
    the whole GPU); KERNEL_GLOBAL streams every instance from global memory;
    KERNEL_NO_WIDE is KERNEL_AUTO without the wide form."""

    def __init__(self, kernel: int = KERNEL_AUTO):
        self._lib = _lib.load()
        h = _vp()
        check(self._lib.sa_batch_create(_c.byref(h)))
        self._h = h
        if kernel != KERNEL_AUTO:
            check(self._lib.sa_batch_set_kernel(self._h, int(kernel)))
        self.instances = []  # (lattice, L, nslots)
        self._ladders = []
        self._final = False

    def add_ladder(self, T) -> int:
        T = np.ascontiguousarray(T, dtype=np.float64)
        i = _c.c_int()
        check(self._lib.sa_batch_add_ladder(self._h, _p(T, _c.c_double), len(T), _c.byref(i)))
        self._ladders.append(np.sort(T))
        return i.value

    def add_schedule(self, T, sweeps_per_step: int) -> int:
        T = np.ascontiguousarray(T, dtype=np.float64)
        i = _c.c_int()
        check(self._lib.sa_batch_add_schedule(self._h, _p(T, _c.c_double), len(T), int(sweeps_per_step),
                                              _c.byref(i)))
        return i.value

    def add_instance(self, lattice, L: int, *, ladder: int = -1, schedule: int = -1, seed_J: int, seed: int) -> int:
        if isinstance(lattice, str):
            lattice = LATTICE[lattice]
        i = _c.c_int()
        check(self._lib.sa_batch_add_instance(self._h, int(lattice), int(L), int(ladder), int(schedule),
                                              int(seed_J) & (2**64 - 1), int(seed) & (2**64 - 1), _c.byref(i)))
        nslots = len(self._ladders[ladder]) if ladder >= 0 else 1
        self.instances.append((int(lattice), int(L), nslots))
        return i.value

    def finalize(self) -> None:
        check(self._lib.sa_batch_finalize(self._h))
        self._final = True

    def set_tuning(self, entries) -> None:
        """Launch shapes per bucket, rows of (lattice, L, slots, C, SL, warps,
        hr); None: back to the built-in table; []: heuristics only."""
        if entries is None:
            check(self._lib.sa_batch_set_tuning(self._h, None, -1))
            return
        a = np.ascontiguousarray(np.asarray(entries, dtype=np.int32).reshape(-1, 7))
        check(self._lib.sa_batch_set_tuning(self._h, _p(a, _c.c_int32), len(a)))

    def set_group_timing(self, on: bool) -> None:
        check(self._lib.sa_batch_set_group_timing(self._h, int(bool(on))))

    def group_times(self):
        """Per launch group of the last run: dicts of lattice, L, instances,
        C, warps and the ms from the run's start to the group's end."""
        n = _c.c_int()
        check(self._lib.sa_batch_group_times(self._h, None, None, 0, _c.byref(n)))
        info = np.zeros((max(n.value, 1), 5), dtype=np.int32)
        ms = np.zeros(max(n.value, 1), dtype=np.float32)
        check(self._lib.sa_batch_group_times(self._h, _p(info, _c.c_int32), _p(ms, _c.c_float), n.value,
                                             _c.byref(n)))
        return [{"lattice": int(r[0]), "L": int(r[1]), "instances": int(r[2]), "C": int(r[3]), "warps": int(r[4]),
                 "end_ms": round(float(t), 3)} for r, t in zip(info[: n.value], ms[: n.value])]

    def set_spread(self, on: bool) -> None:
        check(self._lib.sa_batch_set_spread(self._h, int(bool(on))))

    def shape(self, i: int):
        """(lattice, L, slots, C, SL, warps, hr) instance i runs with."""
        out = np.zeros(7, dtype=np.int32)
        check(self._lib.sa_batch_instance_shape(self._h, i, _p(out, _c.c_int32)))
        return tuple(int(v) for v in out)

    def set_exchange_interval(self, k: int) -> None:
        check(self._lib.sa_batch_set_exchange_interval(self._h, int(k)))

    def set_histograms(self, stride: int) -> None:
        check(self._lib.sa_batch_set_histograms(self._h, int(stride)))

    def histogram(self, i: int, slot: int) -> np.ndarray:
        n = _c.c_long()
        check(self._lib.sa_batch_histogram(self._h, i, slot, None, 0, _c.byref(n)))
        out = np.zeros(n.value, dtype=np.int32)
        check(self._lib.sa_batch_histogram(self._h, i, slot, _p(out, _c.c_int32), n.value, _c.byref(n)))
        return out

    def set_measure_stride(self, k: int) -> None:
        check(self._lib.sa_batch_set_measure_stride(self._h, int(k)))

    def record_exchanges(self, cap: int) -> None:
        check(self._lib.sa_batch_record_exchanges(self._h, int(cap)))

    def run(self, nsweeps: int) -> None:
        check(self._lib.sa_batch_run(self._h, int(nsweeps)))

    def sync(self) -> None:
        check(self._lib.sa_batch_sync(self._h))

    def set_stream(self, stream_ptr: int) -> None:
        check(self._lib.sa_batch_set_stream(self._h, _vp(stream_ptr)))

    def launches_per_run(self) -> int:
        n = _c.c_int()
        check(self._lib.sa_batch_launches_per_run(self._h, _c.byref(n)))
        return n.value

    def site_slots(self) -> int:
        n = _c.c_longlong()
        check(self._lib.sa_batch_site_slots(self._h, _c.byref(n)))
        return n.value

    def N(self, i: int) -> int:
        lat, L, _ = self.instances[i]
        return L ** 3 if lat == _lib.SA_LATTICE_3D else L * L

    def spins(self, i: int, slot: int) -> np.ndarray:
        s = np.zeros(self.N(i), dtype=np.uint64)
        check(self._lib.sa_batch_get_spins(self._h, i, slot, _p(s, _c.c_uint64)))
        return s

    def J(self, i: int):
        lat = self.instances[i][0]
        n = self.N(i)
        arrs = [np.zeros(2 * n, dtype=np.uint64) for _ in range(3 if lat == _lib.SA_LATTICE_3D else 2)]
        jz = _p(arrs[2], _c.c_uint64) if len(arrs) == 3 else None
        check(self._lib.sa_batch_get_J(self._h, i, _p(arrs[0], _c.c_uint64), _p(arrs[1], _c.c_uint64), jz))
        return tuple(arrs)

    def measure(self, i: int, slot: int) -> np.ndarray:
        E = np.zeros(64, dtype=np.int64)
        check(self._lib.sa_batch_measure(self._h, i, slot, _p(E, _c.c_int64)))
        return E

    def acceptance(self, i: int):
        n = max(0, self.instances[i][2] - 1)
        a = np.zeros(max(n, 1), dtype=np.int64)
        t = np.zeros(max(n, 1), dtype=np.int64)
        check(self._lib.sa_batch_acceptance(self._h, i, _p(a, _c.c_int64), _p(t, _c.c_int64)))
        return a[:n], t[:n]

    def exchanges(self, i: int):
        cnt = _c.c_long()
        check(self._lib.sa_batch_exchanges(self._h, i, None, None, 0, _c.byref(cnt)))
        n = cnt.value
        pairs = np.zeros(max(n, 1), dtype=np.int32)
        masks = np.zeros(max(n, 1), dtype=np.uint64)
        check(self._lib.sa_batch_exchanges(self._h, i, _p(pairs, _c.c_int), _p(masks, _c.c_uint64), n,
                                           _c.byref(cnt)))
        return pairs[:n], masks[:n]

    def energy_count(self) -> int:
        n = _c.c_longlong()
        check(self._lib.sa_batch_energy_count(self._h, _c.byref(n)))
        return n.value

    def num_pairs(self) -> int:
        n = _c.c_longlong()
        check(self._lib.sa_batch_num_pairs(self._h, _c.byref(n)))
        return n.value

    def energies_into(self, host_ptr: int) -> None:
        """Async: all slots' energies into host memory at host_ptr (int64, energy_count())."""
        check(self._lib.sa_batch_energies(self._h, _vp(host_ptr)))

    def acceptance_into(self, acc_ptr: int, att_ptr: int) -> None:
        check(self._lib.sa_batch_acceptance_all(self._h, _vp(acc_ptr), _vp(att_ptr)))

    def energies(self) -> np.ndarray:
        out = np.zeros(self.energy_count(), dtype=np.int64)
        self.energies_into(out.ctypes.data)
        self.sync()
        return out

    def last_h2d_bytes(self) -> int:
        n = _c.c_longlong()
        check(self._lib.sa_batch_last_h2d_bytes(self._h, _c.byref(n)))
        return n.value

    def anneal_result(self, i: int):
        E = np.zeros(64, dtype=np.int64)
        n = _c.c_long()
        check(self._lib.sa_batch_anneal_result(self._h, i, _p(E, _c.c_int64), _c.byref(n)))
        return E, n.value

    def sweeps_done(self, i: int) -> int:
        n = _c.c_long()
        check(self._lib.sa_batch_sweeps_done(self._h, i, _c.byref(n)))
        return n.value

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.sa_batch_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tuning_table() -> np.ndarray:
    """The built-in launch shapes, rows of (lattice, L, slots, C, SL, warps, hr)."""
    lib = _lib.load()
    n = _c.c_int()
    check(lib.sa_tuning_table(None, 0, _c.byref(n)))
    out = np.zeros((max(n.value, 1), 7), dtype=np.int32)
    check(lib.sa_tuning_table(_p(out, _c.c_int32), n.value, _c.byref(n)))
    return out[: n.value]
