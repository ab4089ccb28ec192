"""ctypes binding of the engine's C ABI (libsa_b200.so).

The library is the product: there is no Python or CPU fallback. Importing this
module on a machine without the built library raises; calls that need a GPU
return SA_ERR_NO_DEVICE / SA_ERR_CUDA, which are raised as SAError.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libsa_b200.so")

SA_OK = 0
SA_ERR_INVALID = 1
SA_ERR_ODD_L = 2
SA_ERR_CUDA = 3
SA_ERR_NO_DEVICE = 4
SA_ERR_MISMATCH = 5
SA_ERR_J_INCONSISTENT = 6
SA_ERR_BUFFER = 7
SA_ERR_BUDGET = 8
SA_ERR_TIMEOUT = 9
SA_ERR_UNSUPPORTED = 10

SA_LATTICE_2D = 0
SA_LATTICE_2D_OPEN_X = 1
SA_LATTICE_3D = 2
SA_RNG_PHILOX, SA_RNG_MT19937_64 = 0, 1


class SAError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


_c = ctypes
_vp = _c.c_void_p
_u64 = _c.c_uint64
_i64 = _c.c_int64
_u64p = _c.POINTER(_c.c_uint64)
_i64p = _c.POINTER(_c.c_int64)
_f32p = _c.POINTER(_c.c_float)
_f64p = _c.POINTER(_c.c_double)
_i32p = _c.POINTER(_c.c_int32)
_szp = _c.POINTER(_c.c_size_t)

# name -> (restype, argtypes); mirrors include/sa_b200.h and include/sa_b200_batch.h
_PROTOS = {
    "sa_last_error": (_c.c_char_p, []),
    "sa_status_string": (_c.c_char_p, [_c.c_int]),
    "sa_version": (_c.c_char_p, []),
    "sa_sys_create": (_c.c_int, [_c.c_int, _c.c_int, _c.c_double, _c.c_double, _c.POINTER(_vp)]),
    "sa_sys_destroy": (_c.c_int, [_vp]),
    "sa_sys_set_stream": (_c.c_int, [_vp, _vp]),
    "sa_sys_set_T": (_c.c_int, [_vp, _c.c_double]),
    "sa_sys_set_h": (_c.c_int, [_vp, _c.c_double]),
    "sa_sys_get_T": (_c.c_int, [_vp, _f64p]),
    "sa_sys_set_first_colour": (_c.c_int, [_vp, _c.c_int]),
    "sa_sys_get_first_colour": (_c.c_int, [_vp, _c.POINTER(_c.c_int)]),
    "sa_sys_set_split_field": (_c.c_int, [_vp, _c.c_int]),
    "sa_sys_get_split_field": (_c.c_int, [_vp, _c.POINTER(_c.c_int)]),
    "sa_sys_set_seed": (_c.c_int, [_vp, _u64]),
    "sa_sys_init_J": (_c.c_int, [_vp]),
    "sa_sys_init_rand": (_c.c_int, [_vp]),
    "sa_sys_init_order": (_c.c_int, [_vp]),
    "sa_sys_set_J": (_c.c_int, [_vp, _u64p, _u64p, _u64p]),
    "sa_sys_get_J": (_c.c_int, [_vp, _u64p, _u64p, _u64p]),
    "sa_sys_set_spins": (_c.c_int, [_vp, _u64p]),
    "sa_sys_get_spins": (_c.c_int, [_vp, _u64p]),
    "sa_sys_sweep": (_c.c_int, [_vp, _c.c_long]),
    "sa_sys_measure": (_c.c_int, [_vp, _i64p, _i64p]),
    "sa_sys_measure_float": (_c.c_int, [_vp, _f32p]),
    "sa_sys_measure_async": (_c.c_int, [_vp, _i64p, _i64p]),
    "sa_sys_swap": (_c.c_int, [_vp, _vp, _u64]),
    "sa_sys_get_N": (_c.c_int, [_vp, _c.POINTER(_c.c_long)]),
    "sa_sys_get_rng": (_c.c_int, [_vp, _u64p, _u64p, _u64p]),
    "sa_sys_set_rng_mode": (_c.c_int, [_vp, _c.c_int]),
    "sa_sys_get_rng_mode": (_c.c_int, [_vp, _c.POINTER(_c.c_int)]),
    "sa_sys_save_reference": (_c.c_int, [_vp, _vp, _c.c_size_t, _szp]),
    "sa_sys_load_reference": (_c.c_int, [_vp, _vp, _c.c_size_t]),
    "sa_sys_set_rng": (_c.c_int, [_vp, _u64, _u64, _u64]),
    "sa_sys_sync": (_c.c_int, [_vp]),
    "sa_sys_save": (_c.c_int, [_vp, _vp, _c.c_size_t, _szp]),
    "sa_sys_load": (_c.c_int, [_vp, _vp, _c.c_size_t]),
    "sa_sys_device_buffers": (_c.c_int, [_vp, _c.POINTER(_u64p), _c.POINTER(_u64p)]),
    "sa_measure_noalloc": (_c.c_int, [_c.c_int, _c.c_int, _vp, _vp, _vp, _vp, _vp]),
    "sa_sys_anneal": (_c.c_int, [_vp, _f64p, _c.c_int, _c.c_int, _c.c_int, _f32p, _i64p]),
    "sa_pt_sequence": (_c.c_int, [_c.c_int, _c.c_long, _c.c_long, _i32p, _f64p]),
    "sa_pt_mask": (_c.c_uint64, [_f32p, _f32p, _c.c_double, _c.c_double, _c.c_double]),
}

_LIB = None


def load(path: str = LIB_PATH):
    """Load libsa_b200.so (raises if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m simulated_annealing_b200.build` "
            "(nvcc, sm_100a). There is no CPU fallback.")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue  # checked by the ABI test against include/*.h
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def register(name: str, restype, argtypes):
    """Declare an extra entry point's prototype (used by submodules)."""
    _PROTOS[name] = (restype, argtypes)
    if _LIB is not None and hasattr(_LIB, name):
        fn = getattr(_LIB, name)
        fn.restype = restype
        fn.argtypes = argtypes


def check(status: int) -> None:
    if status != SA_OK:
        msg = load().sa_last_error()
        raise SAError(status, msg.decode() if msg else "")
