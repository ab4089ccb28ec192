"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares (no compute calls: this runs on CPU-only machines)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(r"\b(?:int|char|void|double|long|uint64_t)\s*\**\s*(sa_[A-Za-z0-9_]+)\s*\(")


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(DECL.findall(text))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared()
    assert "sa_sys_create" in names and "sa_sys_sweep" in names and len(names) >= 25


def test_library_exports_every_declared_symbol(sab):
    lib = ctypes.CDLL(os.path.join(ROOT, "simulated_annealing_b200", "libsa_b200.so"))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version(sab):
    lib = sab.load()
    assert b"sm_100a" in lib.sa_version()
    assert lib.sa_status_string(0) == b"ok"
    assert lib.sa_status_string(2) == b"L must be even"


def test_create_rejects_bad_arguments_before_touching_the_device(sab):
    from simulated_annealing_b200 import _lib
    lib = sab.load()
    h = ctypes.c_void_p()
    assert lib.sa_sys_create(0, 7, 1.0, 0.0, ctypes.byref(h)) == _lib.SA_ERR_ODD_L
    assert b"even" in lib.sa_last_error()
    assert lib.sa_sys_create(5, 8, 1.0, 0.0, ctypes.byref(h)) == _lib.SA_ERR_INVALID
    assert lib.sa_sys_create(0, 8, -1.0, 0.0, ctypes.byref(h)) == _lib.SA_ERR_INVALID
    assert lib.sa_sys_create(0, 8, 1.0, 0.0, None) == _lib.SA_ERR_INVALID
