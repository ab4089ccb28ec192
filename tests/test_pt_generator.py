"""The parallel-tempering exchange generator on the host (no GPU).

sa_pt_gen_* keep the template's std::mt19937(123) / uniform_int_distribution
/ uniform_real_distribution members (src/parallel_tempering.hpp:28-30) as an
object; its checkpoint bytes must be the ones the reference template itself
writes into a .tempsys stream (src/parallel_tempering.hpp:284-287).
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O


def _lib():
    from simulated_annealing_b200 import drivers  # noqa: F401  (registers the prototypes)
    from simulated_annealing_b200 import _lib as L

    return L.load()


def _gen(lib, n):
    g = ctypes.c_void_p()
    assert lib.sa_pt_gen_create(n, ctypes.byref(g)) == 0
    return g


def _next(lib, g, k):
    p = np.zeros(k, dtype=np.int32)
    r = np.zeros(k, dtype=np.float64)
    assert lib.sa_pt_gen_next(g, k, p.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                              r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    return p, r


def _bytes(lib, g):
    n = ctypes.c_size_t()
    assert lib.sa_pt_gen_save(g, None, 0, ctypes.byref(n)) == 0
    buf = ctypes.create_string_buffer(n.value)
    assert lib.sa_pt_gen_save(g, buf, n.value, ctypes.byref(n)) == 0
    return buf.raw[: n.value]


def test_generator_object_follows_the_sequence():
    lib = _lib()
    g = _gen(lib, 16)
    p, r = _next(lib, g, 300)
    sp = np.zeros(300, dtype=np.int32)
    sr = np.zeros(300, dtype=np.float64)
    assert lib.sa_pt_sequence(16, 0, 300, sp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                              sr.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    assert np.array_equal(p, sp) and np.array_equal(r, sr)
    lib.sa_pt_gen_destroy(g)


def test_generator_checkpoint_resumes():
    lib = _lib()
    g = _gen(lib, 9)
    _next(lib, g, 57)
    blob = _bytes(lib, g)
    assert len(blob) == 5024  # libstdc++ on LP64: 624 x 8 + 8, 2 x 4, 2 x 8
    want = _next(lib, g, 40)
    h = _gen(lib, 2)
    assert lib.sa_pt_gen_load(h, blob, len(blob)) == 0
    got = _next(lib, h, 40)
    assert all(np.array_equal(a, b) for a, b in zip(want, got))
    assert lib.sa_pt_gen_load(h, blob, len(blob) - 1) != 0
    for x in (g, h):
        lib.sa_pt_gen_destroy(x)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("k", [0, 1, 13])
def test_generator_bytes_are_the_templates(k):
    """After k exchange attempts the bytes equal those the reference's own
    parallel_tempering<cpu_sys>::save writes after k steps (offset 10: after
    steps, print_E, print_min)."""
    lib = _lib()
    T = [0.5, 0.9, 1.4, 2.0]
    rs = [O.RefSystem(O.LAT_3D, 4) for _ in T]
    for s in rs:
        s.set_seed(3)
        s.init_J()
        s.set_seed(4)
        s.init_rand()
    rp = O.RefPT(rs, T, 1)
    for _ in range(k):
        rp.step(0)
    ref = rp.save()
    g = _gen(lib, len(T))
    _next(lib, g, k)
    blob = _bytes(lib, g)
    assert ref[10:10 + len(blob)] == blob
    lib.sa_pt_gen_destroy(g)
