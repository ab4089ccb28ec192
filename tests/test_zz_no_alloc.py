"""sa_measure_noalloc: the energy measurement that allocates nothing.

Some callers cannot allocate device memory when they need an energy (their
HBM budget is reserved up front, or cudaMalloc's latency and implicit
synchronisation are not acceptable in their loop). For them the library keeps
its measurement scratch in a fixed device array. This test calls that entry
point through the C ABI on a system's own device buffers and checks it against
sa_sys_measure, on two calls in a row (with a sweep between them, and a second
lattice shape that reuses the same shared scratch).

Collected last (file name) so that a failure here comes after every other
test has run; it must also pass alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, sysobj, d_E, d_M, stream=None):
    spins = ctypes.POINTER(ctypes.c_uint64)()
    J = ctypes.POINTER(ctypes.c_uint64)()
    assert lib.sa_sys_device_buffers(sysobj._h, ctypes.byref(spins), ctypes.byref(J)) == 0
    st = lib.sa_measure_noalloc(sysobj.lattice, sysobj.L, ctypes.cast(spins, ctypes.c_void_p),
                                ctypes.cast(J, ctypes.c_void_p), ctypes.c_void_p(d_E.data_ptr()),
                                ctypes.c_void_p(d_M.data_ptr()), stream)
    assert st == 0, lib.sa_last_error()


@pytest.mark.parametrize("lattice,L,T,h", [(0, 32, 1.0, 0.0), (2, 12, 0.7, 0.3), (1, 18, 2.0, -0.4)])
def test_noalloc_measure_matches_sa_sys_measure_twice(sab, lattice, L, T, h):
    import torch

    from simulated_annealing_b200.system import GpuSystem

    lib = sab.load()
    g = GpuSystem(lattice, L, T, h)
    g.set_seed(5)
    g.init_J()
    g.set_seed(6)
    g.init_rand()
    d_E = torch.zeros(64, dtype=torch.int64, device="cuda")
    d_M = torch.zeros(64, dtype=torch.int64, device="cuda")
    for _ in range(2):
        g.sync()
        _noalloc(lib, g, d_E, d_M)  # default stream; the system's stream is synchronised
        torch.cuda.synchronize()
        E, M = g.measure_exact()
        assert np.array_equal(d_E.cpu().numpy(), E)
        assert np.array_equal(d_M.cpu().numpy(), M)
        g.sweep(3)


def test_noalloc_rejects_oversized_lattice(sab):
    from simulated_annealing_b200._lib import SA_ERR_BUDGET

    lib = sab.load()
    one = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.sa_measure_noalloc(2, 1024, one, one, one, one, None)
    assert st == SA_ERR_BUDGET
    assert b"too large" in lib.sa_last_error()
