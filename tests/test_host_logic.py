"""Host-side logic of the library that needs no GPU: the exchange generator,
the exchange test, and the integer thresholds / accept intervals the kernels
use in place of the reference's floating-point comparisons."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O


def _lib(sab):
    return sab.load()


def test_pt_sequence_matches_reference_generator(sab):
    lib = _lib(sab)
    for n in (2, 3, 5, 16, 32):
        systems = [O.OracleSystem(O.LAT_3D, 2, mode=O.MODE_MT) for _ in range(n)]
        for s in systems:
            s.set_seed(1)
            s.init_J()
            s.init_rand()
        pt = O.OraclePT(systems, list(np.linspace(0.5, 2.0, n)), 1)
        steps = [pt.step(0) for _ in range(40)]
        pair = np.zeros(40, dtype=np.int32)
        r = np.zeros(40, dtype=np.float64)
        assert lib.sa_pt_sequence(n, 0, 40, pair.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                  r.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
        assert pair.tolist() == [p for p, _, _ in steps]
        assert r.tolist() == [x for _, _, x in steps]
        # skipping into the sequence
        p2 = np.zeros(10, dtype=np.int32)
        r2 = np.zeros(10, dtype=np.float64)
        lib.sa_pt_sequence(n, 30, 10, p2.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                           r2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert p2.tolist() == pair[30:].tolist() and r2.tolist() == r[30:].tolist()


def test_pt_mask_matches_reference_test(sab):
    import math
    lib = _lib(sab)
    rng = np.random.default_rng(3)
    for _ in range(200):
        Ei = rng.integers(-3000, 3000, 64).astype(np.float32)
        Ej = (Ei + rng.integers(-40, 40, 64)).astype(np.float32)
        Ti, Tj = sorted(rng.uniform(0.3, 3.0, 2))
        r = float(rng.random())
        m = lib.sa_pt_mask(Ei.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                           Ej.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), Ti, Tj, r)
        dB = 1.0 / Ti - 1.0 / Tj
        ref = 0
        for j in range(64):
            dE = float(np.float32(-(Ei[j] - Ej[j])))
            if dE * dB > 0.0 or r < math.exp(dB * dE):
                ref |= 1 << j
        assert m == ref


@pytest.mark.parametrize("lattice", [0, 1, 2])
@pytest.mark.parametrize("T,h", [(0.3, 0.0), (1.0, 0.0), (2.27, 0.0), (0.8, 0.4), (5.0, -1.2)])
def test_thresholds_are_the_float_comparisons(oracle, lattice, T, h):
    """u < thr[k] must equal uniform(u) < (float)boltz[k] for every table entry
    (checked at the threshold and its neighbours and on random u)."""
    tab = oracle.boltz_table(lattice, T, h)
    rng = np.random.default_rng(int(T * 100))
    for b in tab:
        bf = float(np.float32(b))
        t = oracle.threshold(bf)
        for u in [t - 2, t - 1, t, t + 1] + list(rng.integers(0, 1 << 32, 50)):
            if 0 <= u < (1 << 32):
                assert (oracle.uniform_from_u32(int(u)) < bf) == (int(u) < t)
