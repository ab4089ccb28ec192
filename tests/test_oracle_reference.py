"""The oracle's restatement (MT mode) against the reference's own CPU classes.

oracle/_ref/libsa_ref.so holds cpu_2d / cpu_2dp / cpu_3d, annealing<> and
parallel_tempering<> compiled unmodified from the reference sources. Driving
both with the same std::mt19937_64 seeds must give identical spin words, float
energies, exchange decisions and running minima -- this pins the lattice logic,
sweep order, energy convention and PT/annealing steps the GPU parity tests use.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")

CASES = [(O.LAT_2D, 8), (O.LAT_2D, 16), (O.LAT_2D, 6), (O.LAT_2D_OPEN_X, 8), (O.LAT_2D_OPEN_X, 12),
         (O.LAT_2D_OPEN_X, 2), (O.LAT_3D, 4), (O.LAT_3D, 6), (O.LAT_3D, 2)]


@pytest.mark.parametrize("lat,L", CASES)
@pytest.mark.parametrize("T,h", [(1.0, 0.0), (0.7, 0.3), (2.2, -0.5)])
def test_sweep_and_measure_match_reference(lat, L, T, h):
    r = O.RefSystem(lat, L, T, h)
    o = O.OracleSystem(lat, L, T, h, O.MODE_MT)
    for x in (r, o):
        x.set_seed(11)
        x.init_J()
        x.set_seed(22)
        x.init_rand()
    s, jx, jy, jz = r.state()
    J = o.J()
    assert np.array_equal(J[0], jx) and np.array_equal(J[1], jy)
    if lat == O.LAT_3D:
        assert np.array_equal(J[2], jz)
    for _ in range(4):
        r.sweep(3)
        o.sweep(3)
        assert np.array_equal(r.state()[0], o.spins())
        assert np.array_equal(r.measure_float(), o.measure_float())


@pytest.mark.parametrize("lat,L", [(O.LAT_2D, 32), (O.LAT_2D, 64), (O.LAT_2D_OPEN_X, 64), (O.LAT_3D, 16),
                                   (O.LAT_3D, 32)])
def test_large_lattices_match_reference(lat, L):
    """The configurations' lattice sizes (2D L=32/64, 3D L=16/32): spins and
    float energies after 1, 10 and 25 sweeps, at two temperatures."""
    r = O.RefSystem(lat, L, 1.0, 0.0)
    o = O.OracleSystem(lat, L, 1.0, 0.0, O.MODE_MT)
    for x in (r, o):
        x.set_seed(3)
        x.init_J()
        x.set_seed(4)
        x.init_rand()
    for n, T in ((1, 1.0), (9, 1.0), (15, 0.4)):
        r.set_T(T)
        o.set_T(T)
        r.sweep(n)
        o.sweep(n)
        assert np.array_equal(r.state()[0], o.spins())
        assert np.array_equal(r.measure_float(), o.measure_float())


def test_init_order_and_swap_match_reference():
    a, b = O.RefSystem(O.LAT_3D, 4), O.RefSystem(O.LAT_3D, 4)
    c, d = O.OracleSystem(O.LAT_3D, 4, mode=O.MODE_MT), O.OracleSystem(O.LAT_3D, 4, mode=O.MODE_MT)
    for x, seed in ((a, 1), (b, 2), (c, 1), (d, 2)):
        x.set_seed(seed)
        x.init_rand()
    a.swap(b, 0x00FF00FF00FF00F1)
    c.swap(d, 0x00FF00FF00FF00F1)
    assert np.array_equal(a.state()[0], c.spins()) and np.array_equal(b.state()[0], d.spins())
    a.init_order()
    c.init_order()
    assert np.array_equal(a.state()[0], c.spins())


@pytest.mark.parametrize("lat,L,n", [(O.LAT_3D, 4, 5), (O.LAT_2D, 8, 4), (O.LAT_2D_OPEN_X, 6, 3)])
def test_parallel_tempering_matches_reference(lat, L, n):
    T = list(np.geomspace(0.5, 2.0, n))[::-1]  # the template sorts them
    rs = [O.RefSystem(lat, L) for _ in range(n)]
    os_ = [O.OracleSystem(lat, L, mode=O.MODE_MT) for _ in range(n)]
    for x in rs + os_:
        x.set_seed(5)
        x.init_J()
        x.set_seed(6)
        x.init_rand()
    rp, op = O.RefPT(rs, T, 1), O.OraclePT(os_, T, 1)
    for _ in range(40):
        pr, mr = rp.step(0)
        po, mo, _r = op.step(0)
        assert (pr, mr) == (po, mo)
    for r, o in zip(rs, os_):
        assert np.array_equal(r.state()[0], o.spins())
    acc = [float(line.split(":")[1]) for line in rp.print_swap().strip().splitlines()]
    # print_swap writes with the stream default of 6 significant digits
    assert np.allclose(acc, op.acceptance(), rtol=1e-5, atol=0)


@pytest.mark.parametrize("lat,L", [(O.LAT_2D, 8), (O.LAT_3D, 4)])
def test_annealing_matches_reference(lat, L):
    r = O.RefSystem(lat, L, 3.0)
    o = O.OracleSystem(lat, L, 3.0, mode=O.MODE_MT)
    for x in (r, o):
        x.set_seed(1)
        x.init_J()
        x.set_seed(2)
        x.init_rand()
    a = r.anneal(3.0, 0.9, 8, 15, 1)
    b, _ = o.anneal(3.0, 0, 0.9, 8, 15, 1)
    assert np.array_equal(a, b)
    assert np.array_equal(r.state()[0], o.spins())
