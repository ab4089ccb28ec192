"""The mt19937_64 mode against the reference's own CPU classes.

In SA_RNG_MT19937_64 mode a system draws from one std::mt19937_64 generated on
the device and consumes it the way cpu_2d / cpu_2dp / cpu_3d do (seeding,
init_J, init_rand, one uniform draw per site update in their visiting order).
oracle/_ref holds those classes compiled unmodified from the reference
sources, so spins, couplings, energies, annealing minima and
parallel-tempering decisions must agree bit for bit.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref (reference CPU classes) not built")]

CASES = [(O.LAT_2D, 4), (O.LAT_2D, 16), (O.LAT_2D_OPEN_X, 2), (O.LAT_2D_OPEN_X, 10), (O.LAT_3D, 2),
         (O.LAT_3D, 4), (O.LAT_3D, 8)]


def _mt(lat, L, T=1.0, h=0.0):
    from simulated_annealing_b200.system import GpuSystem
    g = GpuSystem(lat, L, T, h)
    g.set_rng_mode("mt19937_64")
    return g


def _same(g, r):
    s, jx, jy, jz = r.state()
    assert np.array_equal(g.get_spins(), s)
    J = g.get_J()
    assert np.array_equal(J[0], jx) and np.array_equal(J[1], jy)
    if len(J) == 3:
        assert np.array_equal(J[2], jz)
    assert np.array_equal(np.asarray(g.measure(), dtype=np.float32), r.measure_float())


@pytest.mark.parametrize("lat,L", CASES)
@pytest.mark.parametrize("T,h", [(1.0, 0.0), (0.6, 0.4), (2.5, -1.0)])
def test_mt_stream_matches_reference_classes(sab, lat, L, T, h):
    g, r = _mt(lat, L, T, h), O.RefSystem(lat, L, T, h)
    for x in (g, r):
        x.set_seed(11)
        x.init_J()
        x.set_seed(22)
        x.init_rand()
    _same(g, r)
    for n in (1, 2, 5, 20):
        g.sweep(n)
        r.sweep(n)
        _same(g, r)
    g.set_T(0.3)
    r.set_T(0.3)
    g.sweep(7)
    r.sweep(7)
    _same(g, r)


@pytest.mark.parametrize("lat,L", [(O.LAT_2D, 32), (O.LAT_2D, 64), (O.LAT_2D_OPEN_X, 64), (O.LAT_3D, 16),
                                   (O.LAT_3D, 32)])
def test_mt_large_lattices_match_reference_classes(sab, lat, L):
    """The configurations' lattice sizes in the reference's random stream."""
    g, r = _mt(lat, L, 1.0), O.RefSystem(lat, L, 1.0)
    for x in (g, r):
        x.set_seed(3)
        x.init_J()
        x.set_seed(4)
        x.init_rand()
    _same(g, r)
    for n, T in ((1, 1.0), (9, 1.0), (40, 0.4)):
        g.set_T(T)
        r.set_T(T)
        g.sweep(n)
        r.sweep(n)
        _same(g, r)


@pytest.mark.parametrize("lat,L", [(O.LAT_2D, 8), (O.LAT_3D, 4), (O.LAT_2D_OPEN_X, 6)])
def test_mt_anneal_matches_reference_template(sab, lat, L):
    """annealing<> (geometric cooling, measure every sweep) on the reference
    classes vs the device anneal in MT mode over the same temperatures."""
    g, r = _mt(lat, L, 3.0), O.RefSystem(lat, L, 3.0)
    for x in (g, r):
        x.set_seed(1)
        x.init_J()
        x.set_seed(2)
        x.init_rand()
    nsteps, sweeps, alfa = 8, 15, 0.9
    Ts, t = [], 3.0
    for _ in range(nsteps):  # T *= alfa after every step (src/annealing.hpp:96)
        Ts.append(t)
        t = t * alfa
    mn, _ = g.anneal(Ts, sweeps, 1)
    ref = r.anneal(3.0, alfa, nsteps, sweeps, 1)
    assert np.array_equal(mn, ref)
    assert np.array_equal(g.get_spins(), r.state()[0])


@pytest.mark.parametrize("lat,L,n", [(O.LAT_2D, 6, 4), (O.LAT_3D, 4, 5)])
def test_mt_parallel_tempering_matches_reference(sab, lat, L, n):
    """parallel_tempering<> over MT-mode systems: the same exchange pairs and
    masks as the reference template over its own CPU classes."""
    from simulated_annealing_b200.drivers import ParallelTempering
    T = list(np.geomspace(0.5, 2.0, n))
    gs = [_mt(lat, L) for _ in range(n)]
    rs = [O.RefSystem(lat, L) for _ in range(n)]
    for x in gs + rs:
        x.set_seed(5)
        x.init_J()
        x.set_seed(6)
        x.init_rand()
    gp, rp = ParallelTempering(gs, T, 1), O.RefPT(rs, T[::-1], 1)
    for _ in range(30):
        assert gp.step(0) == rp.step(0)
    for g, r in zip(gs, rs):
        assert np.array_equal(g.get_spins(), r.state()[0])


def test_mt_checkpoint_continues_the_stream(sab):
    g, r = _mt(O.LAT_3D, 6, 0.8), O.RefSystem(O.LAT_3D, 6, 0.8)
    for x in (g, r):
        x.set_seed(3)
        x.init_J()
        x.set_seed(4)
        x.init_rand()
        x.sweep(3)
    blob = g.save()
    g.sweep(4)
    g.load(blob)  # back to the saved spins and generator position
    g.sweep(4)
    r.sweep(4)
    _same(g, r)
    assert g.rng_mode() == 1


def test_switching_back_to_philox_follows_the_oracle(sab):
    from simulated_annealing_b200.system import GpuSystem
    g = GpuSystem(O.LAT_2D, 8, 1.1)
    g.set_rng_mode("mt19937_64")
    g.set_rng_mode("philox")
    o = O.OracleSystem(O.LAT_2D, 8, 1.1, mode=O.MODE_PHILOX)
    for x in (g, o):
        x.set_seed(9)
        x.init_J()
        x.set_seed(10)
        x.init_rand()
        x.sweep(5)
    assert np.array_equal(g.get_spins(), o.spins())


@pytest.mark.parametrize("lat,L", [(O.LAT_2D, 6), (O.LAT_2D_OPEN_X, 8), (O.LAT_3D, 4)])
def test_reference_checkpoint_record_both_ways(sab, lat, L):
    """The engine writes the reference classes' save() record byte for byte,
    and a record the reference wrote continues here draw for draw."""
    g, r = _mt(lat, L, 1.3, 0.2), O.RefSystem(lat, L, 1.3, 0.2)
    for x in (g, r):
        x.set_seed(21)
        x.init_J()
        x.set_seed(22)
        x.init_rand()
        x.sweep(3)
    assert g.save_reference() == r.save()
    # reference -> engine: a fresh system picks up the stream mid-way
    from simulated_annealing_b200.system import GpuSystem
    h = GpuSystem(lat, L, 2.0)
    h.load_reference(r.save())
    assert h.rng_mode() == 1
    h.sweep(5)
    r.sweep(5)
    _same(h, r)
    # engine -> reference
    r2 = O.RefSystem(lat, L)
    r2.load(h.save_reference())
    h.sweep(4)
    r2.sweep(4)
    _same(h, r2)
