"""Parallel-tempering checkpoints (.tempsys) and adaptive temperatures
against the reference's own template.

In mt19937_64 mode the engine's ParallelTempering writes the stream that
parallel_tempering<cpu_sys>::save writes over cpu_2d / cpu_3d systems
(src/parallel_tempering.hpp:280-318), byte for byte; a run saved by either
program resumes in the other draw for draw (:320-377). update_T inserts the
same temperatures and clones the same systems (:384-413).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref (reference CPU classes) not built")]

FNAME = "unused_%"  # the name the oracle's reference driver gives its template


def _gpu(lat, L, n, mode="mt19937_64", seeds=(3, 4)):
    from simulated_annealing_b200.system import GpuSystem

    out = []
    for _ in range(n):
        g = GpuSystem(lat, L)
        g.set_rng_mode(mode)
        g.set_seed(seeds[0])
        g.init_J()
        g.set_seed(seeds[1])
        g.init_rand()
        out.append(g)
    return out


def _ref(lat, L, n, seeds=(3, 4)):
    out = []
    for _ in range(n):
        r = O.RefSystem(lat, L)
        r.set_seed(seeds[0])
        r.init_J()
        r.set_seed(seeds[1])
        r.init_rand()
        out.append(r)
    return out


CASES = [(O.LAT_3D, 4, [0.5, 0.9, 1.4, 2.0]), (O.LAT_2D, 8, [0.4, 1.0, 1.9]),
         (O.LAT_2D_OPEN_X, 6, [0.7, 1.1, 1.6, 2.2, 3.0])]


@pytest.mark.parametrize("lat,L,T", CASES)
def test_tempsys_stream_is_the_templates(sab, lat, L, T):
    from simulated_annealing_b200.drivers import ParallelTempering

    rp = O.RefPT(_ref(lat, L, len(T)), T, 1)
    ep = ParallelTempering(_gpu(lat, L, len(T)), T, 1, FNAME)
    for _ in range(7):
        assert rp.step(0)[1] == ep.step(0)[1]
    assert ep.save() == rp.save()


@pytest.mark.parametrize("lat,L,T", CASES)
def test_tempsys_resumes_across_programs(sab, lat, L, T):
    from simulated_annealing_b200.drivers import ParallelTempering

    rs = _ref(lat, L, len(T))
    rp = O.RefPT(rs, T, 1)
    gs = _gpu(lat, L, len(T))
    ep = ParallelTempering(gs, T, 1, FNAME)
    for _ in range(6):
        rp.step(0)
        ep.step(0)
    from_ref, from_eng = rp.save(), ep.save()
    # the engine resumes the reference's run, the reference the engine's
    gs2 = _gpu(lat, L, len(T), seeds=(90, 91))
    ep2 = ParallelTempering(gs2, T, 1, "other_%")
    ep2.load(from_ref)
    rs2 = _ref(lat, L, len(T), seeds=(92, 93))
    rp2 = O.RefPT(rs2, T, 1)
    rp2.load(from_eng)
    for _ in range(5):
        a, b, c, d = rp.step(0), ep.step(0), ep2.step(0), rp2.step(0)
        assert a == b == c == d
    for r, g, g2, r2 in zip(rs, gs, gs2, rs2):
        s = r.state()[0]
        assert np.array_equal(g.get_spins(), s) and np.array_equal(g2.get_spins(), s)
        assert np.array_equal(r2.state()[0], s)


def test_tempsys_philox_mode_roundtrip(sab):
    from simulated_annealing_b200.drivers import ParallelTempering

    T = [0.6, 1.0, 1.5, 2.3]
    ep = ParallelTempering(_gpu(O.LAT_3D, 6, 4, mode="philox"), T, 1, "x_%")
    for _ in range(5):
        ep.step(0)
    blob = ep.save()
    want = [ep.step(0) for _ in range(4)]
    ep2 = ParallelTempering(_gpu(O.LAT_3D, 6, 4, mode="philox", seeds=(50, 51)), T, 1, "y_%")
    ep2.load(blob)
    assert ep2.fname == "x_%"
    assert [ep2.step(0) for _ in range(4)] == want
    for a, b in zip(ep.sys, ep2.sys):
        assert np.array_equal(a.get_spins(), b.get_spins())


def test_update_T_matches_reference(sab):
    """Wide gaps in the ladder give pairs with acceptance below 0.3; update_T
    inserts their midpoints on both sides, and the runs stay identical."""
    from simulated_annealing_b200.drivers import ParallelTempering

    T = [0.3, 0.6, 1.5, 3.5]
    rs = _ref(O.LAT_3D, 4, len(T))
    gs = _gpu(O.LAT_3D, 4, len(T))
    rp = O.RefPT(rs, T, 1)
    ep = ParallelTempering(gs, T, 1, FNAME)
    for _ in range(40):
        assert rp.step(0)[1] == ep.step(0)[1]
    before = len(ep.T)
    rp.update_T()
    ep.update_T()
    assert len(ep.T) > before
    assert ep.print_swap() == rp.print_swap()
    for _ in range(30):
        _, mr = rp.step(0)
        pe, me = ep.step(0)
        assert mr == me
        assert ep.T[pe] == pytest.approx(rp.last_T(), abs=0, rel=0)
    assert ep.print_swap() == rp.print_swap()
    for r, g in zip(rs, gs):
        assert np.array_equal(g.get_spins(), r.state()[0])
