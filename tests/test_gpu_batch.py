"""GPU parity of the batched persistent engine against the oracle.

Each batched instance must reproduce, bit for bit, the reference's
parallel_tempering<> (src/parallel_tempering.hpp:81-115) over systems built as
its driver builds them (src/main_gpu.cu:262-276) -- restated by the oracle in
PHILOX mode: every exchange pair and mask, every spin word of every slot, the
acceptance counters; anneal instances reproduce annealing<> with a linear
schedule (running maximum of -H per replica, src/annealing.hpp:67-100).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# every batch test runs with the cluster-resident kernel and with the
# global-memory kernel
KERNELS = pytest.mark.parametrize("kernel", [0, 1], ids=["resident", "global"])


def oracle_pt(lat, L, T, seed_J, seed, nsweeps, interval=1):
    systems = [O.OracleSystem(lat, L, mode=O.MODE_PHILOX) for _ in T]
    for s in systems:
        s.set_seed(seed_J)
        s.init_J()
        s.set_seed(seed)
        s.init_rand()
    pt = O.OraclePT(systems, T, interval)
    steps = [pt.step(0) for _ in range(nsweeps // interval)]
    return systems, pt, steps


def check_instance(b, i, lat, L, T, seed_J, seed, nsweeps, interval=1):
    systems, pt, steps = oracle_pt(lat, L, T, seed_J, seed, nsweeps, interval)
    pairs, masks = b.exchanges(i)
    assert pairs.tolist() == [p for p, _, _ in steps]
    assert [int(m) for m in masks] == [m for _, m, _ in steps]
    for slot, s in enumerate(systems):
        assert np.array_equal(b.spins(i, slot), s.spins()), (i, slot)
        assert np.array_equal(b.measure(i, slot), s.measure()[0]), (i, slot)
    acc, att = b.acceptance(i)
    ref = pt.acceptance()
    assert np.allclose(acc / np.maximum(att, 1) / 64.0, ref, rtol=0, atol=1e-12)
    jo = systems[0].J()
    for a, c in zip(b.J(i), jo):
        assert np.array_equal(a, c)


@KERNELS
@pytest.mark.parametrize("nslots", [2, 3, 5, 8, 16, 32])
def test_pt_batch_all_lane_classes(sab, nslots, kernel):
    from simulated_annealing_b200.batch import Batch
    T = list(np.geomspace(0.4, 2.1, nslots))
    b = Batch(kernel)
    lad = b.add_ladder(T)
    specs = [(O.LAT_2D, 6, 11), (O.LAT_2D_OPEN_X, 8, 12), (O.LAT_3D, 4, 13), (O.LAT_3D, 6, 14)]
    for lat, L, s in specs:
        b.add_instance(lat, L, ladder=lad, seed_J=s, seed=s + 50)
    b.finalize()
    b.record_exchanges(64)
    b.run(5)
    b.run(4)  # continuation across launches
    b.sync()
    for i, (lat, L, s) in enumerate(specs):
        check_instance(b, i, lat, L, T, s, s + 50, 9)


@KERNELS
def test_c4_shapes_subset(sab, kernel):
    """One instance of each C4 shape, 16 geometric slots, 12 sweeps (the
    resident kernel runs them in clusters of 1, 2, 4 and 8 CTAs)."""
    from simulated_annealing_b200.batch import Batch
    b = Batch(kernel)
    l2 = b.add_ladder(np.geomspace(0.3, 1.6, 16))
    l3 = b.add_ladder(np.geomspace(0.5, 2.0, 16))
    specs = [(O.LAT_2D, L, 1000 + k) for k, L in enumerate([16, 24, 32, 48, 64])]
    specs += [(O.LAT_3D, L, 1005 + k) for k, L in enumerate([8, 12, 16, 20, 24])]
    for lat, L, s in specs:
        b.add_instance(lat, L, ladder=(l3 if lat == O.LAT_3D else l2), seed_J=s, seed=s)
    b.finalize()
    b.record_exchanges(32)
    b.run(12)
    b.sync()
    for i, (lat, L, s) in enumerate(specs):
        T = np.geomspace(0.5, 2.0, 16) if lat == O.LAT_3D else np.geomspace(0.3, 1.6, 16)
        check_instance(b, i, lat, L, list(T), s, s, 12)


@KERNELS
def test_exchange_interval(sab, kernel):
    from simulated_annealing_b200.batch import Batch
    T = [0.5, 0.8, 1.3]
    b = Batch(kernel)
    lad = b.add_ladder(T)
    b.add_instance(O.LAT_3D, 4, ladder=lad, seed_J=3, seed=4)
    b.finalize()
    b.set_exchange_interval(3)
    b.record_exchanges(16)
    b.run(9)
    b.sync()
    check_instance(b, 0, O.LAT_3D, 4, T, 3, 4, 9, interval=3)


@KERNELS
def test_anneal_instances_linear_schedule(sab, kernel):
    from simulated_annealing_b200.batch import Batch
    nsteps, per = 6, 5
    T0, T1 = 3.0, 0.2
    Ts = [T0 + (T1 - T0) * k / (nsteps - 1) for k in range(nsteps)]
    b = Batch(kernel)
    sch = b.add_schedule(Ts, per)
    specs = [(O.LAT_2D, 8, 21), (O.LAT_3D, 6, 22), (O.LAT_2D_OPEN_X, 10, 23)]
    for lat, L, s in specs:
        b.add_instance(lat, L, schedule=sch, seed_J=s, seed=s + 1)
    b.finalize()
    b.run(7)
    b.run(100)  # stops at the end of the schedule
    b.sync()
    for i, (lat, L, s) in enumerate(specs):
        o = O.OracleSystem(lat, L, mode=O.MODE_PHILOX)
        o.set_seed(s)
        o.init_J()
        o.set_seed(s + 1)
        o.init_rand()
        mn, _ = o.anneal(T0, 1, T1, nsteps, per, 1)
        E, done = b.anneal_result(i)
        assert done == nsteps * per
        assert np.array_equal(E.astype(np.float32), mn)
        assert np.array_equal(b.spins(i, 0), o.spins())


def test_bad_instances_rejected(sab):
    from simulated_annealing_b200._lib import SAError
    from simulated_annealing_b200.batch import Batch
    b = Batch()
    lad = b.add_ladder([1.0, 2.0])
    with pytest.raises(SAError):
        b.add_instance(O.LAT_2D, 7, ladder=lad, seed_J=1, seed=1)
    with pytest.raises(SAError):
        b.add_instance(O.LAT_3D, 128, ladder=lad, seed_J=1, seed=1)
    with pytest.raises(SAError):
        b.add_ladder(np.linspace(1, 2, 33))


@KERNELS
def test_large_single_slot_anneal_uses_big_clusters(sab, kernel):
    """3D L=32 and 2D L=128 single-slot anneals (serving-sized requests)."""
    from simulated_annealing_b200.batch import Batch
    Ts = [2.5, 1.5, 0.8]
    b = Batch(kernel)
    sch = b.add_schedule(Ts, 2)
    specs = [(O.LAT_3D, 32, 41), (O.LAT_2D, 128, 42)]
    for lat, L, s in specs:
        b.add_instance(lat, L, schedule=sch, seed_J=s, seed=s)
    b.finalize()
    b.run(6)
    b.sync()
    for i, (lat, L, s) in enumerate(specs):
        o = O.OracleSystem(lat, L, mode=O.MODE_PHILOX)
        o.set_seed(s)
        o.init_J()
        o.set_seed(s)
        o.init_rand()
        for T in Ts:
            o.set_T(T)
            o.sweep(2)
        assert np.array_equal(b.spins(i, 0), o.spins())


def test_uneven_cluster_row_split(sab):
    """Instances whose y-rows do not divide evenly over their cluster's CTAs
    (2D L=44 x 32 slots on 3 CTAs, 3D L=26 x 4 slots on 3 CTAs, a 3D L=46
    single-slot anneal on 4 CTAs) reproduce the oracle."""
    from simulated_annealing_b200.batch import Batch
    b = Batch()
    T32 = list(np.geomspace(0.3, 1.6, 32))
    T4 = list(np.geomspace(0.5, 2.0, 4))
    l32 = b.add_ladder(T32)
    l4 = b.add_ladder(T4)
    Ts = [2.5, 1.2]
    sch = b.add_schedule(Ts, 2)
    b.add_instance(O.LAT_2D, 44, ladder=l32, seed_J=61, seed=62)
    b.add_instance(O.LAT_3D, 26, ladder=l4, seed_J=63, seed=64)
    b.add_instance(O.LAT_3D, 46, schedule=sch, seed_J=65, seed=66)
    b.finalize()
    b.record_exchanges(16)
    b.run(3)
    b.run(2)
    b.sync()
    check_instance(b, 0, O.LAT_2D, 44, T32, 61, 62, 5)
    check_instance(b, 1, O.LAT_3D, 26, T4, 63, 64, 5)
    o = O.OracleSystem(O.LAT_3D, 46, mode=O.MODE_PHILOX)
    o.set_seed(65)
    o.init_J()
    o.set_seed(66)
    o.init_rand()
    mn, _ = o.anneal(2.5, 1, 1.2, 2, 2, 1)
    E, done = b.anneal_result(2)
    assert done == 4
    assert np.array_equal(E.astype(np.float32), mn)
    assert np.array_equal(b.spins(2, 0), o.spins())


def test_resident_groups(sab):
    """The C4 mix needs one launch per (lanes-per-site, cluster size) group."""
    from simulated_annealing_b200.batch import Batch
    b = Batch()
    lad = b.add_ladder(np.geomspace(0.5, 2.0, 16))
    for L in (8, 12, 16, 20, 24):
        b.add_instance(O.LAT_3D, L, ladder=lad, seed_J=L, seed=L)
    b.finalize()
    assert 1 <= b.launches_per_run() <= 5


@pytest.mark.parametrize("lat,L,nslots", [(O.LAT_3D, 6, 8), (O.LAT_2D, 10, 5)])
def test_energy_histograms_and_decisions(sab, lat, L, nslots):
    """C3-style run: exchange every sweep, per-slot energy histograms (taken
    before the exchange, like the reference's E[]), acceptance and every
    decision, against the oracle's parallel_tempering<> restatement."""
    from simulated_annealing_b200.batch import Batch
    T = list(np.geomspace(0.5, 2.0, nslots))
    sweeps = 40
    b = Batch()
    lad = b.add_ladder(T)
    b.add_instance(lat, L, ladder=lad, seed_J=4, seed=4)
    b.set_histograms(1)
    b.finalize()
    b.record_exchanges(sweeps)
    b.run(15)
    b.run(sweeps - 15)
    b.sync()
    systems = [O.OracleSystem(lat, L, mode=O.MODE_PHILOX) for _ in T]
    for s in systems:
        s.set_seed(4)
        s.init_J()
        s.set_seed(4)
        s.init_rand()
    pt = O.OraclePT(systems, T, 1)
    N = L ** 3 if lat == O.LAT_3D else L * L
    nbonds = (3 if lat == O.LAT_3D else 2) * N
    hist = np.zeros((nslots, nbonds + 1), dtype=np.int64)
    steps = []
    for _ in range(sweeps):
        steps.append(pt.step(0))
        E = pt.energies().astype(np.int64)
        for s in range(nslots):
            np.add.at(hist[s], (E[s] + nbonds) // 2, 1)
    pairs, masks = b.exchanges(0)
    assert pairs.tolist() == [p for p, _, _ in steps]
    assert [int(m) for m in masks] == [m for _, m, _ in steps]
    for s in range(nslots):
        assert np.array_equal(b.histogram(0, s), hist[s]), s
    acc, att = b.acceptance(0)
    assert np.allclose(acc / np.maximum(att, 1) / 64.0, pt.acceptance(), rtol=0, atol=1e-12)


@pytest.mark.parametrize("stride", [1, 3])
def test_fused_single_slot_measurement_full_batch(sab, stride):
    """Single-slot 3D anneals in a batch too large to spread over extra SMs
    count each measured sweep's energy inside the half-sweeps (lagged by half a
    sweep); the running maxima and spins must still match annealing<>."""
    from simulated_annealing_b200.batch import Batch
    nsteps, per = 3, 4
    T0, T1 = 2.8, 0.4
    Ts = [T0 + (T1 - T0) * k / (nsteps - 1) for k in range(nsteps)]
    b = Batch()
    b.set_measure_stride(stride)
    sch = b.add_schedule(Ts, per)
    specs = [(O.LAT_3D, 8 if k % 3 else 10, 300 + k) for k in range(96)]
    for lat, L, s in specs:
        b.add_instance(lat, L, schedule=sch, seed_J=s, seed=s + 1)
    b.finalize()
    b.run(5)
    b.run(100)
    b.sync()
    for i in (0, 1, 2, 47, 95):
        lat, L, s = specs[i]
        o = O.OracleSystem(lat, L, mode=O.MODE_PHILOX)
        o.set_seed(s)
        o.init_J()
        o.set_seed(s + 1)
        o.init_rand()
        mn, _ = o.anneal(T0, 1, T1, nsteps, per, stride)
        E, done = b.anneal_result(i)
        assert done == nsteps * per
        assert np.array_equal(E.astype(np.float32), mn), i
        assert np.array_equal(b.spins(i, 0), o.spins()), i


@pytest.mark.parametrize("L,stride", [(40, 1), (42, 3), (64, 1)])
def test_wide_single_slot_anneal(sab, L, stride):
    """A lone single-slot 3D anneal of L >= 40 runs wide (every column of a
    colour a lane group anywhere on the GPU, three launches per sweep); its
    running maxima and spins match annealing<> and the resident form."""
    from simulated_annealing_b200.batch import KERNEL_AUTO, KERNEL_NO_WIDE, Batch
    nsteps, per = 3, 3
    T0, T1 = 2.8, 0.4
    Ts = [T0 + (T1 - T0) * k / (nsteps - 1) for k in range(nsteps)]
    o = O.OracleSystem(O.LAT_3D, L, mode=O.MODE_PHILOX)
    o.set_seed(77)
    o.init_J()
    o.set_seed(78)
    o.init_rand()
    mn, _ = o.anneal(T0, 1, T1, nsteps, per, stride)
    for kernel in (KERNEL_AUTO, KERNEL_NO_WIDE):
        b = Batch(kernel)
        b.set_measure_stride(stride)
        sch = b.add_schedule(Ts, per)
        b.add_instance(O.LAT_3D, L, schedule=sch, seed_J=77, seed=78)
        b.finalize()
        b.run(4)  # ends inside a step
        b.run(100)  # stops at the end of the schedule
        b.sync()
        E, done = b.anneal_result(0)
        assert done == nsteps * per
        assert np.array_equal(E.astype(np.float32), mn), kernel
        assert np.array_equal(b.spins(0, 0), o.spins()), kernel
        b.close()


def test_large_anneal_in_a_full_batch(sab):
    """A large single-slot 3D anneal beside many other instances stays on its
    cluster (the wide form is for a GPU with idle SMs); every instance still
    matches annealing<>."""
    from simulated_annealing_b200.batch import Batch
    nsteps, per = 2, 3
    T0, T1 = 2.5, 0.5
    Ts = [T0 + (T1 - T0) * k / (nsteps - 1) for k in range(nsteps)]
    b = Batch()
    sch = b.add_schedule(Ts, per)
    specs = [(O.LAT_3D, 48, 500)] + [(O.LAT_3D, 8, 501 + k) for k in range(300)]
    for lat, L, s in specs:
        b.add_instance(lat, L, schedule=sch, seed_J=s, seed=s + 1)
    b.finalize()
    b.run(5)
    b.run(100)
    b.sync()
    for i in (0, 1, 299):
        lat, L, s = specs[i]
        o = O.OracleSystem(lat, L, mode=O.MODE_PHILOX)
        o.set_seed(s)
        o.init_J()
        o.set_seed(s + 1)
        o.init_rand()
        mn, _ = o.anneal(T0, 1, T1, nsteps, per, 1)
        E, done = b.anneal_result(i)
        assert done == nsteps * per
        assert np.array_equal(E.astype(np.float32), mn), i
        assert np.array_equal(b.spins(i, 0), o.spins()), i
