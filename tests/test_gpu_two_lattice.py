"""The reference GPU systems' 128-replica shape (two-lattice trick).

gpu_2d / gpu_3d update every site of one lattice from the other
(src/gpu_2d.cu:109-120), which carries two configurations: A updates colour 0
then colour 1, B colour 1 then colour 0 (each half-sweep drawing the next
Philox number of every site). The engine's first-colour option gives B; the
oracle has the same option. TwoLatticeSystem / b200_sys128 pair an A and a B
system with the same couplings: measure() is A's 64 values then B's, swap()
takes a mask word for each, the parallel-tempering driver makes one mask word
per 64 replicas from one shared uniform (src/parallel_tempering.hpp:141-162).
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "simulated_annealing_b200", "sa_anneal")


def _oracle(lat, L, first, seed_J=3, seed=4, T=1.0, h=0.0):
    o = O.OracleSystem(lat, L, T, h, O.MODE_PHILOX)
    o.set_first_colour(first)
    o.set_seed(seed_J)
    o.init_J()
    o.set_seed(seed)
    o.init_rand()
    return o


@pytest.mark.parametrize("lat,L", [(O.LAT_2D_OPEN_X, 8), (O.LAT_2D, 16), (O.LAT_3D, 6), (O.LAT_3D, 12)])
@pytest.mark.parametrize("T,h", [(1.0, 0.0), (0.6, 0.3)])
def test_first_colour_one_matches_oracle(sab, lat, L, T, h):
    from simulated_annealing_b200.system import GpuSystem

    g = GpuSystem(lat, L, T, h)
    g.set_first_colour(1)
    assert g.first_colour() == 1
    g.set_seed(3)
    g.init_J()
    g.set_seed(4)
    g.init_rand()
    o = _oracle(lat, L, 1, T=T, h=h)
    assert np.array_equal(g.get_spins(), o.spins())
    for n in (1, 3, 20):  # 20: a run long enough for the resident path of colour-0-first systems
        g.sweep(n)
        o.sweep(n)
        assert np.array_equal(g.get_spins(), o.spins())
        assert np.array_equal(g.measure_exact()[0], o.measure()[0])
    # the two orders differ: B is not A
    a = _oracle(lat, L, 0, T=T, h=h)
    a.sweep(24)
    assert not np.array_equal(a.spins(), o.spins())


def test_first_colour_rules(sab):
    from simulated_annealing_b200._lib import SAError
    from simulated_annealing_b200.system import GpuSystem

    g = GpuSystem("3d", 4)
    g.set_rng_mode("mt19937_64")
    with pytest.raises(SAError):
        g.set_first_colour(1)
    h = GpuSystem("3d", 4)
    h.set_first_colour(1)
    with pytest.raises(SAError):
        h.set_rng_mode("mt19937_64")
    with pytest.raises(SAError):
        h.set_first_colour(2)
    # the checkpoint record keeps the order
    h.set_seed(5)
    h.init_J()
    h.init_rand()
    h.sweep(3)
    blob = h.save()
    k = GpuSystem("3d", 4)
    k.load(blob)
    assert k.first_colour() == 1
    h.sweep(4)
    k.sweep(4)
    assert np.array_equal(h.get_spins(), k.get_spins())


def test_anneal_of_a_first_colour_one_system(sab):
    from simulated_annealing_b200.system import GpuSystem

    g = GpuSystem("3d", 8, 2.0)
    g.set_first_colour(1)
    g.set_seed(3)
    g.init_J()
    g.set_seed(4)
    g.init_rand()
    Ts = [2.0, 1.4, 0.9, 0.5]
    mn, stepE = g.anneal(Ts, 5, 1)
    o = _oracle(O.LAT_3D, 8, 1, T=2.0)
    ref = None
    for k, T in enumerate(Ts):
        o.set_T(T)
        for _ in range(5):
            o.sweep(1)
            e = o.measure_float()
            ref = e if ref is None else np.maximum(ref, e)
        assert np.array_equal(stepE[k], o.measure()[0])
    assert np.array_equal(mn, ref)


@pytest.mark.parametrize("lat,L", [(O.LAT_2D_OPEN_X, 8), (O.LAT_3D, 4)])
def test_128_replica_system_and_pt(sab, lat, L):
    from simulated_annealing_b200.drivers import ParallelTempering
    from simulated_annealing_b200.system import TwoLatticeSystem

    T = [0.5, 1.0, 1.7]
    sys128 = []
    for _ in T:
        s = TwoLatticeSystem(lat, L)
        s.set_seed(3)
        s.init_J()
        s.set_seed(4)
        s.init_rand()
        sys128.append(s)
    A = [_oracle(lat, L, 0) for _ in T]
    B = [_oracle(lat, L, 1) for _ in T]
    e = np.asarray(sys128[0].measure(), dtype=np.float32)
    assert e.size == 128
    assert np.array_equal(e[:64], A[0].measure_float()) and np.array_equal(e[64:], B[0].measure_float())
    ep = ParallelTempering(sys128, T, 1)
    pa, pb = O.OraclePT(A, T, 1), O.OraclePT(B, T, 1)
    for _ in range(12):
        pair, masks = ep.step(0)
        qa, ma, _ = pa.step(0)
        qb, mb, _ = pb.step(0)
        assert pair == qa == qb
        assert list(masks) == [ma, mb]
    for s, a, b in zip(sys128, A, B):
        assert np.array_equal(s.a.get_spins(), a.spins()) and np.array_equal(s.b.get_spins(), b.spins())
    # acceptance: accepted replicas of both words over 64 per attempt, as the template counts
    acc_ref = pa.acceptance() + pb.acceptance()
    assert np.allclose(ep.acceptance(), acc_ref, rtol=0, atol=1e-12)
    # checkpoint of the pair driver resumes
    blob = ep.save()
    want = [ep.step(0) for _ in range(3)]
    fresh = []
    for _ in T:
        s = TwoLatticeSystem(lat, L)
        fresh.append(s)
    ep2 = ParallelTempering(fresh, T, 1)
    ep2.load(blob)
    assert [ep2.step(0) for _ in range(3)] == want


@pytest.mark.skipif(not os.path.exists(EXE), reason="sa_anneal not built")
def test_cli_two_lattice_anneal_prints_128(sab, tmp_path):
    r = subprocess.run([EXE, "--two-lattice", "-d", "3", "-L", "4", "-T", "1.5", "-a", "0.8", "-s", "2", "-S", "2",
                        "--seed", "6"], capture_output=True, text=True, cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stderr
    rows = [np.array([float(v) for v in ln.split("\t") if v.strip()], dtype=np.float32)
            for ln in r.stdout.splitlines() if ln and not ln.startswith("#")]
    A, B = _oracle(O.LAT_3D, 4, 0, 6, 6, 1.5), _oracle(O.LAT_3D, 4, 1, 6, 6, 1.5)
    want, T = [], 1.5
    for _ in range(2):
        for o in (A, B):
            o.set_T(T)
        for _ in range(2):
            A.sweep(1)
            B.sweep(1)
            want.append(np.concatenate([A.measure_float(), B.measure_float()]))
        T *= 0.8
    assert len(rows) == 4
    for g, w in zip(rows, want):
        assert np.array_equal(g, w)
    t = subprocess.run([EXE, "--two-lattice", "-t", "-d", "2p", "-L", "32", "-s", "10", "-T", "1"],
                       capture_output=True, text=True, cwd=str(tmp_path), timeout=300)
    assert t.returncode == 0, t.stderr
