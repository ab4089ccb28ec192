"""The configuration fixtures against the oracle, on the CPU.

tests/golden/configs/*.npz hold the oracle's (and, for C1 in mt19937_64
mode, the reference's own) results at the five workload configurations; the
GPU tests compare the engine with them. Here a cheap prefix of each fixture
is recomputed from the oracle, so a fixture that drifted from the oracle (or
an oracle that drifted from the reference) fails on the CPU.
"""
import hashlib
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "configs")
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, os.path.dirname(HERE))

import gen_config_golden as G  # noqa: E402


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def test_c1_philox_first_dump(oracle):
    f = gold("c1_philox")
    assert f["spins_sha"].shape == (10,) and f["E"].shape == (10, 64)
    o = O.OracleSystem(O.LAT_2D, 64, 1.0, 0.0, O.MODE_PHILOX)
    o.set_seed(1)
    o.init_J()
    o.set_seed(2)
    o.init_rand()
    o.sweep(G.C1_EVERY)
    assert digest(o.spins()) == f["spins_sha"][0]
    assert np.array_equal(o.measure()[0], f["E"][0])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_c1_mt_first_dump_is_cpu_2d_and_the_oracle(oracle):
    """The mt19937_64 fixture is the reference's cpu_2d; the oracle's MT mode
    reproduces its first dump."""
    f = gold("c1_mt")
    r = O.RefSystem(O.LAT_2D, 64, 1.0, 0.0)
    o = O.OracleSystem(O.LAT_2D, 64, 1.0, 0.0, O.MODE_MT)
    for x in (r, o):
        x.set_seed(1)
        x.init_J()
        x.set_seed(2)
        x.init_rand()
        x.sweep(G.C1_EVERY)
    assert digest(r.state()[0]) == digest(o.spins()) == f["spins_sha"][0]
    assert np.array_equal(r.measure_float(), f["E_float"][0])
    assert np.array_equal(o.measure_float(), f["E_float"][0])


def test_c2_first_step(oracle):
    f = gold("c2")
    assert f["E_step"].shape == (G.C2_STEPS, 64)
    o = O.OracleSystem(O.LAT_3D, 32, 3.0, 0.0, O.MODE_PHILOX)
    o.set_seed(3)
    o.init_J()
    o.set_seed(3)
    o.init_rand()
    o.set_T(G.c2_schedule()[0])
    o.sweep(G.C2_SWEEPS)
    assert np.array_equal(o.measure()[0], f["E_step"][0])
    # the running max can only be at or above every step's last energy
    assert np.all(f["Emax"] >= f["E_step"].max(axis=0))


def test_c3_first_exchanges(oracle):
    f = gold("c3")
    assert f["pairs"].shape == (G.C3_SWEEPS,) and f["hist"].shape[0] == G.C3_SLOTS
    # every slot's histogram counts 64 replicas per sweep
    assert np.all(f["hist"].sum(axis=1) == 64 * G.C3_SWEEPS)
    n = 6
    systems = [O.OracleSystem(O.LAT_3D, G.C3_L, mode=O.MODE_PHILOX) for _ in range(G.C3_SLOTS)]
    for s in systems:
        s.set_seed(4)
        s.init_J()
        s.set_seed(4)
        s.init_rand()
    pt = O.OraclePT(systems, G.c3_ladder(), 1)
    for k in range(n):
        p, m, _ = pt.step(0)
        assert p == f["pairs"][k] and m == int(f["masks"][k]), k


def test_c4_sample_smallest_instance(oracle):
    import bench

    f = gold("c4_sample")
    insts = bench.c4_instances(4096)
    picks, _ = G.c4_picks()
    assert f["index"].tolist() == picks
    shapes = {insts[i][:2] for i in picks}
    assert len(shapes) == 10  # every shape of the mix
    k = next(k for k, i in enumerate(picks) if insts[i][:2] == (0, 16))
    lat, L, seed = insts[picks[k]]
    r = G.run_pt(lat, L, list(bench.LADDER_2D), seed, seed, G.C4_SWEEPS)
    for key in ("pairs", "masks", "spins_sha", "E_last"):
        assert np.array_equal(r[key], f[key][k]), key
