"""GPU parity at the workload configurations themselves, at full size.

Each test runs one configuration through the engine exactly as bench.py runs
it and compares with tests/golden/configs/<name>.npz, which
tests/golden/gen_config_golden.py made from the oracle (PHILOX mode) and, for
C1 in mt19937_64 mode, from the reference's own cpu_2d (oracle/_ref). Spin
words are compared through SHA-256 digests of the reference row-major layout;
energies, exchange pairs and masks in full; everything bit for bit.
"""
import hashlib
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden", "configs")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(HERE, "golden"))

import gen_config_golden as G  # noqa: E402


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def _c1(mode):
    from simulated_annealing_b200.system import GpuSystem

    g = GpuSystem("2d", 64, 1.0)
    if mode == "mt":
        g.set_rng_mode("mt19937_64")
    g.set_seed(1)
    g.init_J()
    g.set_seed(2)
    g.init_rand()
    return g


def test_c1_philox_every_1000_sweeps(sab):
    """C1: 2D L=64, 10,000 sweeps at T=1.0; spins and integer -H after every
    1,000 sweeps against the oracle."""
    f = gold("c1_philox")
    g = _c1("philox")
    for k in range(G.C1_SWEEPS // G.C1_EVERY):
        g.sweep(G.C1_EVERY)
        assert digest(g.get_spins()) == f["spins_sha"][k], k
        assert np.array_equal(g.measure_exact()[0], f["E"][k]), k


def test_c1_mt19937_every_1000_sweeps_matches_cpu_2d(sab):
    """C1 in the reference's own random stream: spins and cpu_2d's float
    measure() after every 1,000 sweeps, against the unmodified cpu_2d."""
    f = gold("c1_mt")
    g = _c1("mt")
    for k in range(G.C1_SWEEPS // G.C1_EVERY):
        g.sweep(G.C1_EVERY)
        assert digest(g.get_spins()) == f["spins_sha"][k], k
        assert np.array_equal(np.asarray(g.measure(), dtype=np.float32), f["E_float"][k]), k


def test_c2_full_anneal(sab):
    """C2: 3D L=32 anneal, linear T 3.0 -> 0.2 over 200 steps x 100 sweeps,
    -H every sweep: the running max per replica, the last -H of all 200 steps
    and the final spins."""
    from simulated_annealing_b200.system import GpuSystem

    f = gold("c2")
    g = GpuSystem("3d", 32, 3.0)
    g.set_seed(3)
    g.init_J()
    g.set_seed(3)
    g.init_rand()
    mn, stepE = g.anneal(G.c2_schedule(), G.C2_SWEEPS, 1)
    assert np.array_equal(np.asarray(mn).astype(np.int64), f["Emax"])
    assert np.array_equal(np.asarray(stepE).astype(np.int64), f["E_step"])
    assert digest(g.get_spins()) == f["spins_sha"][0]


def _check_pt(b, i, f, k=None):
    sel = (lambda key: f[key]) if k is None else (lambda key: f[key][k])
    pairs, masks = b.exchanges(i)
    assert np.array_equal(pairs, sel("pairs"))
    assert np.array_equal(masks.astype(np.uint64), sel("masks").astype(np.uint64))
    acc, att = b.acceptance(i)
    assert np.allclose(acc / np.maximum(att, 1) / 64.0, sel("acceptance"), rtol=0, atol=1e-12)
    for slot in range(len(sel("spins_sha"))):
        assert digest(b.spins(i, slot)) == sel("spins_sha")[slot], (i, slot)
        assert np.array_equal(b.measure(i, slot), sel("E_last")[slot]), (i, slot)


def test_c3_ensemble_32_temperatures(sab):
    """C3: 3D L=16 x 32 temperatures, an exchange attempt after every sweep,
    1,000 sweeps (in two launches): every pair and mask, acceptance per pair,
    the energy histogram of every slot, final spins and energies."""
    from simulated_annealing_b200.batch import Batch

    f = gold("c3")
    b = Batch()
    lad = b.add_ladder(G.c3_ladder())
    b.add_instance(O.LAT_3D, G.C3_L, ladder=lad, seed_J=4, seed=4)
    b.set_histograms(1)
    b.finalize()
    b.record_exchanges(G.C3_SWEEPS)
    b.run(400)
    b.run(G.C3_SWEEPS - 400)
    b.sync()
    _check_pt(b, 0, f)
    for slot in range(G.C3_SLOTS):
        assert np.array_equal(b.histogram(0, slot).astype(np.int64), f["hist"][slot]), slot
    b.close()


def test_c4_bench_batch_sample(sab):
    """C4: the bench's own 4,096-instance batch (same ladders, instance order,
    groups, clusters and streams), one run of 100 sweeps with an exchange per
    sweep; the first two instances of each of the ten shapes against the
    oracle's parallel_tempering<>."""
    import torch

    import bench

    f = gold("c4_sample")
    stream = torch.cuda.Stream()
    b = bench.build_c4_batch(bench.c4_instances(4096), stream.cuda_stream)
    b.record_exchanges(G.C4_SWEEPS)
    b.run(G.C4_SWEEPS)
    b.sync()
    for k, i in enumerate(f["index"]):
        _check_pt(b, int(i), f, k)
    b.close()
