#!/usr/bin/env python
"""Fixture generator: the five workload configurations run by the oracle.

Writes tests/golden/configs/<name>.npz, one file per configuration, from
the oracle's restatement (PHILOX mode: the engine's semantics) and, for the
mt19937_64 case, from the reference's own CPU classes compiled by
oracle/Makefile (oracle/_ref). The GPU tests in tests/test_gpu_configs.py
compare the engine with these files at the configurations' full sizes;
tests/test_config_golden.py re-derives a cheap prefix of each file from the
oracle on the CPU, so a fixture cannot drift from the oracle unnoticed.

Spin words are stored as SHA-256 digests of their little-endian bytes in the
reference's row-major site order (32 KB-2 MB per lattice would not be small
fixtures); energies, exchange pairs and masks are stored in full.

  c1_philox  2D L=64 periodic, J seed 1, spins seed 2, T=1.0, 10,000 sweeps:
             spins and integer -H every 1,000 sweeps (oracle, PHILOX).
  c1_mt      the same run in the reference's mt19937_64 stream: spins and the
             float measure() of cpu_2d itself every 1,000 sweeps (oracle/_ref).
  c2         3D L=32, J seed 3, spins seed 3, linear T 3.0 -> 0.2 over 200
             steps of 100 sweeps, -H measured every sweep: the running max per
             replica, the last -H of every step, the final spins.
  c3         3D L=16, seed 4, 32 temperatures geometric over 0.5-2.0, one sweep
             + one exchange attempt per sweep, 1,000 sweeps: every pair and
             mask, acceptance per pair, the energy histogram of every slot
             (all sweeps, before the exchange), final spins of every slot.
  c4_sample  the batched mix's first two instances of each of its ten shapes
             (bench.c4_instances(4096)), 16 slots, 100 sweeps with an exchange
             per sweep: pairs, masks, acceptance, final spins of every slot.

Run from the repository root (takes a few minutes on 8 cores):
  python tests/golden/gen_config_golden.py
"""
from __future__ import annotations

import hashlib
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "configs")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

C1_SWEEPS, C1_EVERY = 10_000, 1_000
C2_STEPS, C2_SWEEPS = 200, 100
C3_L, C3_SLOTS, C3_SWEEPS = 16, 32, 1_000
C4_SWEEPS = 100


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def c2_schedule():
    return [3.0 + (0.2 - 3.0) * k / (C2_STEPS - 1) for k in range(C2_STEPS)]


def c3_ladder():
    return list(np.geomspace(0.5, 2.0, C3_SLOTS))


def c4_picks():
    """Indices into bench.c4_instances(4096): the first two of each shape."""
    import bench

    insts = bench.c4_instances(4096)
    seen: dict = {}
    picks = []
    for i, (lat, L, _) in enumerate(insts):
        if seen.get((lat, L), 0) < 2:
            seen[(lat, L)] = seen.get((lat, L), 0) + 1
            picks.append(i)
    assert len(picks) == 20
    return picks, insts


def gen_c1_philox():
    from oracle import oracle as O

    o = O.OracleSystem(O.LAT_2D, 64, 1.0, 0.0, O.MODE_PHILOX)
    o.set_seed(1)
    o.init_J()
    o.set_seed(2)
    o.init_rand()
    digests, E = [], []
    for _ in range(C1_SWEEPS // C1_EVERY):
        o.sweep(C1_EVERY)
        digests.append(digest(o.spins()))
        E.append(o.measure()[0])
    return "c1_philox", {"spins_sha": np.array(digests), "E": np.array(E, dtype=np.int64)}


def gen_c1_mt():
    from oracle import oracle as O

    r = O.RefSystem(O.LAT_2D, 64, 1.0, 0.0)
    r.set_seed(1)
    r.init_J()
    r.set_seed(2)
    r.init_rand()
    digests, E = [], []
    for _ in range(C1_SWEEPS // C1_EVERY):
        r.sweep(C1_EVERY)
        digests.append(digest(r.state()[0]))
        E.append(r.measure_float())
    return "c1_mt", {"spins_sha": np.array(digests), "E_float": np.array(E, dtype=np.float32)}


def gen_c2():
    from oracle import oracle as O

    o = O.OracleSystem(O.LAT_3D, 32, 3.0, 0.0, O.MODE_PHILOX)
    o.set_seed(3)
    o.init_J()
    o.set_seed(3)
    o.init_rand()
    Ts = c2_schedule()
    mn = None
    last = np.zeros((C2_STEPS, 64), dtype=np.float32)
    for k, T in enumerate(Ts):  # annealing<>::step over an explicit schedule, stride 1
        o.set_T(T)
        for _ in range(C2_SWEEPS):
            o.sweep(1)
            res = o.measure_float()
            mn = res.copy() if mn is None else np.maximum(mn, res)
        last[k] = res
    return "c2", {"Emax": mn.astype(np.int64), "E_step": last.astype(np.int64), "spins_sha": np.array([digest(o.spins())])}


def run_pt(lat, L, T, seed_J, seed, nsweeps, hist=False):
    from oracle import oracle as O

    systems = [O.OracleSystem(lat, L, mode=O.MODE_PHILOX) for _ in T]
    for s in systems:
        s.set_seed(seed_J)
        s.init_J()
        s.set_seed(seed)
        s.init_rand()
    pt = O.OraclePT(systems, T, 1)
    nb = (3 if lat == O.LAT_3D else 2) * systems[0].N - (L if lat == O.LAT_2D_OPEN_X else 0)
    H = np.zeros((len(T), nb + 1), dtype=np.int64) if hist else None
    pairs, masks = [], []
    for _ in range(nsweeps):
        p, m, _ = pt.step(0)
        pairs.append(p)
        masks.append(m)
        if hist:
            # the energies the step measured before its exchange
            E = pt.energies().astype(np.int64)
            for i in range(len(T)):
                np.add.at(H[i], (E[i] + nb) // 2, 1)
    out = {"pairs": np.array(pairs, dtype=np.int32), "masks": np.array(masks, dtype=np.uint64),
           "acceptance": pt.acceptance(), "spins_sha": np.array([digest(s.spins()) for s in systems]),
           "E_last": np.array([s.measure()[0] for s in systems], dtype=np.int64)}
    if hist:
        out["hist"] = H
    return out


def gen_c3():
    from oracle import oracle as O

    return "c3", run_pt(O.LAT_3D, C3_L, c3_ladder(), 4, 4, C3_SWEEPS, hist=True)


def gen_c4_one(i):
    import bench

    lat, L, seed = bench.c4_instances(4096)[i]
    T = list(bench.LADDER_3D if lat == 2 else bench.LADDER_2D)
    return i, run_pt(lat, L, T, seed, seed, C4_SWEEPS)


def main():
    from oracle import oracle as O

    if not O.ref_available():
        raise SystemExit("oracle/_ref is not built (make -f oracle/Makefile REF_SRC=<reference>/src)")
    os.makedirs(OUT, exist_ok=True)
    ctx = mp.get_context("spawn")
    picks, _ = c4_picks()
    with ctx.Pool(min(8, os.cpu_count() or 1)) as pool:
        big = [pool.apply_async(f) for f in (gen_c2, gen_c3, gen_c1_philox, gen_c1_mt)]
        c4 = pool.map(gen_c4_one, picks)
        results = [r.get() for r in big]
    for name, d in results:
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)
        print(name, {k: v.shape for k, v in d.items()})
    c4d = {"index": np.array([i for i, _ in c4], dtype=np.int32)}
    for key in ("pairs", "masks", "acceptance", "spins_sha", "E_last"):
        c4d[key] = np.stack([r[key] for _, r in c4])
    np.savez_compressed(os.path.join(OUT, "c4_sample.npz"), **c4d)
    print("c4_sample", {k: v.shape for k, v in c4d.items()})


if __name__ == "__main__":
    main()
