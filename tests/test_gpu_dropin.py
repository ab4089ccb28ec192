"""Drop-in proof: the reference's own templates drive the engine.

tests/dropin/_build/dropin is compiled (tests/dropin/Makefile) from the
reference's unmodified annealing.hpp / parallel_tempering.hpp / gpu_sys.cuh
and this repository's include/sa_b200_sys.hpp. Its exchanges, energies,
spins, acceptance and running minimum must equal the oracle's restatement of
the same templates over the same systems.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(__file__), "dropin", "_build", "dropin")
needs_bin = pytest.mark.skipif(not os.path.exists(BIN), reason="drop-in program not built (needs the reference tree)")


def run(*args):
    out = subprocess.run([BIN, *map(str, args)], check=True, capture_output=True, text=True).stdout
    return [line.split() for line in out.strip().splitlines()]


@needs_bin
@pytest.mark.parametrize("lat,L,T", [(O.LAT_3D, 4, [2.0, 0.55, 0.8, 1.3, 1.0]),
                                      (O.LAT_2D_OPEN_X, 8, [0.4, 0.9, 1.7]),
                                      (O.LAT_2D, 6, [0.3, 0.6, 1.2, 2.4])])
def test_parallel_tempering_template_on_b200(lat, L, T):
    steps = 25
    lines = run("pt", lat, L, len(T), 17, 29, steps, *T)
    xs = [(int(l[1]), int(l[2])) for l in lines if l[0] == "X"]
    systems = [O.OracleSystem(lat, L, mode=O.MODE_PHILOX) for _ in T]
    for s in systems:
        s.set_seed(17)
        s.init_J()
        s.set_seed(29)
        s.init_rand()
    pt = O.OraclePT(systems, T, 1)
    ref = [pt.step(0)[:2] for _ in range(steps)]
    assert xs == ref
    for l in lines:
        if l[0] == "E":
            i = int(l[1])
            assert np.array_equal(np.array(l[2:], dtype=np.float32), systems[i].measure_float())
        if l[0] == "S":
            i = int(l[1])
            assert np.array_equal(np.array(l[2:], dtype=np.uint64), systems[i].spins())
    acc = [float(x) for l in lines if l[0] == "A" for x in l[1:]]
    assert np.allclose(acc, pt.acceptance(), rtol=1e-5, atol=0)


@needs_bin
@pytest.mark.parametrize("lat,L", [(O.LAT_2D, 8), (O.LAT_3D, 6)])
def test_annealing_template_on_b200(lat, L):
    lines = run("anneal", lat, L, 3, 4, 3.0, 0.85, 7, 12)
    mn = np.array([x for l in lines if l[0] == "M" for x in l[1:]], dtype=np.float32)
    spins = np.array([x for l in lines if l[0] == "S" for x in l[2:]], dtype=np.uint64)
    o = O.OracleSystem(lat, L, 3.0, mode=O.MODE_PHILOX)
    o.set_seed(3)
    o.init_J()
    o.set_seed(4)
    o.init_rand()
    ref, _ = o.anneal(3.0, 0, 0.85, 7, 12, 1)
    assert np.array_equal(mn, ref)
    assert np.array_equal(spins, o.spins())
