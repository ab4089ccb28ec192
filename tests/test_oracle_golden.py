"""The oracle's Philox4x32-10 and u32->uniform map against cuRAND's own outputs.

tests/golden/curand_philox_golden.json was produced on a B200 by
tests/golden/gen_curand_golden.cu, which only calls curand_init / curand /
curand_uniform (the reference's src/random.cu:15-35, src/device_2d.cu:96-97).
"""
import json
import os
import struct

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "curand_philox_golden.json")


def _bits(f: float) -> int:
    return struct.unpack("<I", struct.pack("<f", f))[0]


def test_philox_draws_match_curand(oracle):
    g = json.load(open(GOLDEN))
    assert len(g["cases"]) >= 100
    n = 0
    for c in g["cases"]:
        seed, sub, off = int(c["seed"]), int(c["subsequence"]), int(c["offset"])
        for k, u in enumerate(c["u32"]):
            assert oracle.philox_draw(seed, sub, off + k) == u, (seed, sub, off, k)
            n += 1
    assert n == len(g["cases"]) * g["draws_per_case"]


def test_uniform_matches_curand_uniform(oracle):
    g = json.load(open(GOLDEN))
    for c in g["cases"]:
        for u, fb in zip(c["u32"], c["uniform_bits"]):
            assert _bits(oracle.uniform_from_u32(u)) == fb


def test_uniform_edges(oracle):
    assert oracle.uniform_from_u32(0xFFFFFFFF) == 1.0
    assert 0.0 < oracle.uniform_from_u32(0) < 1e-9
    # strictly inside (0,1] and non-decreasing on a dense sample
    us = np.unique(np.concatenate([np.arange(0, 1 << 20, 7), np.arange((1 << 32) - (1 << 20), 1 << 32, 5),
                                   np.random.default_rng(1).integers(0, 1 << 32, 200000)]))
    fs = np.array([oracle.uniform_from_u32(int(u)) for u in us[::97]])
    assert np.all(np.diff(fs) >= 0)


def test_threshold_definition(oracle):
    rng = np.random.default_rng(2)
    for b in [1.0, 0.5, np.exp(-4.0), np.exp(-8.0 / 0.3), 2.0 ** -33, 1e-12, 0.9999999]:
        b = float(np.float32(b))
        t = oracle.threshold(b)
        assert 0 <= t < (1 << 32)
        if t > 0:
            assert oracle.uniform_from_u32(t - 1) < b
        assert not (oracle.uniform_from_u32(t) < b)
        for u in rng.integers(0, 1 << 32, 200):
            assert (oracle.uniform_from_u32(int(u)) < b) == (int(u) < t)


BULK = os.path.join(os.path.dirname(__file__), "golden", "curand_philox_bulk.json")


@pytest.mark.skipif(not os.path.exists(BULK), reason="bulk cuRAND digests not generated")
def test_philox_bulk_matches_curand(oracle):
    """Subsequences 0..4095 x draws 0..63 for nine seeds (2.36 M draws and
    their uniforms), as SHA-256 digests of cuRAND's outputs on a B200."""
    import ctypes
    import hashlib

    g = json.load(open(BULK))
    subs, draws = g["subsequences"], g["draws"]
    lib = oracle.oracle_lib()
    lib.sao_philox_bulk.argtypes = [ctypes.c_uint64, ctypes.c_long, ctypes.c_long,
                                    ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]
    assert len(g["seeds"]) == 9
    for seed, h in g["seeds"].items():
        u = np.zeros(subs * draws, dtype="<u4")
        f = np.zeros(subs * draws, dtype="<u4")
        lib.sao_philox_bulk(int(seed), subs, draws, u.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                            f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        assert hashlib.sha256(u.tobytes()).hexdigest() == h["u32_sha256"], seed
        assert hashlib.sha256(f.tobytes()).hexdigest() == h["uniform_bits_sha256"], seed


def test_uniform_is_monotone_over_every_u32(oracle):
    """Exhaustive over all 2^32 inputs: the u32 -> uniform map (pinned to
    curand_uniform above) is non-decreasing, lies in (0, 1] and reaches 1.
    With it, "uniform(u) < b" is "u < thr(b)" for every u, which is what the
    engine's integer thresholds compute."""
    assert oracle.oracle_lib().sao_check_uniform_monotone() == 0
