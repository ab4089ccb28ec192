"""The reference's SPLIT_H update (its alternative build, off by default).

The reference's GPU kernels define it (src/device_2d.cu:27-50 with the
open-x handling of :114-125, src/device_3d.cu:216-245 with the boundary
branch :76-89) and its tables (src/gpu_2d.cu:133-139, src/gpu_3d.cu:57-63);
neither that GPU code nor the CPU version (src/cpu_2dp.cpp:161-163) compiles,
so the pin is a literal transcription of those formulas here -- the p0/p1/p2
"exactly k satisfied" terms, the float tables, two uniforms per site per
half-sweep -- checked against the oracle's restatement on the CPU; the GPU
test checks the engine against the oracle.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

MASK = (1 << 64) - 1


def _f32(x):
    return np.float32(x)


def reference_split_sweeps(o, lat, L, T, h, seed, draw0, nsweeps):
    """SPLIT_H sweeps of the oracle system's current state, computed from the
    reference's formulas in Python; returns the spin words."""
    s = [int(v) for v in o.spins()]
    J = [[int(v) for v in a] for a in o.J()]
    N = len(s)
    if lat == O.LAT_3D:
        boltz = [_f32(math.exp(-2. * (2 + 2 * i) * (1. / T))) for i in range(3)] + [_f32(math.exp(-2 * h / T))]
    else:
        boltz = [_f32(math.exp(-2. * (1 + i) * (1. / T))) for i in range(4)] + [_f32(math.exp(-2. * h / T))]
    draw = draw0
    for _ in range(nsweeps):
        for colour in (0, 1):
            for i in range(N):
                x, y, z = i % L, (i // L) % L, i // (L * L)
                if (x + y) % 2 != colour:
                    continue
                r1 = _f32(O.uniform_from_u32(O.philox_draw(seed, i, draw + 2 * colour)))
                r2 = _f32(O.uniform_from_u32(O.philox_draw(seed, i, draw + 2 * colour + 1)))
                si = s[i]
                full = lambda b: MASK if b else 0  # noqa: E731
                if lat == O.LAT_3D:
                    L2 = L * L
                    w = i - 1 if x else i + L - 1
                    e = i + 1 if x < L - 1 else i - L + 1
                    n_ = i - L if y else i + L2 - L
                    so = i + L if y < L - 1 else i - L2 + L
                    u = i - L2 if z else i + N - L2
                    d = i + L2 if z < L - 1 else i - N + L2
                    sw = J[0][2 * i] ^ si ^ s[w]
                    se = J[0][2 * i + 1] ^ si ^ s[e]
                    sn = J[1][2 * i] ^ si ^ s[n_]
                    ss = J[1][2 * i + 1] ^ si ^ s[so]
                    su = J[2][2 * i] ^ si ^ s[u]
                    sd = J[2][2 * i + 1] ^ si ^ s[d]
                    if x == 0 or y == 0 or z == 0 or x == L - 1 or y == L - 1 or z == L - 1:
                        r1 = r2  # the boundary branch passes rand2 twice
                    p0 = sw & se & sn & ss & su & sd
                    p1 = ((sw ^ se) & sn & ss & su & sd) | (sw & se & (sn ^ ss) & su & sd) | \
                         (sw & se & sn & ss & (su ^ sd))
                    p2 = ((sw ^ se) & (sn ^ ss) & su & sd) | ((sw ^ se) & sn & ss & (su ^ sd)) | \
                         (sw & se & (sn ^ ss) & (su ^ sd)) | ((sw ^ sd) & (se ^ su) & sn & ss) | \
                         (sw & (se ^ sn) & (ss ^ su) & sd)
                    d0, d1, d2 = full(r1 < boltz[2]), full(r1 < boltz[1]), full(r1 < boltz[0])
                    dh = full(r2 < boltz[3])
                    mh = (~si & MASK) | dh
                    s[i] = si ^ (((p0 & d0) | (p1 & d1) | (p2 & d2) | (~(p0 | p1 | p2) & MASK)) & mh)
                else:
                    open_x = lat == O.LAT_2D_OPEN_X
                    w = i - 1 if x else i + L - 1
                    e = i + 1 if x < L - 1 else i - L + 1
                    n_ = i - L if y else i + N - L
                    so = i + L if y < L - 1 else i - N + L
                    sw = MASK if (open_x and x == 0) else J[0][2 * i] ^ si ^ s[w]
                    se = MASK if (open_x and x == L - 1) else J[0][2 * i + 1] ^ si ^ s[e]
                    sn = J[1][2 * i] ^ si ^ s[n_]
                    ss = J[1][2 * i + 1] ^ si ^ s[so]
                    border = MASK if (open_x and (x == 0 or x == L - 1)) else 0
                    p0 = sw & sn & se & ss
                    p1 = ((sw ^ sn) & se & ss) | (sw & sn & (se ^ ss))
                    d01, d11 = full(r1 < boltz[2]), full(r1 < boltz[0])
                    d00, d10 = full(r1 < boltz[3]), full(r1 < boltz[1])
                    dh = full(r2 < boltz[4])
                    d0 = (d00 | border) & (d01 | (~border & MASK))
                    d1 = (d10 | border) & (d11 | (~border & MASK))
                    mh = (~si & MASK) | dh
                    s[i] = si ^ (((p0 & d0) | (p1 & d1) | (~(p0 | p1) & MASK)) & mh)
        draw += 4
    return np.array(s, dtype=np.uint64)


CASES = [(O.LAT_2D_OPEN_X, 6), (O.LAT_2D, 6), (O.LAT_3D, 4)]
FIELDS = [(1.0, 0.0), (0.7, 0.4), (1.5, -0.6)]


@pytest.mark.parametrize("lat,L", CASES)
@pytest.mark.parametrize("T,h", FIELDS)
def test_oracle_split_is_the_reference_formulas(lat, L, T, h):
    o = O.OracleSystem(lat, L, T, h, O.MODE_PHILOX)
    o.set_seed(7)
    o.init_J()
    o.set_seed(8)
    o.init_rand()
    o.set_split(True)
    draw0 = o.draw
    want = reference_split_sweeps(o, lat, L, T, h, 8, draw0, 3)
    o.sweep(3)
    assert np.array_equal(o.spins(), want)
    assert o.draw == draw0 + 12


@pytest.mark.gpu
@pytest.mark.parametrize("lat,L", [(O.LAT_2D_OPEN_X, 16), (O.LAT_2D, 18), (O.LAT_3D, 8), (O.LAT_3D, 12)])
@pytest.mark.parametrize("T,h", FIELDS)
def test_engine_split_matches_oracle(sab, lat, L, T, h):
    from simulated_annealing_b200.system import GpuSystem

    g = GpuSystem(lat, L, T, h)
    o = O.OracleSystem(lat, L, T, h, O.MODE_PHILOX)
    for x in (g, o):
        x.set_seed(3)
        x.init_J()
        x.set_seed(4)
        x.init_rand()
    g.set_split_field(True)
    o.set_split(True)
    for n in (1, 4, 20):
        g.sweep(n)
        o.sweep(n)
        assert np.array_equal(g.get_spins(), o.spins())
        assert np.array_equal(g.measure_exact()[0], o.measure()[0])
    assert g.rng_state()[1] == o.draw
    g.set_T(0.5)
    o.set_T(0.5)
    g.sweep(5)
    o.sweep(5)
    assert np.array_equal(g.get_spins(), o.spins())
    # the mode travels with the checkpoint record
    k = GpuSystem(lat, L)
    k.load(g.save())
    assert k.split_field()
    k.sweep(3)
    o.sweep(3)
    assert np.array_equal(k.get_spins(), o.spins())


@pytest.mark.gpu
def test_split_rules(sab):
    from simulated_annealing_b200._lib import SAError
    from simulated_annealing_b200.system import GpuSystem

    g = GpuSystem("3d", 4)
    g.set_rng_mode("mt19937_64")
    with pytest.raises(SAError):
        g.set_split_field(True)
    h = GpuSystem("3d", 4)
    h.set_split_field(True)
    with pytest.raises(SAError):
        h.set_rng_mode("mt19937_64")
