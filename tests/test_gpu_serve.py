"""Serving engine: continuous batching of anneal requests.

Each request is annealing<gpu_sys> (src/annealing.hpp:67-100) on its own
disorder instance; the server must give every request exactly the result it
gets alone -- and that the oracle gets -- whatever else is admitted beside it,
whenever it arrives and however the rounds are chunked.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def linear(T0, T1, n):
    return [T0 + (T1 - T0) * k / (n - 1) for k in range(n)] if n > 1 else [T0]


def oracle_result(lat, L, sJ, s, T0, T1, nsteps, per):
    o = O.OracleSystem(lat, L, mode=O.MODE_PHILOX)
    o.set_seed(sJ)
    o.init_J()
    o.set_seed(s)
    o.init_rand()
    mn, _ = o.anneal(T0, 1, T1, nsteps, per, 1)
    return mn, o.spins()


def drain(srv, chunk, out):
    while srv.active()[0]:
        srv.step(chunk)
        done = srv.poll()
        if done:
            srv.sync()
            for rid in done:
                out[rid] = srv.result(rid, spins=True)


def test_serve_matches_oracle(sab):
    from simulated_annealing_b200.serve import Server
    srv = Server(budget_bytes=64 << 20, max_requests=16)
    specs = [(O.LAT_2D, 8, 31, 32, 5, 4), (O.LAT_3D, 6, 33, 34, 3, 7), (O.LAT_2D_OPEN_X, 10, 35, 36, 6, 3),
             (O.LAT_3D, 4, 37, 38, 2, 2)]
    ids = {}
    for lat, L, sJ, s, n, per in specs:
        ids[srv.submit(lat, L, sJ, s, linear(3.0, 0.2, n), per)] = (lat, L, sJ, s, n, per)
    out = {}
    drain(srv, 5, out)  # chunks that end inside steps
    assert set(out) == set(ids)
    for rid, (lat, L, sJ, s, n, per) in ids.items():
        mn, spins = oracle_result(lat, L, sJ, s, 3.0, 0.2, n, per)
        assert np.array_equal(out[rid].emax.astype(np.float32), mn)
        assert np.array_equal(out[rid].spins, spins)


def test_serve_result_same_alone_and_in_mix(sab):
    from simulated_annealing_b200.serve import Server
    rng = np.random.default_rng(5)
    shapes = [(O.LAT_3D, 24), (O.LAT_3D, 16), (O.LAT_3D, 10), (O.LAT_2D, 64), (O.LAT_2D, 32),
              (O.LAT_2D_OPEN_X, 48), (O.LAT_3D, 32), (O.LAT_2D, 128), (O.LAT_3D, 8), (O.LAT_2D, 16)]
    reqs = []
    for k, (lat, L) in enumerate(shapes):
        n = int(rng.integers(2, 6))
        per = int(rng.integers(3, 20))
        reqs.append((lat, L, 100 + k, 200 + k, linear(2.5, 0.3, n), per))
    # mixed: half submitted up front, the rest after some rounds
    srv = Server(budget_bytes=256 << 20, max_requests=64)
    ids = [None] * len(reqs)
    for k in range(0, len(reqs), 2):
        ids[k] = srv.submit(*reqs[k])
    mixed = {}
    for _ in range(2):
        srv.step(7)
        for rid in srv.poll():
            srv.sync()
            mixed[rid] = srv.result(rid, spins=True)
    for k in range(1, len(reqs), 2):
        ids[k] = srv.submit(*reqs[k])
    drain(srv, 11, mixed)
    assert all(i in mixed for i in ids)
    for k, r in enumerate(reqs):
        alone = Server(budget_bytes=64 << 20, max_requests=1)
        rid = alone.submit(*r)
        one = {}
        drain(alone, 1000, one)
        alone.close()
        a, m = one[rid], mixed[ids[k]]
        assert np.array_equal(a.emax, m.emax), k
        assert np.array_equal(a.elast, m.elast), k
        assert np.array_equal(a.spins, m.spins), k


def test_serve_budget_admission_and_reuse(sab):
    from simulated_annealing_b200.serve import Server
    srv = Server(budget_bytes=4 << 20, max_requests=8)
    T = linear(2.0, 0.5, 2)
    # 3D L=32: 4 * 32768 words = 1 MiB each; the word pool holds three
    got = []
    while True:
        rid = srv.submit("3d", 32, 1, 2, T, 2)
        if rid is None:
            break
        got.append(rid)
    assert 1 <= len(got) <= 3
    n0, free0 = srv.active()
    assert n0 == len(got)
    out = {}
    drain(srv, 100, out)
    assert set(out) == set(got)
    n1, free1 = srv.active()
    assert n1 == 0 and free1 > free0
    # the freed space is reusable and results repeat
    rid = srv.submit("3d", 32, 1, 2, T, 2)
    assert rid is not None
    again = {}
    drain(srv, 100, again)
    assert np.array_equal(again[rid].emax, out[got[0]].emax)
    assert np.array_equal(again[rid].spins, out[got[0]].spins)


def test_serve_rejects_bad_requests(sab):
    from simulated_annealing_b200._lib import SAError
    from simulated_annealing_b200.serve import Server
    srv = Server(budget_bytes=4 << 20, max_requests=2)
    with pytest.raises(SAError):
        srv.submit("2d", 7, 1, 2, [1.0], 1)
    with pytest.raises(SAError):
        srv.submit("2d", 8, 1, 2, [1.0, -1.0], 1)
    with pytest.raises(SAError):
        srv.submit("2d", 8, 1, 2, [1.0], 0)
    assert srv.submit("3d", 64, 1, 2, [1.0], 1) is None  # 4 MiB of words > the pool


def test_serve_many_wide_requests(sab):
    """Large 3D requests served one at a time each run wide (alone on the
    GPU) with their own captured graphs; more of them than the graph cache
    holds still give annealing<>'s results."""
    from simulated_annealing_b200.serve import Server
    srv = Server(budget_bytes=64 << 20, max_requests=4)
    T = linear(2.5, 0.5, 3)
    out = {}
    ids = []
    for k in range(36):
        rid = srv.submit(O.LAT_3D, 40, 900 + k, 950 + k, T, 20)
        assert rid is not None
        ids.append(rid)
        drain(srv, 100, out)
    for k in (0, 17, 35):
        mn, spins = oracle_result(O.LAT_3D, 40, 900 + k, 950 + k, 2.5, 0.5, 3, 20)
        assert np.array_equal(out[ids[k]].emax.astype(np.float32), mn), k
        assert np.array_equal(out[ids[k]].spins, spins), k
