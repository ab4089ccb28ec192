"""GPU parity of the single-system path (the gpu_sys boundary) against the oracle.

Every spin word, coupling word and integer energy after N sweeps must be
bit-identical to the oracle's PHILOX mode (cpu_2d / cpu_2dp / cpu_3d logic and
sweep order, the reference GPU's per-site Philox draws).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

LATS = [(O.LAT_2D, 4), (O.LAT_2D, 8), (O.LAT_2D, 18), (O.LAT_2D, 64), (O.LAT_2D_OPEN_X, 2),
        (O.LAT_2D_OPEN_X, 8), (O.LAT_2D_OPEN_X, 14), (O.LAT_3D, 2), (O.LAT_3D, 4), (O.LAT_3D, 6),
        (O.LAT_3D, 10), (O.LAT_3D, 16)]


def _pair(sab, lat, L, T=1.0, h=0.0):
    from simulated_annealing_b200.system import GpuSystem
    return GpuSystem(lat, L, T, h), O.OracleSystem(lat, L, T, h, O.MODE_PHILOX)


def _setup(systems, j_seed, s_seed):
    # the reference driver's order: set_seed, init_J, set_seed, init_rand (src/main_gpu.cu:262-276)
    for x in systems:
        x.set_seed(j_seed)
        x.init_J()
        x.set_seed(s_seed)
        x.init_rand()


def _check(g, o):
    assert np.array_equal(g.get_spins(), o.spins())
    E, M = g.measure_exact()
    Eo, Mo = o.measure()
    assert np.array_equal(E, Eo) and np.array_equal(M, Mo)
    assert g.measure() == o.measure_float().tolist()


@pytest.mark.parametrize("lat,L", LATS)
@pytest.mark.parametrize("T,h", [(1.0, 0.0), (0.45, 0.25), (3.0, -1.0)])
def test_sweeps_bit_exact(sab, lat, L, T, h):
    g, o = _pair(sab, lat, L, T, h)
    _setup((g, o), 1, 2)
    J = g.get_J()
    for a, b in zip(J, o.J()):
        assert np.array_equal(a, b)
    _check(g, o)
    for n in (1, 2, 5):
        g.sweep(n)
        o.sweep(n)
        _check(g, o)
    assert g.rng_state()[1] == o.draw


@pytest.mark.parametrize("lat,L", [(lat, L) for lat, L in LATS if L >= 4])
def test_long_sweeps_resident_path(sab, lat, L):
    """Zero-field runs of >= 16 sweeps go through the shared-memory-resident
    kernel (one launch); short runs keep two launches per sweep. Alternating
    them must follow the oracle draw for draw."""
    g, o = _pair(sab, lat, L, 0.9)
    _setup((g, o), 7, 8)
    for n in (40, 3, 17, 1, 64):
        g.sweep(n)
        o.sweep(n)
        _check(g, o)
    assert g.rng_state()[1] == o.draw
    g.set_T(2.3)
    o.set_T(2.3)
    g.sweep(25)
    o.sweep(25)
    _check(g, o)


@pytest.mark.parametrize("L", [40, 48])
def test_long_sweeps_wide_path(sab, L):
    """Zero-field runs of >= 16 sweeps of a 3D lattice of L >= 40 go through
    the wide form (the lattice over the whole GPU, three launches per sweep)."""
    g, o = _pair(sab, O.LAT_3D, L, 0.7)
    _setup((g, o), 11, 12)
    for n in (20, 2, 17):
        g.sweep(n)
        o.sweep(n)
        _check(g, o)
    assert g.rng_state()[1] == o.draw


def test_init_J_without_reset_consumes_draws(sab):
    # timing-mode flow (src/main_gpu.cu:165-166): init_J then sweeps continue at draw t
    g, o = _pair(sab, O.LAT_3D, 6, 0.8)
    for x in (g, o):
        x.set_seed(77)
        x.init_J()
        x.init_rand()
    assert g.rng_state()[1] == o.draw == 6
    g.sweep(3)
    o.sweep(3)
    _check(g, o)


def test_set_T_between_sweeps(sab):
    g, o = _pair(sab, O.LAT_2D, 16, 3.0)
    _setup((g, o), 3, 4)
    for T in np.linspace(3.0, 0.2, 12):
        g.set_T(T)
        o.set_T(T)
        g.sweep(2)
        o.sweep(2)
    _check(g, o)


def test_set_J_set_spins_roundtrip_and_external_data(sab):
    g, o = _pair(sab, O.LAT_3D, 4, 0.9)
    _setup((o,), 5, 6)
    g.set_J(*o.J())
    g.set_spins(o.spins())
    g.set_rng_state(6, o.draw, 1)  # last set_seed of _setup was 6
    _check(g, o)
    g.sweep(4)
    o.sweep(4)
    _check(g, o)


def test_inconsistent_J_is_rejected(sab):
    from simulated_annealing_b200._lib import SAError
    g, o = _pair(sab, O.LAT_2D, 8)
    _setup((o,), 1, 1)
    jx, jy = o.J()
    jx = jx.copy()
    jx[3] ^= np.uint64(1)
    with pytest.raises(SAError):
        g.set_J(jx, jy)


def test_swap_and_init_order(sab):
    from simulated_annealing_b200.system import GpuSystem
    a, b = GpuSystem(O.LAT_2D, 8), GpuSystem(O.LAT_2D, 8)
    oa, ob = O.OracleSystem(O.LAT_2D, 8), O.OracleSystem(O.LAT_2D, 8)
    for x, s in ((a, 1), (b, 2), (oa, 1), (ob, 2)):
        x.set_seed(s)
        x.init_rand()
    a.swap(b, 0xF0F0_0000_FFFF_0001)
    oa.swap(ob, 0xF0F0_0000_FFFF_0001)
    assert np.array_equal(a.get_spins(), oa.spins()) and np.array_equal(b.get_spins(), ob.spins())
    a.init_order()
    assert np.all(a.get_spins() == np.uint64(0xFFFFFFFFFFFFFFFF))
    E, M = a.measure_exact()
    assert np.all(M == 64)


def test_checkpoint_roundtrip(sab):
    from simulated_annealing_b200.system import GpuSystem
    g, o = _pair(sab, O.LAT_2D_OPEN_X, 10, 0.6, 0.1)
    _setup((g, o), 9, 10)
    g.sweep(3)
    blob = g.save()
    g.sweep(5)
    after = g.get_spins()
    g2 = GpuSystem(O.LAT_2D_OPEN_X, 10, 2.0)
    g2.load(blob)
    g2.sweep(5)
    assert np.array_equal(g2.get_spins(), after)


def test_j_file_roundtrip(sab, tmp_path):
    g, o = _pair(sab, O.LAT_3D, 4)
    _setup((g,), 3, 3)
    f = str(tmp_path / "J.bin")
    g.save_J(f)
    from simulated_annealing_b200.system import GpuSystem
    h = GpuSystem(O.LAT_3D, 4)
    h.load_J(f)
    for a, b in zip(g.get_J(), h.get_J()):
        assert np.array_equal(a, b)


def test_c1_prefix_bit_exact(sab):
    # 2D periodic L=64, J seed 1, spins seed 2, T=1.0: first 1,000 sweeps
    g, o = _pair(sab, O.LAT_2D, 64, 1.0)
    _setup((g, o), 1, 2)
    g.sweep(1000)
    o.sweep(1000)
    _check(g, o)


def oracle_anneal(o, Ts, sweeps, stride):
    """annealing<> over an explicit schedule, restated with the oracle system:
    step k at Ts[k]; measure when i % stride == 0; running max of the float -H."""
    mn = None
    last = np.zeros((len(Ts), 64), dtype=np.float32)
    res = np.zeros(64, dtype=np.float32)
    for k, T in enumerate(Ts):
        o.set_T(T)
        for i in range(sweeps):
            o.sweep(1)
            if stride != 0 and i % stride == 0:
                res = o.measure_float()
                mn = res.copy() if mn is None else np.maximum(mn, res)
        last[k] = res
    return mn, last


@pytest.mark.parametrize("lat,L,h", [(O.LAT_3D, 8, 0.0), (O.LAT_2D, 16, 0.3), (O.LAT_2D_OPEN_X, 12, 0.0)])
def test_device_anneal_matches_annealing_template(sab, lat, L, h):
    """sa_sys_anneal vs annealing<> restated by the oracle (linear schedule)."""
    nsteps, sweeps = 9, 6
    T0, T1 = 3.0, 0.2
    Ts = [T0 + (T1 - T0) * k / (nsteps - 1) for k in range(nsteps)]
    g, o = _pair(sab, lat, L, T0, h)
    _setup((g, o), 1, 2)
    mn, stepE = g.anneal(Ts, sweeps, 1)
    ref, last = oracle_anneal(o, Ts, sweeps, 1)
    assert np.array_equal(mn, ref)
    assert np.array_equal(g.get_spins(), o.spins())
    if h == 0.0:
        assert np.array_equal(stepE.astype(np.float32), last)
    # and the oracle's own C restatement of the template agrees for the same schedule
    o2 = O.OracleSystem(lat, L, T0, h, O.MODE_PHILOX)
    _setup((o2,), 1, 2)
    ref2, _ = o2.anneal(T0, 1, T1, nsteps, sweeps, 1)
    assert np.array_equal(ref, ref2)


def test_device_anneal_stride_and_geometric(sab):
    g, o = _pair(sab, O.LAT_3D, 6, 2.5, 0.0)
    _setup((g, o), 4, 5)
    Ts = [2.5 * 0.8 ** k for k in range(5)]
    mn, _ = g.anneal(Ts, 7, 3)
    ref, _ = oracle_anneal(o, Ts, 7, 3)
    assert np.array_equal(mn, ref)
    assert np.array_equal(g.get_spins(), o.spins())


def test_c2_prefix(sab):
    """C2 shape: 3D L=32, J seed 3, linear T 3.0 -> 0.2 over 200 steps of 100
    sweeps; the first 3 steps against the oracle, per-step integer energies too."""
    Ts = [3.0 + (0.2 - 3.0) * k / 199 for k in range(200)][:3]
    g, o = _pair(sab, O.LAT_3D, 32, 3.0)
    _setup((g, o), 3, 3)
    mn, stepE = g.anneal(Ts, 100, 1)
    ref_mn, ref_last = oracle_anneal(o, Ts, 100, 1)
    assert np.array_equal(mn, ref_mn)
    assert np.array_equal(stepE.astype(np.float32), ref_last)
    assert np.array_equal(g.get_spins(), o.spins())
