"""The command-line front end (simulated_annealing_b200/sa_anneal): the
reference's annealing_gpu flags (src/main_gpu.cu:56-131) and modes.

Argument errors are checked on the CPU (they exit before any CUDA call); the
modes run on the GPU and are checked against the oracle: the anneal output
(-H after every sweep, or the running maximum per restart with -r), the
parallel-tempering energy files and swap statistics, the repeat-until-ground-
state loop with its .tempsys checkpoints, J files and temperature blocks.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "simulated_annealing_b200", "sa_anneal")

pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="sa_anneal not built")


def run(args, cwd, timeout=300):
    return subprocess.run([EXE, *args], capture_output=True, text=True, cwd=cwd, timeout=timeout)


def rows(text):
    """Numeric rows of a reference-style output (lines of tab-separated floats;
    '#' lines are the info header)."""
    out = []
    for ln in text.splitlines():
        if ln.startswith("#") or not ln.strip():
            continue
        out.append(np.array([float(v) for v in ln.split("\t") if v.strip()], dtype=np.float32))
    return out


@pytest.mark.parametrize("args,msg", [
    ([], "exactly one of"),
    (["-T", "1", "-P", "1"], "exactly one of"),
    (["-T", "1", "-d", "4"], "-d must be"),
    (["-T", "x"], "bad value"),
    (["-T", "1", "--bogus"], "unknown argument"),
    (["--Pb", "2 0.1 1"], "bad temperature block"),
    (["-T", "1", "-r", "0"], "-r must be"),
    (["-T", "1", "--rng", "xorwow"], "--rng must be"),
])
def test_argument_errors(tmp_path, args, msg):
    r = run(args, str(tmp_path))
    assert r.returncode == 1
    assert msg in r.stderr


def _oracle(lat, L, seed, T=1.0, mode=O.MODE_PHILOX):
    o = O.OracleSystem(lat, L, T, 0.0, mode)
    o.set_seed(seed)
    o.init_J()
    o.set_seed(seed)
    o.init_rand()
    return o


@pytest.mark.gpu
@pytest.mark.parametrize("dim,lat", [("3", O.LAT_3D), ("2p", O.LAT_2D_OPEN_X), ("2", O.LAT_2D)])
def test_anneal_prints_every_sweep(sab, tmp_path, dim, lat):
    r = run(["-d", dim, "-L", "6", "-T", "2.0", "-a", "0.8", "-s", "3", "-S", "4", "--seed", "7"], str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("# ") and "# Version : " in r.stdout
    got = rows(r.stdout)
    o = _oracle(lat, 6, 7)
    want, T = [], 2.0
    for _ in range(3):
        o.set_T(T)
        for _ in range(4):
            o.sweep(1)
            want.append(o.measure_float())
        T *= 0.8
    assert len(got) == 12
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


@pytest.mark.gpu
def test_anneal_repeat_prints_running_maximum(sab, tmp_path):
    r = run(["-d", "3", "-L", "6", "-T", "2.5", "-a", "0.7", "-s", "4", "-S", "3", "--seed", "11", "-r", "2"],
            str(tmp_path))
    assert r.returncode == 0, r.stderr
    got = rows(r.stdout)
    assert len(got) == 2
    o = _oracle(O.LAT_3D, 6, 11)
    last = 2.5 * 0.7 ** 4
    for run_i in range(2):
        sched = [2.5 * 0.7 ** k for k in range(4)]
        if run_i == 1:
            sched[0] = last  # annealing::set_T leaves the system at the last cooled T
            o.init_rand()
        mn = None
        for T in sched:
            o.set_T(T)
            for _ in range(3):
                o.sweep(1)
                e = o.measure_float()
                mn = e if mn is None else np.maximum(mn, e)
        assert np.array_equal(got[run_i], mn), run_i


@pytest.mark.gpu
def test_parallel_tempering_files_and_swap(sab, tmp_path):
    T = [0.5, 1.0, 1.6]
    args = ["-d", "3", "-L", "4", "-S", "1", "-s", "10", "--seed", "5", "--swap", "--outputT",
            str(tmp_path / "out_%.dat")]
    for t in T:
        args += ["-P", str(t)]
    r = run(args, str(tmp_path))
    assert r.returncode == 0, r.stderr
    systems = [_oracle(O.LAT_3D, 4, 5) for _ in T]
    pt = O.OraclePT(systems, T, 1)
    E = []
    for _ in range(10):
        pt.step(1)
        E.append(pt.energies())
    for i, t in enumerate(T):
        f = tmp_path / f"out_T{t:f}.dat"
        got = rows(f.read_text())
        assert len(got) == 10
        for k in range(10):
            assert np.array_equal(got[k], E[k][i]), (t, k)
    # swap statistics: "T_i -> T_i+1\t: acceptance" (src/parallel_tempering.hpp:164-169)
    lines = [ln for ln in r.stdout.splitlines() if "->" in ln]
    acc = pt.acceptance()
    assert len(lines) == 2
    for ln, a in zip(lines, acc):
        assert float(ln.split(":")[1]) == pytest.approx(a, rel=1e-5, abs=1e-9)


@pytest.mark.gpu
def test_temperature_blocks_and_file(sab, tmp_path):
    """--Pb "0.5 0.5 1.5" and a --P_file with the same block give 0.5, 1, 1.5."""
    (tmp_path / "blocks").write_text("0.5 0.5 1.5\n")
    outs = []
    for extra in (["--Pb", "0.5 0.5 1.5"], ["--P_file", str(tmp_path / "blocks")]):
        r = run(["-d", "2p", "-L", "6", "-S", "1", "-s", "4", "--swap", "--outputT", str(tmp_path / "b_%.dat"),
                 *extra], str(tmp_path))
        assert r.returncode == 0, r.stderr
        outs.append([ln for ln in r.stdout.splitlines() if "->" in ln])
    assert outs[0] == outs[1]
    assert [ln.split("\t")[0] for ln in outs[0]] == ["0.5 -> 1", "1 -> 1.5"]


@pytest.mark.gpu
def test_repeat_until_ground_state_checkpoints(sab, tmp_path):
    tmp = str(tmp_path) + "/"
    r = run(["-d", "3", "-L", "4", "-P", "0.4", "-P", "0.8", "-P", "1.5", "-S", "2", "-s", "5", "-r", "3",
             "--maxiter", "2", "--tmp", tmp, "--outputT", str(tmp_path / "pt_%.dat")], str(tmp_path))
    assert r.returncode == 0, r.stderr
    ckpts = sorted(f for f in os.listdir(tmp_path) if f.endswith(".tempsys"))
    assert len(ckpts) == 3
    emin = rows((tmp_path / "pt_E_min.dat").read_text())
    assert len(emin) >= 3 and all(len(e) == 64 for e in emin)
    # the checkpoints are the template's stream over this engine's records
    from simulated_annealing_b200.drivers import ParallelTempering
    from simulated_annealing_b200.system import GpuSystem
    ep = ParallelTempering([GpuSystem("3d", 4) for _ in range(3)], [0.4, 0.8, 1.5], 2, "x_%")
    ep.load((tmp_path / ckpts[0]).read_bytes())
    assert ep.T == [0.4, 0.8, 1.5] and ep.steps == 2


@pytest.mark.gpu
def test_J_files_and_timing(sab, tmp_path):
    J = str(tmp_path / "J.bin")
    a = run(["-d", "3", "-L", "4", "-T", "1.5", "-s", "2", "-S", "2", "--seed", "3", "-J", J], str(tmp_path))
    b = run(["-d", "3", "-L", "4", "-T", "1.5", "-s", "2", "-S", "2", "--seed", "3", "-j", J], str(tmp_path))
    assert a.returncode == 0 and b.returncode == 0
    assert rows(a.stdout) and all(np.array_equal(x, y) for x, y in zip(rows(a.stdout), rows(b.stdout)))
    r = O.RefSystem(O.LAT_3D, 4) if O.ref_available() else None
    if r is not None:
        r.load_J(J)  # the reference's own reader takes the file
    t = run(["-t", "-d", "3", "-L", "16", "-s", "20", "-T", "1"], str(tmp_path))
    assert t.returncode == 0, t.stderr
    sec, rate = (float(v) for v in t.stdout.split())
    assert sec > 0 and rate > 0


@pytest.mark.gpu
def test_mt19937_mode_matches_the_reference_classes(sab, tmp_path):
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    res = run(["-d", "3", "-L", "4", "-T", "1.2", "-a", "0.9", "-s", "2", "-S", "3", "--seed", "9", "--rng",
               "mt19937_64"], str(tmp_path))
    assert res.returncode == 0, res.stderr
    r = O.RefSystem(O.LAT_3D, 4, 1.2)
    r.set_seed(9)
    r.init_J()
    r.set_seed(9)
    r.init_rand()
    want, T = [], 1.2
    for _ in range(2):
        r.set_T(T)
        for _ in range(3):
            r.sweep(1)
            want.append(r.measure_float())
        T *= 0.9
    got = rows(res.stdout)
    assert len(got) == 6 and all(np.array_equal(g, w) for g, w in zip(got, want))
