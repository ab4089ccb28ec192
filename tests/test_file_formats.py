"""File formats shared with the reference, byte for byte.

J files (src/sys_file.cpp:10-110: int dim; long N; Jx[2N]; Jy[2N]; (Jz[2N]))
written by one side must load on the other: the reference's own
cpu_2dp / cpu_3d save_J / load_J (oracle/_ref) against the engine's writer
and reader (simulated_annealing_b200.system.read_J_file / write_J_file on the
CPU; GpuSystem.save_J / load_J on the GPU).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")

CASES = [(O.LAT_2D, 8), (O.LAT_2D_OPEN_X, 10), (O.LAT_3D, 6)]


def _ref_J(r):
    s, jx, jy, jz = r.state()
    return (jx, jy, jz) if r.lattice == O.LAT_3D else (jx, jy)


@pytest.mark.parametrize("lat,L", CASES)
def test_reference_written_J_file_reads_back_identically(tmp_path, lat, L):
    from simulated_annealing_b200.system import read_J_file, write_J_file

    r = O.RefSystem(lat, L)
    r.set_seed(17)
    r.init_J()
    f = str(tmp_path / "ref.J")
    r.save_J(f)
    dim = 3 if lat == O.LAT_3D else 2
    arrs = read_J_file(f, dim, r.N)
    for a, b in zip(arrs, _ref_J(r)):
        assert np.array_equal(a, b)
    g = str(tmp_path / "ours.J")
    write_J_file(g, arrs)
    assert open(g, "rb").read() == open(f, "rb").read()


@pytest.mark.parametrize("lat,L", CASES)
def test_engine_written_J_file_loads_in_the_reference(tmp_path, lat, L):
    from simulated_annealing_b200.system import write_J_file

    o = O.OracleSystem(lat, L, mode=O.MODE_PHILOX)
    o.set_seed(5)
    o.init_J()
    f = str(tmp_path / "ours.J")
    write_J_file(f, o.J())
    r = O.RefSystem(lat, L)
    r.load_J(f)
    for a, b in zip(o.J(), _ref_J(r)):
        assert np.array_equal(a, b)


def test_J_file_errors_follow_the_reference(tmp_path):
    from simulated_annealing_b200.system import read_J_file, write_J_file

    o = O.OracleSystem(O.LAT_2D, 8)
    o.set_seed(1)
    o.init_J()
    f = str(tmp_path / "J")
    write_J_file(f, o.J())
    with pytest.raises(ValueError, match="2D"):
        read_J_file(f, 3, 64)  # the reference's load_J_3d returns -2
    with pytest.raises(ValueError, match="N="):
        read_J_file(f, 2, 100)  # -3
    with pytest.raises(ValueError, match="cannot open"):
        read_J_file(str(tmp_path / "missing"), 2, 64)  # -1
    open(f, "r+b").truncate(40)
    with pytest.raises(ValueError, match="truncated"):
        read_J_file(f, 2, 64)


@pytest.mark.gpu
@pytest.mark.parametrize("lat,L", CASES)
def test_gpu_system_J_files_against_reference(sab, tmp_path, lat, L):
    from simulated_annealing_b200.system import GpuSystem

    g = GpuSystem(lat, L)
    g.set_seed(9)
    g.init_J()
    f = str(tmp_path / "gpu.J")
    g.save_J(f)
    r = O.RefSystem(lat, L)
    r.load_J(f)
    for a, b in zip(g.get_J(), _ref_J(r)):
        assert np.array_equal(a, b)
    r2 = O.RefSystem(lat, L)
    r2.set_seed(33)
    r2.init_J()
    f2 = str(tmp_path / "ref.J")
    r2.save_J(f2)
    h = GpuSystem(lat, L)
    h.load_J(f2)
    for a, b in zip(h.get_J(), _ref_J(r2)):
        assert np.array_equal(a, b)
    h.save_J(str(tmp_path / "again.J"))
    assert open(str(tmp_path / "again.J"), "rb").read() == open(f2, "rb").read()
