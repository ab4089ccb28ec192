"""The tuned launch shapes of the batched engine.

simulated_annealing_b200/autotune.py times candidate shapes per bucket on the
GPU and writes the winners into the table compiled into the library
(csrc/sa_tuning.inc, record in tuning.json). Every tuned shape must keep the
engine bit-exact: one instance of each bucket runs in exactly that shape
(checked through sa_batch_instance_shape) against the oracle's
parallel_tempering<>.
"""
import json
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
ROOT = os.path.dirname(HERE)
JSON = os.path.join(ROOT, "simulated_annealing_b200", "tuning.json")
INC = os.path.join(ROOT, "simulated_annealing_b200", "csrc", "sa_tuning.inc")


def _inc_rows():
    rows = []
    for ln in open(INC):
        ln = ln.strip()
        if ln.startswith("{"):
            rows.append([int(v) for v in ln.strip("{},").split(",")])
    return rows


def test_table_and_record_agree():
    rows = _inc_rows()
    for r in rows:
        assert len(r) == 7 and r[0] in (0, 1, 2) and r[1] % 2 == 0 and r[3] >= 1 and r[4] in (1, 2)
        assert r[5] >= 2  # threads 0..63 hold one replica each
    if os.path.exists(JSON):
        rec = json.load(open(JSON))
        assert [list(map(int, e)) for e in rec["table"]] == rows
        for b in rec["buckets"]:
            if b["best"] is not None:
                assert b["best_rate"] > b["heuristic_rate"]


@pytest.mark.gpu
def test_every_tuned_shape_is_bit_exact(sab):
    from simulated_annealing_b200.batch import Batch, tuning_table
    from test_gpu_batch import check_instance

    table = tuning_table()
    assert table.tolist() == _inc_rows()
    for row in table:
        lat, L, nslots = (int(v) for v in row[:3])
        if nslots == 1:
            _check_single_slot(row)
            continue
        T = list(np.geomspace(0.5, 2.0, nslots) if lat == O.LAT_3D else np.geomspace(0.3, 1.6, nslots))
        b = Batch()
        lad = b.add_ladder(T)
        b.add_instance(lat, L, ladder=lad, seed_J=70 + L, seed=71 + L)
        b.set_spread(False)
        b.finalize()
        assert b.shape(0) == tuple(int(v) for v in row), row
        b.record_exchanges(16)
        b.run(5)
        b.run(4)
        b.sync()
        check_instance(b, 0, lat, L, T, 70 + L, 71 + L, 9)
        b.close()


def _check_single_slot(row):
    """A single-slot anneal (a serving request's shape) in its tuned shape,
    two instances, against the oracle's annealing<> restatement."""
    from simulated_annealing_b200.batch import Batch

    lat, L = int(row[0]), int(row[1])
    Ts = [2.5, 1.6, 0.7]  # linear, as the oracle's anneal(2.5, 1, 0.7, 3, ...) steps
    b = Batch()
    sch = b.add_schedule(Ts, 2)
    for k in range(2):
        b.add_instance(lat, L, schedule=sch, seed_J=80 + k, seed=90 + k)
    b.set_spread(False)
    b.finalize()
    assert b.shape(0) == tuple(int(v) for v in row), row
    b.run(6)
    b.sync()
    for k in range(2):
        o = O.OracleSystem(lat, L, mode=O.MODE_PHILOX)
        o.set_seed(80 + k)
        o.init_J()
        o.set_seed(90 + k)
        o.init_rand()
        mn, _ = o.anneal(2.5, 1, 0.7, 3, 2, 1)
        E, done = b.anneal_result(k)
        assert done == 6
        assert np.array_equal(E.astype(np.float32), mn), (row, k)
        assert np.array_equal(b.spins(k, 0), o.spins()), (row, k)
    b.close()


@pytest.mark.gpu
def test_explicit_shapes_and_fallback(sab):
    """A shape given through sa_batch_set_tuning is used (two-slot high-register
    3D walk on a larger cluster); an unusable one (odd slots with SL = 2)
    falls back to the heuristic shape; both stay bit-exact."""
    from simulated_annealing_b200.batch import Batch
    from test_gpu_batch import check_instance

    T = list(np.geomspace(0.5, 2.0, 6))
    b = Batch()
    lad = b.add_ladder(T)
    b.add_instance(O.LAT_3D, 10, ladder=lad, seed_J=5, seed=6)
    b.set_tuning([[O.LAT_3D, 10, 6, 2, 2, 5, 1]])
    b.set_spread(False)
    b.finalize()
    assert b.shape(0) == (O.LAT_3D, 10, 6, 2, 2, 5, 1)
    b.record_exchanges(8)
    b.run(7)
    b.sync()
    check_instance(b, 0, O.LAT_3D, 10, T, 5, 6, 7)
    b.close()
    T5 = list(np.geomspace(0.5, 2.0, 5))
    b = Batch()
    lad = b.add_ladder(T5)
    b.add_instance(O.LAT_3D, 10, ladder=lad, seed_J=5, seed=6)
    b.set_tuning([[O.LAT_3D, 10, 5, 2, 2, 5, 1]])
    b.set_spread(False)
    b.finalize()
    assert b.shape(0)[4] == 1
    b.record_exchanges(8)
    b.run(7)
    b.sync()
    check_instance(b, 0, O.LAT_3D, 10, T5, 5, 6, 7)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("lat,L,nslots,shape", [
    # 3D on one CTA of two warps: 144 column tasks for 64 threads, so the
    # exchange pass's lanes loop over tasks and walk every plane themselves
    (O.LAT_3D, 12, 16, (1, 1, 2, 0)),
    (O.LAT_3D, 12, 6, (1, 1, 2, 0)),
    # 2D on small blocks: each warp walks and counts many tiles, with a warp
    # sum every three sites
    (O.LAT_2D, 32, 16, (1, 2, 2, 0)),
    (O.LAT_2D_OPEN_X, 24, 10, (1, 2, 2, 0)),
])
def test_exchange_counts_in_narrow_blocks(sab, lat, L, nslots, shape):
    """The exchange's difference counter in blocks with far fewer threads
    than the lattice has columns (or sites per colour): decisions, masks and
    spins still match parallel_tempering<>."""
    from simulated_annealing_b200.batch import Batch
    from test_gpu_batch import check_instance

    T = list(np.geomspace(0.5, 2.0, nslots) if lat == O.LAT_3D else np.geomspace(0.3, 1.6, nslots))
    b = Batch()
    lad = b.add_ladder(T)
    b.add_instance(lat, L, ladder=lad, seed_J=31 + L, seed=32 + L)
    b.set_tuning([[lat, L, nslots, *shape]])
    b.set_spread(False)
    b.finalize()
    assert b.shape(0) == (lat, L, nslots, *shape)
    b.record_exchanges(16)
    b.run(5)
    b.run(4)
    b.sync()
    check_instance(b, 0, lat, L, T, 31 + L, 32 + L, 9)
    b.close()
