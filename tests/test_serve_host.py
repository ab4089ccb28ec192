"""Host logic of serving, on the CPU: the C5 request stream and the open loop
(admission in arrival order, waiting for room, latency from arrival to
result), driven through a stand-in server with the Server interface."""
import math

import numpy as np

import bench
from simulated_annealing_b200.serve import Request, run_open_loop


def test_c5_stream_shape():
    reqs = bench.c5_requests(4000, 2000.0)
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0)
    assert abs(np.mean(np.diff(t)) - 1 / 2000.0) < 0.05 / 2000.0  # Poisson at 2,000/s
    two = np.array([r.lattice == "2d" for r in reqs])
    assert abs(two.mean() - 0.5) < 0.03
    for r in reqs:
        lo, hi = (16, 128) if r.lattice == "2d" else (8, 64)
        assert lo <= r.L <= hi and r.L % 2 == 0
        assert r.sweeps_per_step == 100 and 10 <= len(r.T) <= 1000
        assert r.T[0] == 3.0 and (len(r.T) == 1 or abs(r.T[-1] - 0.2) < 1e-12)
    # log-uniform sweeps: the median of log10(sweeps) sits near 4
    med = np.median([math.log10(len(r.T) * 100) for r in reqs])
    assert abs(med - 4.0) < 0.1
    assert reqs[0].seed_J == 10_000 and reqs[0].seed == 20_000
    assert bench.request_attempts(reqs[0]) == float(reqs[0].L ** (3 if reqs[0].lattice == "3d" else 2)) * 64 * \
        len(reqs[0].T) * 100


class FakeClock:
    """Advances a little on every reading and by the step cost on every round."""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-5
        return self.t


class FakeServer:
    """The Server interface with `capacity` request slots; a request finishes
    after ceil(total sweeps / chunk) rounds, a round costing 1 ms."""

    def __init__(self, clock, capacity):
        self.clock, self.capacity = clock, capacity
        self.live, self.done, self.next_id = {}, [], 0
        self.submitted, self.max_live = [], 0

    def submit(self, lattice, L, seed_J, seed, T, per):
        if len(self.live) >= self.capacity:
            return None
        rid = self.next_id
        self.next_id += 1
        self.live[rid] = len(T) * per
        self.submitted.append(seed_J)
        self.max_live = max(self.max_live, len(self.live))
        return rid

    def step(self, chunk):
        self.clock.t += 1e-3
        for rid in list(self.live):
            self.live[rid] -= chunk
            if self.live[rid] <= 0:
                del self.live[rid]
                self.done.append(rid)

    def poll(self):
        d, self.done = self.done, []
        return d

    def sync(self):
        pass

    def result(self, rid):
        return ("result", rid)


def test_open_loop_admits_in_arrival_order_and_waits_for_room():
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(40):
        steps = int(rng.integers(1, 9))
        reqs.append(Request(0.0005 * k, "3d", 8, k, 100 + k, np.linspace(2.0, 0.5, steps), 100))
    clock = FakeClock()
    srv = FakeServer(clock, capacity=3)
    lat, res, wall = run_open_loop(srv, list(reqs), chunk=100, clock=clock)
    assert srv.submitted == list(range(40))  # arrival order
    assert srv.max_live <= 3                 # admission waits for room
    assert len(res) == 40 and set(res) == set(range(40))
    assert np.all(lat > 0) and wall > 0
    # a request needs ceil(sweeps / chunk) rounds of 1 ms once admitted
    for k, r in enumerate(reqs):
        assert lat[k] >= 1e-3 * math.ceil(len(r.T) * 100 / 100) - 1e-9
    assert wall >= 1e-3 * sum(len(r.T) for r in reqs) / 3 - 1e-9  # three slots at most


def test_open_loop_latency_is_arrival_to_result():
    # one request arriving at 2 ms, needing 3 rounds: done about 3 ms later
    reqs = [Request(0.002, "2d", 16, 1, 2, np.linspace(3.0, 0.2, 3), 100)]
    clock = FakeClock()
    srv = FakeServer(clock, capacity=4)
    lat, res, wall = run_open_loop(srv, reqs, chunk=100, clock=clock)
    assert res[0] == ("result", 0)
    assert 3e-3 <= lat[0] < 3.5e-3
    assert wall >= 5e-3
