#!/usr/bin/env python
"""Benchmark: replica spin-flip attempts/ns of the batched persistent engine.

Workload (the batched mix): 4,096 independent +-J disorder instances, shapes
drawn uniformly (numpy PCG64, seed 4096) from 2D L in {16,24,32,48,64} and 3D
L in {8,12,16,20,24}, couplings and spins from seed 1000+index, 64 replicas per
word, each a 16-temperature parallel-tempering ensemble (geometric 0.5-2.0 in
3D, 0.3-1.6 in 2D) with an exchange attempt after every sweep. A step is one
persistent launch of `--sweeps-per-step` sweeps over every instance. Data are
synthetic (seeded), generated on the device from the seeds.

value      attempts / device time (CUDA events on the launch stream, state
           resident in HBM; the whole state, 1.9 GB of spins, exceeds L2).
e2e        the same through the public API with host buffers: each step uploads
           its exchange decisions (generated on the host by the reference's
           std::mt19937(123) sequence) and downloads every slot's energies and
           the acceptance counters into pinned host memory; host wall clock.
roofline   algorithmic bytes per launch (per site and slot and sweep: spins read
           twice and written once, 24 B; couplings 2*dim words per site, shared
           by the 16 slots) / average launch time, against the measured HBM copy
           bandwidth.
cpu_baseline / --impl reference: the reference's own CPU classes (cpu_2d,
           cpu_3d, parallel_tempering<>) compiled from its sources, on a bounded
           sample of the same instances, timed on this host: one instance per
           host thread (the template's OpenMP loop over slots set to 1 thread),
           as many threads as cores.
plain      the plain one-instance-per-launch form on the same GPU: each
           instance of a bounded sample alone in its own batch (the engine's
           resident kernel, one launch of --sweeps-per-step sweeps with an
           exchange per sweep), launched back to back on one stream;
           batched_over_plain = value / its rate.
plain_host_driven  the reference's own driving pattern on the same GPU
           (simulated_annealing_b200/sa_plain_pt: one system per slot, one
           launch per half-sweep, a measurement copy per slot per sweep and a
           host exchange per sweep, as parallel_tempering<gpu_sys> drives
           gpu_3d).
serving    continuous batching of anneal requests (simulated_annealing_b200.serve):
           Poisson arrivals at 2,000/s, 2D L 16..128 or 3D L 8..64 with equal
           probability (L log-uniform, rounded to even), sweeps log-uniform in
           [1e3, 1e5], linear T 3.0 -> 0.2 in steps of 100 sweeps, couplings and
           spins from per-request seeds; p50/p99 time from arrival to result on
           the host clock and aggregate attempts/ns. The default run serves the
           first --serve-requests (300) requests of that stream at 2,000/s and
           the first half of them at --serve-sustainable-rate (30/s), a rate the
           GPU keeps up with; --workload serve runs the whole 20,000 (or
           --serve-requests) at --serve-rate.

--gpus N   one process per GPU (torch.distributed over NCCL): when WORLD_SIZE is
           unset the script launches its N ranks itself (torch.distributed.run
           on 127.0.0.1); every rank runs its own block of the instance
           sequence (weak scaling, no collective on the data path) and rank 0
           prints the line with the max-over-ranks times.

--workload c1|c2|c3 time the single-lattice cases instead (2D L=64 T=1.0 for
10,000 sweeps; 3D L=32 anneal 3.0 -> 0.2 over 200 x 100 sweeps; 3D L=16
32-temperature parallel tempering with an exchange every sweep).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPES = [(0, 16), (0, 24), (0, 32), (0, 48), (0, 64), (2, 8), (2, 12), (2, 16), (2, 20), (2, 24)]
LADDER_2D = np.geomspace(0.3, 1.6, 16)
LADDER_3D = np.geomspace(0.5, 2.0, 16)
METRIC = "spin-flip attempts/ns"
UNIT = "attempts/ns"
FALLBACK_HBM_GBS = 6650.0


def c4_instances(n: int, index_offset: int = 0):
    rng = np.random.default_rng(4096)
    picks = rng.integers(0, len(SHAPES), size=n + index_offset)[index_offset:]
    return [(SHAPES[p][0], SHAPES[p][1], 1000 + index_offset + k) for k, p in enumerate(picks)]


def shard_instances(rank: int, world: int, n: int, shape=None):
    """Rank `rank`'s share of a `world`-rank run: instances [rank*n, (rank+1)*n)
    of the global sequence (weak scaling: n per rank, no overlap). With
    `shape` = (lattice, L) every instance has that one shape (a small case of
    one group of the mix, for profiling)."""
    assert 0 <= rank < world
    if shape is not None:
        return [(shape[0], shape[1], 1000 + rank * n + k) for k in range(n)]
    return c4_instances(n, index_offset=rank * n)


def parse_shape(text):
    """'LAT:L' (lattice 0 = 2D, 2 = 3D) -> (lattice, L), or None."""
    if not text:
        return None
    lat, L = (int(v) for v in text.split(":"))
    if (lat, L) not in SHAPES:
        raise SystemExit(f"--shape {text}: not a shape of the mix {SHAPES}")
    return lat, L


def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank timings (the whole job ends when the
    slowest rank does)."""
    import torch

    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def site_count(lat: int, L: int) -> int:
    return L ** 3 if lat == 2 else L * L


def algorithmic_bytes_per_sweep(insts, nslots=16) -> int:
    total = 0
    for lat, L, _ in insts:
        N = site_count(lat, L)
        d = 3 if lat == 2 else 2
        total += 24 * N * nslots + 16 * d * N
    return total


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def launch_traffic_bytes(insts, nslots=16) -> int:
    """DRAM bytes one launch of the resident kernel moves: every instance's
    spins come from HBM into shared memory once and go back once, and its
    couplings (compact: dim words per site) are read once; the sweeps in
    between run out of shared memory and L2. An ncu capture of a small case
    of the same kernel (dram__bytes_read.sum + dram__bytes_write.sum) agrees
    with this count; it does not grow with the sweeps per launch."""
    total = 0
    for lat, L, _ in insts:
        N = site_count(lat, L)
        d = 3 if lat == 2 else 2
        total += 2 * 8 * N * nslots + 8 * d * N
    return total


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        med = statistics.median(sm) if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU
def cpu_reference_sample(insts, budget_s: float, sweeps_per_instance: int = 50, threads: int = 0):
    """The reference's parallel_tempering<cpu_sys> over cpu_2d / cpu_3d systems
    (built as its driver builds them: set_seed; init_J; set_seed; init_rand), on
    the first instances of the workload until `budget_s` of CPU work is done.
    One instance per host thread, each thread's OpenMP loop over the slots set
    to one thread, as many threads as cores (ctypes releases the GIL during
    the reference's calls)."""
    ncpu = threads or os.cpu_count() or 1
    from oracle import oracle as O

    if not O.ref_available():
        O.build()
    lib = O.ref_lib()
    lock = threading.Lock()
    state = {"next": 0, "attempts": 0, "done": 0, "rate": 0.0}
    t0 = time.perf_counter()
    deadline = t0 + budget_s

    def work():
        lib.ref_omp_threads(1)
        att, busy = 0, 0.0
        while True:
            with lock:
                if time.perf_counter() > deadline or state["next"] >= len(insts):
                    state["rate"] += att / busy if busy > 0 else 0.0
                    return
                k = state["next"]
                state["next"] += 1
            lat, L, seed = insts[k]
            T = LADDER_3D if lat == 2 else LADDER_2D
            systems = [O.RefSystem(lat, L) for _ in T]
            for s in systems:
                s.set_seed(seed)
                s.init_J()
                s.set_seed(seed)
                s.init_rand()
            pt = O.RefPT(systems, list(T), 1)
            ts = time.perf_counter()
            for _ in range(sweeps_per_instance):
                pt.step(0)
            busy += time.perf_counter() - ts
            a = sweeps_per_instance * len(T) * site_count(lat, L) * 64
            att += a
            with lock:
                state["attempts"] += a
                state["done"] += 1

    threads_ = [threading.Thread(target=work) for _ in range(ncpu)]
    for th in threads_:
        th.start()
    for th in threads_:
        th.join()
    dt = time.perf_counter() - t0
    # every thread's attempts over its own stepping time (systems are built
    # outside the timed loops), summed over the concurrently running threads
    value = state["rate"] / 1e9
    sample = (f"{state['done']} instances of the mix x 16 slots x {sweeps_per_instance} sweeps "
              f"(+ exchange each sweep; the template measures every slot before it), {ncpu} instance "
              f"threads x 1 OpenMP thread, {dt:.1f} s")
    return {"value": value, "unit": UNIT, "cores": ncpu, "kind": "reference", "sample": sample,
            "per_core": value / ncpu}


# ----------------------------------------------------------------------------- plain form
def plain_host_driven_sample(insts, budget_s: float, sweeps: int = 20):
    """The reference's driving pattern over the first instances of the workload
    (sa_plain_pt: one system per slot, one launch per half-sweep, a blocking
    measurement per slot per sweep and a host exchange), until `budget_s` of
    timed loops."""
    exe = os.path.join(ROOT, "simulated_annealing_b200", "sa_plain_pt")
    lines = []
    for lat, L, seed in insts:
        T = LADDER_3D if lat == 2 else LADDER_2D
        lines.append(f"{lat} {L} {seed} {len(T)} " + " ".join(repr(float(t)) for t in T))
    r = subprocess.run([exe, str(budget_s), str(sweeps)], input="\n".join(lines) + "\n", capture_output=True,
                       text=True, timeout=budget_s * 10 + 120)
    if r.returncode != 0:
        raise RuntimeError(f"sa_plain_pt failed: {r.stderr.strip()[-300:]}")
    f = r.stdout.split()
    done, att, sec = int(f[1]), float(f[3]), float(f[5])
    return {"value": att / sec / 1e9, "unit": UNIT,
            "sample": f"{done} instances of the mix x 16 slots x {sweeps} sweeps (+ exchange each sweep), "
                      f"{sec:.1f} s of timed loops"}


def plain_per_instance_sample(insts, sweeps: int, stream, reps: int = 2):
    """The plain one-instance-per-launch form: every instance of `insts` alone
    in its own batch (the resident kernel, one launch of `sweeps` sweeps with
    an exchange per sweep), the launches back to back on one stream; device
    time (CUDA events) over `reps` rounds after one warm-up round."""
    import torch

    from simulated_annealing_b200.batch import Batch

    batches = []
    for lat, L, seed in insts:
        b = Batch()
        lad = b.add_ladder(LADDER_3D if lat == 2 else LADDER_2D)
        b.add_instance(lat, L, ladder=lad, seed_J=seed, seed=seed)
        b.finalize()
        b.set_stream(stream.cuda_stream)
        batches.append(b)
    for b in batches:
        b.run(sweeps)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        for b in batches:
            b.run(sweeps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    att = reps * sweeps * 64 * sum(b.site_slots() for b in batches)
    launches = reps * sum(b.launches_per_run() for b in batches)
    for b in batches:
        b.close()
    return {"value": att / (ms * 1e6), "unit": UNIT,
            "sample": f"first {len(insts)} instances of the mix, each alone in its own batch, x 16 slots x "
                      f"{sweeps} sweeps (+ exchange each sweep), {reps} rounds of back-to-back launches "
                      f"({launches} launches, {ms:.1f} ms device time)"}


# ----------------------------------------------------------------------------- serving
def c5_requests(n: int, rate: float, seed: int = 2000):
    """The anneal-request stream: Poisson arrivals at `rate`/s (numpy PCG64 seed
    `seed`), 2D L in [16,128] or 3D L in [8,64] with equal probability, L
    log-uniform rounded to even, sweeps log-uniform in [1e3, 1e5] as steps of
    100 sweeps on a linear T 3.0 -> 0.2 schedule, seeds 10000+k / 20000+k."""
    from simulated_annealing_b200.serve import Request

    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for k in range(n):
        two = rng.random() < 0.5
        lo, hi = (16, 128) if two else (8, 64)
        L = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))) / 2)) * 2
        L = max(lo, min(hi, L))
        sweeps = float(np.exp(rng.uniform(np.log(1e3), np.log(1e5))))
        steps = max(1, int(round(sweeps / 100)))
        out.append(Request(float(t[k]), "2d" if two else "3d", L, 10_000 + k, 20_000 + k,
                           np.linspace(3.0, 0.2, steps), 100))
    return out


def request_attempts(r) -> float:
    N = r.L ** 3 if r.lattice == "3d" else r.L * r.L
    return float(N) * 64 * len(r.T) * r.sweeps_per_step


def serving_run(n: int, rate: float, budget_gb: float, chunk: int = 100):
    from simulated_annealing_b200.serve import Server, run_open_loop

    reqs = c5_requests(n, rate)
    srv = Server(budget_bytes=int(budget_gb * (1 << 30)), max_requests=max(n, 1))
    lat, res, wall = run_open_loop(srv, reqs, chunk=chunk)
    srv.close()
    att = sum(request_attempts(r) for r in reqs)
    return {"requests": n, "arrival_rate_per_s": rate, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(np.mean(lat)), "wall_s": wall,
            "attempts_per_ns": att / wall / 1e9, "budget_gb": budget_gb, "sweeps_per_round": chunk,
            "latency": "arrival -> result on the host (host clock)"}


# ----------------------------------------------------------------------------- GPU
def c4_config(args, world: int) -> dict:
    S = args.sweeps_per_step
    shape = parse_shape(getattr(args, "shape", None))
    if shape is not None:
        kind = "3D" if shape[0] == 2 else "2D"
        what = f"one group of the mix: {args.instances} instances of {kind} L={shape[1]} x 16 slots"
    else:
        what = f"batched PT mix: {args.instances} instances x 16 slots, 2D L{{16..64}} / 3D L{{8..24}}"
    return {"workload": f"{what}, {S} sweeps + exchange per sweep per step",
            "instances_per_gpu": args.instances, "slots": 16, "sweeps_per_step": S,
            "l2": ("inputs larger than L2 (1.9 GB of spins)" if shape is None
                   else "one-shape case: spins of all its instances, see instances"),
            "parallelism": f"instances sharded, {world} GPU(s), no collective"}


def build_c4_batch(insts, stream_ptr=None, group_timing=False):
    """The batched mix as the bench runs it: one batch, the two 16-slot
    ladders, the instances in order (tests build the same batch)."""
    from simulated_annealing_b200.batch import Batch

    b = Batch()
    if group_timing:
        b.set_group_timing(True)
    l2 = b.add_ladder(LADDER_2D)
    l3 = b.add_ladder(LADDER_3D)
    for lat, L, seed in insts:
        b.add_instance(lat, L, ladder=(l3 if lat == 2 else l2), seed_J=seed, seed=seed)
    b.finalize()
    if stream_ptr is not None:
        b.set_stream(stream_ptr)
    return b


def init_ranks(backend: str):
    """(world, rank, local_rank, dist module or None) from the torchrun
    environment; the process group has a short timeout so that ranks waiting
    for a dead peer end with an error."""
    import datetime

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        dist_mod.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        dist = dist_mod
    return world, rank, local, dist


def run_stub(args):
    """The multi-rank plumbing without a GPU (gloo): each rank takes its shard
    of the instance sequence, reports a stand-in time that grows with its rank,
    and rank 0 prints the line built from the max over ranks. Used by the CPU
    tests of the launcher."""
    world, rank, _, dist = init_ranks("gloo")
    insts = shard_instances(rank, world, args.instances)
    ms = 10.0 + rank
    seeds = sum(s for _, _, s in insts)
    ms, = max_over_ranks([ms], dist, "cpu")
    tot = max_over_ranks([float(seeds)], None, "cpu")[0]
    if dist:
        import torch

        t = torch.tensor([tot], dtype=torch.float64)
        dist.all_reduce(t)
        tot = float(t[0])
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": None, "unit": UNIT, "n_gpus": world, "ms_per_step": ms,
                          "stub": True, "instances_total": world * args.instances, "seed_sum": tot}), flush=True)
    if dist:
        dist.destroy_process_group()


def run_ours(args):
    import torch

    world, rank, local, dist = init_ranks("nccl")
    torch.cuda.set_device(local)

    insts = shard_instances(rank, world, args.instances, parse_shape(args.shape))
    stream = torch.cuda.Stream()
    b = build_c4_batch(insts, stream.cuda_stream, group_timing=True)
    S = args.sweeps_per_step
    site_slots = b.site_slots()
    attempts_step = site_slots * 64 * S
    n_launch = b.launches_per_run()  # one launch per shape group

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    for _ in range(args.warmup):
        b.run(S)
    b.sync()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        b.run(S)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    barrier()

    # the end of every shape group in the last timed step (one stream per
    # group; the step ends with the slowest)
    groups = b.group_times()

    # e2e through the public API with host buffers (pinned)
    E_host = torch.empty(b.energy_count(), dtype=torch.int64, pin_memory=True)
    npairs = b.num_pairs()
    acc_host = torch.empty(max(npairs, 1), dtype=torch.int64, pin_memory=True)
    att_host = torch.empty(max(npairs, 1), dtype=torch.int64, pin_memory=True)
    h2d = []
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        b.run(S)
        h2d.append(b.last_h2d_bytes())
        b.energies_into(E_host.data_ptr())
        b.acceptance_into(acc_host.data_ptr(), att_host.data_ptr())
        b.sync()
    t_e2e = time.perf_counter() - t0
    barrier()

    ms, e2e_ms = max_over_ranks([ms, t_e2e * 1e3], dist, "cuda")
    total_attempts = attempts_step * args.steps * world
    value = total_attempts / (ms * 1e6)
    e2e_value = total_attempts / (e2e_ms * 1e6)

    if rank == 0:
        peak, peak_src = measured_hbm_peak()
        # the groups of one step run concurrently (one stream each): the unit
        # of the roofline is the step's batched pass over every instance
        bytes_launch = algorithmic_bytes_per_sweep(insts) * S
        launch_s = (ms / 1e3) / args.steps
        achieved = bytes_launch / launch_s / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 (bitwise/int32)", "data": "synthetic",
            "config": dict(c4_config(args, world), site_slots_per_gpu=site_slots),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(np.mean(h2d)) if h2d else 0,
                    "d2h_bytes_per_step": int(E_host.numel() * 8 + 2 * npairs * 8)},
            "gpu_launches": args.steps * n_launch,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": launch_traffic_bytes(insts),
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                         else "fallback 6650 GB/s",
                         "algorithmic_bytes_per_launch": bytes_launch,
                         "note": "state resident in shared memory for a launch: the DRAM traffic per launch "
                                 "(spins in and out once, couplings once) is far below the algorithmic bytes; "
                                 "the kernel is bound by integer-ALU issue"},
            "clocks": clk,
            "groups_last_step": groups,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_reference_sample(insts, args.cpu_budget)
        if world == 1 and args.plain_instances > 0:
            pl = plain_per_instance_sample(insts[:args.plain_instances], S, stream)
            line["plain"] = pl
            line["batched_over_plain"] = value / pl["value"]
        if world == 1 and args.plain_budget > 0:
            line["plain_host_driven"] = plain_host_driven_sample(insts, args.plain_budget)
        if world == 1 and args.serve_requests > 0:
            line["serving"] = serving_run(args.serve_requests, 2000.0, args.serve_budget_gb)
            # the same stream at an arrival rate the GPU sustains (arrivals spread
            # over ~5 s instead of queueing up at once)
            line["serving_sustainable"] = serving_run(args.serve_requests // 2, args.serve_sustainable_rate,
                                                      args.serve_budget_gb)
        print(json.dumps(line), flush=True)
    b.close()
    if dist:
        dist.destroy_process_group()


def launch_ranks(n: int) -> int:
    """Runs this script as n ranks on 127.0.0.1 (torch.distributed.run) and
    returns their exit status; the ranks read WORLD_SIZE/RANK/LOCAL_RANK."""
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    insts = c4_instances(args.instances)
    per_step = []
    samples = []
    for k in range(args.warmup + args.steps):
        r = cpu_reference_sample(insts[(k * 7) % len(insts):], args.ref_step_budget, sweeps_per_instance=20)
        if k >= args.warmup:
            per_step.append(r)
    vals = [r["value"] for r in per_step]
    value = float(np.mean(vals))
    samples = per_step[-1]["sample"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": args.ref_step_budget * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64 (bitwise) + f64 compare", "data": "synthetic",
        "config": c4_config(args, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": per_step[-1]["cores"], "kind": "reference",
                         "sample": "per step: " + samples, "per_core": value / per_step[-1]["cores"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_single(args):
    """One JSON line for the serving stream or a single-lattice case."""
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    base = {"n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 (bitwise/int32)", "data": "synthetic"}
    if args.workload == "serve":
        clocks.start()
        n = args.serve_requests if args.serve_requests else 20_000
        r = serving_run(n, args.serve_rate, min(120.0, args.serve_budget_gb))
        line = dict(base, metric="anneal time-to-result p99 (s)", value=r["p99_s"], unit="s",
                    higher_is_better=False,
                    config={"workload": f"serving: the first {n} anneal requests of the stream, Poisson "
                                        f"{args.serve_rate:g}/s"},
                    serving=r)
        line["clocks"] = clocks.stop()
        print(json.dumps(line), flush=True)
        return
    from simulated_annealing_b200.batch import Batch
    from simulated_annealing_b200.system import GpuSystem

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream()
    if args.workload == "c1":
        s = GpuSystem("2d", 64, 1.0)
        s.set_seed(1); s.init_J(); s.set_seed(2); s.init_rand()
        for _ in range(args.warmup):
            s.sweep(1000)
        s.sync()
        clocks.start()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            s.sweep(10_000)
        s.sync()
        dt = time.perf_counter() - t0
        att = 10_000 * 4096 * 64 * args.steps
        wl = "2D L=64 periodic, T=1.0, 10,000 sweeps per step (one resident-kernel launch per step)"
    elif args.workload == "c2":
        s = GpuSystem("3d", 32, 3.0)
        s.set_seed(3); s.init_J(); s.set_seed(3); s.init_rand()
        T = np.linspace(3.0, 0.2, 200)
        for _ in range(args.warmup):
            s.anneal(T[:10], 100, 1)
        s.sync()
        clocks.start()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            s.anneal(T, 100, 1)
        s.sync()
        dt = time.perf_counter() - t0
        att = 20_000 * 32768 * 64 * args.steps
        wl = "3D L=32 anneal, linear T 3.0 -> 0.2 over 200 steps x 100 sweeps, measure every sweep"
    else:
        b = Batch()
        lad = b.add_ladder(np.geomspace(0.5, 2.0, 32))
        b.add_instance(2, 16, ladder=lad, seed_J=4, seed=4)
        b.finalize()
        b.set_stream(stream.cuda_stream)
        S = 10_000
        for _ in range(args.warmup):
            b.run(1000)
        b.sync()
        clocks.start()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            b.run(S)
        b.sync()
        dt = time.perf_counter() - t0
        att = S * 4096 * 32 * 64 * args.steps
        wl = "3D L=16 x 32 temperatures (geometric 0.5-2.0), exchange every sweep, 10,000 sweeps per step"
    clk = clocks.stop()
    line = dict(base, metric=METRIC, value=att / dt / 1e9, unit=UNIT, ms_per_step=dt * 1e3 / args.steps,
                config={"workload": wl, "timing": "host clock around synchronised steps"}, clocks=clk)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sweeps-per-step", type=int, default=100)
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--shape", default=None, metavar="LAT:L",
                    help="every instance of this one shape of the mix (e.g. 2:24; a small case for profiling)")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-step-budget", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-instances", type=int, default=100,
                    help="instances of the plain one-instance-per-launch sample (0 = skip)")
    ap.add_argument("--plain-budget", type=float, default=6.0,
                    help="seconds of the host-driven plain form (0 = skip)")
    ap.add_argument("--cpu-stub", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--serve-requests", type=int, default=None,
                    help="requests in the serving sample (0 = skip; default 300, or 20,000 for --workload serve)")
    ap.add_argument("--serve-budget-gb", type=float, default=16.0)
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="arrivals/s of --workload serve")
    ap.add_argument("--serve-sustainable-rate", type=float, default=30.0,
                    help="arrivals/s of the default line's second serving sample")
    ap.add_argument("--workload", choices=["c4", "serve", "c1", "c2", "c3"], default="c4")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args.gpus))
    if args.cpu_stub:
        return run_stub(args)
    if args.serve_requests is None and args.workload == "c4":
        args.serve_requests = 300
    if args.workload != "c4" and args.impl == "ours":
        return run_single(args)
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
