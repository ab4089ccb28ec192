"""Autotuner of the batched engine's launch shapes (run on the GPU).

For each bucket (lattice, L, slots) it times the resident kernel over a full
batch of that shape with every candidate shape -- cluster size C (the
smallest whose shared memory fits, and the next three larger ones), slots
per lane SL (1, or 2 for an even slot count), the two-slot 3D walk's
high-register form, warps per block (3 up to one pass over the CTA's
columns, two at least) -- against the engine's built-in heuristics, and keeps a shape only
where it beats them. Results go to a JSON record and to the table compiled
into the library (csrc/sa_tuning.inc):

    python -m simulated_annealing_b200.autotune \\
        --json simulated_annealing_b200/tuning.json --inc simulated_annealing_b200/csrc/sa_tuning.inc

Rebuild the library afterwards; tests/test_gpu_tuning.py checks every tuned
shape bit for bit against the oracle.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

LAT_2D, LAT_2D_OPEN_X, LAT_3D = 0, 1, 2
CLUSTERS = [1, 2, 3, 4, 5, 6, 8, 10, 12, 16]
SMEM_BUDGET = 232448 - 8192  # the resident kernel's per-CTA budget (sa_batch.cu)
LADDER_2D = np.geomspace(0.3, 1.6, 16)
LADDER_3D = np.geomspace(0.5, 2.0, 16)

# the batched mix's buckets (16 slots) and the 32-temperature ensemble
BUCKETS = [(LAT_2D, L, 16) for L in (16, 24, 32, 48, 64)] + [(LAT_3D, L, 16) for L in (8, 12, 16, 20, 24)] + \
          [(LAT_3D, 16, 32)]
# single-slot anneals (the serving requests: every even size they come in,
# -H measured after every sweep), timed as full batches of that size
SERVE_BUCKETS = [(LAT_3D, L, 1) for L in range(8, 65, 2)] + [(LAT_2D, L, 1) for L in range(16, 129, 2)]
SERVE_SITES = 2_500_000  # sites per single-slot batch (~20 MB of spins)


def resident_bytes(lat, L, nslots, C):
    zc = L if lat == LAT_3D else 1
    ny = -(-L // C)
    return 2 * zc * ny * (L // 2) * nslots * 8


def candidates(lat, L, nslots):
    cmin = next((C for C in CLUSTERS if C <= L and resident_bytes(lat, L, nslots, C) <= SMEM_BUDGET), None)
    if cmin is None:
        return []
    Cs = [C for C in CLUSTERS if cmin <= C <= min(16, L)][:4]
    out = []
    for C in Cs:
        ny = -(-L // C)
        cols = ny * (L // 2)
        for SL in ([1, 2] if nslots % 2 == 0 else [1]):
            rp = 1
            while rp * SL < nslots:
                rp <<= 1
            his = [0, 1] if (SL == 2 and lat == LAT_3D) else [0]
            for hr in his:
                # the engine's caps: 12 warps for the high-register form, 8 for
                # two-slot 2D lanes in clusters, 16 for single-slot 3D (its walk
                # keeps more words live), else 20
                if hr:
                    cap = 12
                elif lat != LAT_3D and SL == 2 and C > 1:
                    cap = 8
                else:
                    cap = 16 if (lat == LAT_3D and SL == 1 and rp == 1) else 20
                # 3D: one lane group of rp lanes per column; 2D: warps take
                # tiles of 32 sites (the rp lanes of a site inside a tile)
                passes = max(1, -(-(cols * rp) // 32)) if lat == LAT_3D else max(1, -(-cols // 32))
                # several small blocks per SM often beat one large one: from
                # 3 warps up to one pass over the CTA's work (or the cap); two
                # warps at least (threads 0..63 hold one replica each)
                top = max(2, min(cap, passes))
                ws = sorted({w for w in (3, 4, 5, 6, 7, 8, 10, 12, 16, 20) if w <= top} | {top})
                for w in ws:
                    out.append((lat, L, nslots, C, SL, w, hr))
    return out


def time_shape(lat, L, nslots, n, tuning, sweeps, stream):
    import torch

    from simulated_annealing_b200.batch import Batch

    b = Batch()
    if nslots == 1:
        sch = b.add_schedule(np.linspace(3.0, 0.2, 1000), 100)
        for k in range(n):
            b.add_instance(lat, L, schedule=sch, seed_J=1000 + k, seed=1000 + k)
    else:
        lad = b.add_ladder(np.geomspace(0.5, 2.0, nslots) if lat == LAT_3D else np.geomspace(0.3, 1.6, nslots))
        for k in range(n):
            b.add_instance(lat, L, ladder=lad, seed_J=1000 + k, seed=1000 + k)
    b.set_tuning(tuning)
    b.set_spread(False)
    b.finalize()
    b.set_stream(stream.cuda_stream)
    shape = b.shape(0)
    b.run(sweeps)
    b.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run(sweeps)
    b.run(sweeps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    rate = b.site_slots() * 64 * 2 * sweeps / (ms * 1e6)
    b.close()
    return rate, shape


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--json", default=None)
    ap.add_argument("--inc", default=None)
    ap.add_argument("--instances", type=int, default=410, help="instances per bucket (a full GPU)")
    ap.add_argument("--sweeps", type=int, default=40)
    ap.add_argument("--margin", type=float, default=0.01, help="keep a shape only if this much faster")
    ap.add_argument("--buckets", choices=["mix", "serve", "all"], default="all")
    ap.add_argument("--keep", default=None, help="a JSON record whose table entries for other buckets are kept")
    ap.add_argument("--only", nargs="+", default=None, metavar="LAT:L:SLOTS",
                    help="tune these buckets instead of a --buckets set (e.g. 2:8:1)")
    args = ap.parse_args()
    stream = torch.cuda.Stream()
    record = {"device": torch.cuda.get_device_name(0), "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
              "instances": args.instances, "sweeps": args.sweeps, "buckets": []}
    table = []
    buckets = {"mix": BUCKETS, "serve": SERVE_BUCKETS, "all": BUCKETS + SERVE_BUCKETS}[args.buckets]
    if args.only:
        buckets = [tuple(int(v) for v in b.split(":")) for b in args.only]
    if args.keep:
        old = json.load(open(args.keep))
        mine = {tuple(b) for b in buckets}
        table = [e for e in old["table"] if tuple(e[:3]) not in mine]
        record["buckets"] = [b for b in old["buckets"] if tuple(b["bucket"]) not in mine]
    for lat, L, nslots in buckets:
        n = args.instances if nslots > 1 else max(8, SERVE_SITES // (L ** 3 if lat == LAT_3D else L * L))
        base, base_shape = time_shape(lat, L, nslots, n, [], args.sweeps, stream)
        best, best_rate = None, base
        tried = []
        for cand in candidates(lat, L, nslots):
            try:
                rate, shape = time_shape(lat, L, nslots, n, [list(cand)], args.sweeps, stream)
            except Exception as e:  # a shape the GPU cannot schedule
                tried.append({"shape": list(cand), "error": str(e)[:120]})
                continue
            tried.append({"shape": list(cand), "rate": round(rate, 1)})
            if rate > best_rate * (1 + args.margin) and (best is None or rate > best_rate):
                best, best_rate = list(cand), rate
        record["buckets"].append({"bucket": [lat, L, nslots], "heuristic_shape": list(base_shape),
                                  "heuristic_rate": round(base, 1), "best": best, "best_rate": round(best_rate, 1),
                                  "tried": tried})
        if best is not None:
            table.append(best)
        print(json.dumps(record["buckets"][-1]["bucket"]), "heuristic", round(base, 1), "best", best,
              round(best_rate, 1), flush=True)
    record["table"] = sorted(table)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(record, f, indent=1)
    if args.inc:
        write_inc(args.inc, record["table"], record)


def write_inc(path, table, record):
    with open(path, "w") as f:
        f.write("// Launch shapes of the resident kernel per bucket, measured on a "
                f"{record.get('device', 'GPU')} by simulated_annealing_b200/autotune.py\n")
        f.write("// (lattice, L, slots, C, SL, warps, hr); see simulated_annealing_b200/tuning.json.\n")
        for e in table:
            f.write("{" + ", ".join(str(int(v)) for v in e) + "},\n")


if __name__ == "__main__":
    main()
