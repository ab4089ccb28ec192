#!/usr/bin/env python
"""Digests of the --bulk output of gen_curand_golden.cu (cuRAND's own
Philox4_32_10 outputs, made on a GPU): one SHA-256 per seed for the curand()
words and one for the curand_uniform() bit patterns, each over
[subsequence][draw] little-endian u32. Prints the JSON fixture
tests/golden/curand_philox_bulk.json.

  python tests/golden/hash_curand_bulk.py curand_bulk.bin > tests/golden/curand_philox_bulk.json
"""
import hashlib
import json
import sys

import numpy as np

SEEDS = [1, 2, 3, 4, 1234, 1000, 1001, 1002, 1003]
SUBS, DRAWS = 4096, 64


def main(path):
    a = np.fromfile(path, dtype="<u4")
    per = SUBS * DRAWS
    assert a.size == len(SEEDS) * 2 * per, a.size
    out = {"generator": "curand Philox4_32_10 device API: curand_init(seed, subsequence, 0), curand, curand_uniform",
           "subsequences": SUBS, "draws": DRAWS, "seeds": {}}
    for i, seed in enumerate(SEEDS):
        u = a[(2 * i) * per:(2 * i + 1) * per]
        f = a[(2 * i + 1) * per:(2 * i + 2) * per]
        out["seeds"][str(seed)] = {"u32_sha256": hashlib.sha256(u.tobytes()).hexdigest(),
                                   "uniform_bits_sha256": hashlib.sha256(f.tobytes()).hexdigest()}
    json.dump(out, sys.stdout, indent=1)
    print()


if __name__ == "__main__":
    main(sys.argv[1])
