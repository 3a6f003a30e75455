"""Converged outer-iteration counts of the reference (FP64 build, one OpenMP
thread) on a seeded subsample of the 64-design density-field mix.

Test/benchmark infrastructure: bench.py's reference arm for the many-design
workloads multiplies these counts by per-iteration times it measures on the
host cores, as the reference itself cannot be run to convergence on every
design within a benchmark.  Output: oracle/mix_reference_counts.json.

    python oracle/mix_counts.py [--workers 7]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from multiprocessing import get_context

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

SUBSAMPLE_SEED = 2024
SUBSAMPLE = 8
EPS = 1e-6
MAX_OUTER = 200000


def subsample() -> list:
    import numpy as np
    return sorted(int(k) for k in np.random.default_rng(SUBSAMPLE_SEED).choice(64, SUBSAMPLE, replace=False))


def count(k: int) -> dict:
    from coldplate_solver_b200 import geometry as g
    from oracle import reference
    d = g.batch_mix(64)[k]
    t = time.time()
    out = reference.run(d, MAX_OUTER, precision="f64", eps=EPS, stop_on_conv=True, threads=1, timeout=24 * 3600)
    err = out["err"]
    return {"k": k, "M": d.M, "N": d.N, "iters": int(len(err)), "last_err": float(err[-1]),
            "residMassDof": float(out["residMassDof"][-1]), "seconds": time.time() - t}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=max(1, (os.cpu_count() or 2) - 1))
    args = ap.parse_args()
    ks = subsample()
    rows = []
    with get_context("spawn").Pool(args.workers) as pool:
        for r in pool.imap_unordered(count, ks):
            rows.append(r)
            print(json.dumps(r), flush=True)
    rows.sort(key=lambda r: r["k"])
    with open(os.path.join(HERE, "mix_reference_counts.json"), "w") as f:
        json.dump({"mix": "geometry.batch_mix(64)", "subsample_seed": SUBSAMPLE_SEED, "eps": EPS,
                   "binary": "oracle/_ref/ref_f64, OMP_NUM_THREADS=1", "designs": rows}, f, indent=1)


if __name__ == "__main__":
    main()
