"""The batched sweep of many small dots (qudos_b200.configs.batch_lenses):
solves per second of the batched mixed-precision path (eigenstates_batched,
several solves in flight) against a sequential loop of the plain FP64 path,
and the largest eigenvalue difference between the two.

    python -m qudos_b200.batch [--instances 64] [--threads 8] [--seed 0]

Prints one JSON line.  Table building is part of every solve in both arms.
"""

import argparse
import json
import os
import tempfile
import time

import numpy as np

import qudos_b200 as q
from qudos_b200 import configs
from qudos_b200 import lib as L


def measure(instances=64, threads=8, seed=0):
    """Both arms on the generated dots; returns the result dict."""
    decks = configs.batch_lenses(instances, seed)
    with tempfile.TemporaryDirectory() as d:
        dirs = [configs.write_deck(os.path.join(d, "dot%03d" % i), p, c) for i, (p, c, _) in enumerate(decks)]
        # warm-up (module loading, pools) on the smallest and largest sizes
        for m in sorted({desc["mg"] for _, _, desc in decks}):
            k = next(i for i, (_, _, desc) in enumerate(decks) if desc["mg"] == m)
            q.Problem(dirs[k]).solve(q.QD_PREC_MIXED)
            q.Problem(dirs[k]).solve(q.QD_PREC_FP64)
        seq = [q.Problem(x) for x in dirs]
        L.check(L.lib.qd_device_synchronize())
        t0 = time.perf_counter()
        w64 = [p.solve(q.QD_PREC_FP64)[0] for p in seq]
        t_seq = time.perf_counter() - t0
        bat = [q.Problem(x) for x in dirs]
        L.check(L.lib.qd_device_synchronize())
        t0 = time.perf_counter()
        out = q.solve_batch(bat, q.QD_PREC_MIXED, threads)
        t_bat = time.perf_counter() - t0
    dE = max(float(np.abs(o[0] - w).max()) for o, w in zip(out, w64)) * 1e6
    sizes = {}
    for _, _, desc in decks:
        sizes[str(8 * (2 * desc["mg"] + 1) ** 3)] = sizes.get(str(8 * (2 * desc["mg"] + 1) ** 3), 0) + 1
    return {"instances": instances, "threads": threads, "n_h_counts": sizes,
            "sequential_fp64_solves_per_s": instances / t_seq,
            "batched_mixed_solves_per_s": instances / t_bat, "speedup": t_seq / t_bat,
            "max_dE_ueV_batched_mixed_vs_sequential_fp64": dE,
            "note": "wall clock, host-driven; every solve builds its tables, assembles H and solves "
                    "16 states (4 e + 4 h Kramers pairs)"}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--threads", type=int, default=8)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    print(json.dumps(measure(a.instances, a.threads, a.seed)), flush=True)


if __name__ == "__main__":
    main()
