"""Autotuner of the dense->band reduction's aggregation depth.

The reduction (eig_stage1.cu) accumulates the Householder panels' (V, W)
pairs and applies them to the trailing matrix in one rank-2K update every
K / 32 panels.  K trades the trailing matrix's HBM traffic (one read and
write per flush) against the tall-skinny correction products, which grow
with K; the best K depends on the matrix order and on the precision.

    python -m qudos_b200.autotune [--mg 3,4,5,7] [--depths 128,192,256] [--reps 2] [--out tuning.json]

times one assembly + windowed solve of the lens-molecule deck
(configs.molecule_15 at each plane-wave cutoff) for every depth and both
precisions, with CUDA events on the device, and writes the fastest depth per
(N_H, precision) to a JSON cache.  `load()` puts a cache into the library's
tuning table (qd_tuning_set): an entry covers every order up to its N_H, the
largest entry every order above.  `qudos_b200.Problem` loads the package's
cache (qudos_b200/tuning.json) the first time it is used, so the solves and
the batched solves of the package run with the tuned depths.
"""

import argparse
import json
import os
import tempfile

import numpy as np

from . import configs
from . import lib as L

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")
PRECS = {"fp64": L.QD_PREC_FP64, "mixed": L.QD_PREC_MIXED}
_loaded = None


def load(path=CACHE):
    """Fills the library's tuning table from a cache; returns the number of
    entries (0 when the file does not exist)."""
    global _loaded
    L.check(L.lib.qd_tuning_set(0, 0, 0))
    _loaded = path
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        cache = json.load(f)
    n = 0
    for prec in PRECS:
        ent = sorted((e for e in cache["entries"] if e["prec"] == prec), key=lambda e: e["n_h"])
        for i, e in enumerate(ent):
            bound = e["n_h"] if i + 1 < len(ent) else (1 << 62)
            L.check(L.lib.qd_tuning_set(PRECS[prec], bound, int(e["depth"])))
            n += 1
    return n


def ensure_loaded(path=CACHE):
    """load() once per process."""
    if _loaded is None:
        load(path)


def _time_solves(pr, prec, reps):
    """Mean device time (ms) of assembly + windowed solve, after one warm-up."""
    n, lo, hi = pr.n_h, pr.lo, pr.hi
    M = hi - lo + 1
    H = L.DeviceBuffer(n * n * 16)
    Z = L.DeviceBuffer(n * M * 16)
    W = L.DeviceBuffer(M * 8)
    e0, e1 = L.Event(), L.Event()
    try:
        def step():
            L.check(L.lib.qd_problem_assemble_dev(pr.handle, H.ptr, n, 0, L.QD_PREC_FP64, None))
            L.check(L.lib.qd_eigh_window_dev(n, H.ptr, n, lo, hi, prec, W.ptr, Z.ptr, n, None))

        step()
        L.check(L.lib.qd_device_synchronize())
        e0.record()
        for _ in range(reps):
            step()
        e1.record()
        return e0.elapsed_ms(e1) / reps
    finally:
        H.free()
        Z.free()
        W.free()


def sweep(mgs=(3, 4, 5, 7), depths=(128, 160, 192, 224, 256), precs=("mixed", "fp64"), reps=2, path=CACHE):
    """Times every depth for every cutoff and precision and writes the cache;
    returns it."""
    from . import pwem
    entries = []
    for mg in mgs:
        with tempfile.TemporaryDirectory() as d:
            configs.write_deck(d, *configs.molecule_15(mg=mg))
            pr = pwem.Problem(d, tuned=False)
            pr.build_tables()
        for prec in precs:
            times = {}
            for k in depths:
                L.check(L.lib.qd_tuning_set(0, 0, 0))
                L.check(L.lib.qd_tuning_set(PRECS[prec], 1 << 62, int(k)))
                times[str(k)] = _time_solves(pr, PRECS[prec], reps)
            best = min(times, key=times.get)
            entries.append({"n_h": pr.n_h, "prec": prec, "depth": int(best), "ms": times})
            print("N_H=%d %s: depth %s (%s)" % (pr.n_h, prec, best,
                                               ", ".join("%s: %.1f ms" % kv for kv in times.items())), flush=True)
    L.check(L.lib.qd_tuning_set(0, 0, 0))
    cache = {"workload": "configs.molecule_15 at each cutoff: assembly + windowed solve of 32 states, "
                         "mean of %d solves after one warm-up, CUDA events" % reps,
             "entries": entries}
    with open(path, "w") as f:
        json.dump(cache, f, indent=1)
    load(path)
    return cache


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mg", default="3,4,5,7")
    ap.add_argument("--depths", default="128,160,192,224,256")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--out", default=CACHE)
    a = ap.parse_args(argv)
    sweep([int(x) for x in a.mg.split(",")], [int(x) for x in a.depths.split(",")], reps=a.reps, path=a.out)


if __name__ == "__main__":
    main()
