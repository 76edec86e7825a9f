"""Run a few solves of the two-lens molecule deck (qudos_b200.configs.molecule_15)
and print the per-stage times: the command that the committed ncu summaries
under profiles/ were captured from.

    python -m qudos_b200.profile_solve [--mg 7] [--prec mixed|fp64] [--solves 1]

One solve = H assembly (FP64, lower triangle) + the windowed eigensolve on
the device.  With QD_PROFILE=1 in the environment the dense->band reduction
is also broken down into its steps.
"""

import argparse
import os
import sys
import tempfile
import time

import qudos_b200 as q
from qudos_b200 import configs
from qudos_b200 import lib as L

STAGES = ["assembly", "band reduction", "bulge chasing", "bisection", "inverse iteration", "back-transform",
          "refinement"]
STEPS = ["panel refresh", "panel QR", "T and VT", "X = A22 VT", "corrections", "W", "append", "trailing update"]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mg", type=int, default=7)
    ap.add_argument("--prec", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--solves", type=int, default=1)
    a = ap.parse_args(argv)
    with tempfile.TemporaryDirectory() as d:
        configs.write_deck(d, *configs.molecule_15(mg=a.mg))
        pr = q.Problem(d)
        pr.build_tables()
    n, lo, hi = pr.n_h, pr.lo, pr.hi
    m = hi - lo + 1
    prec = q.QD_PREC_MIXED if a.prec == "mixed" else q.QD_PREC_FP64
    H = L.DeviceBuffer(n * n * 16)
    Z = L.DeviceBuffer(n * m * 16)
    W = L.DeviceBuffer(m * 8)
    for s in range(a.solves):
        t0 = time.perf_counter()
        L.check(L.lib.qd_problem_assemble_dev(pr.handle, H.ptr, n, 0, q.QD_PREC_FP64, None))
        L.check(L.lib.qd_eigh_window_dev(n, H.ptr, n, lo, hi, prec, W.ptr, Z.ptr, n, None))
        L.check(L.lib.qd_device_synchronize())
        t = (time.perf_counter() - t0) * 1e3
        st = L.last_timings()
        print("solve %d (%s, N_H = %d): %.1f ms wall; " % (s, a.prec, n, t) +
              ", ".join("%s %.1f" % (k, v) for k, v in zip(STAGES[1:], st[1:7])))
        if os.environ.get("QD_PROFILE", "0") not in ("", "0"):
            pf = L.stage1_profile()
            print("    band reduction steps (ms): " + ", ".join("%s %.1f" % (k, v) for k, v in zip(STEPS, pf)))
    sys.stdout.flush()


if __name__ == "__main__":
    main()
