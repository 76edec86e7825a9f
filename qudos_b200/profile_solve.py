"""Run a few solves of one of the measured decks (qudos_b200.configs:
molecule_15 by default, lens_7, pyramid_11) and print the per-stage times:
the command that the committed ncu summaries under profiles/ were captured
from.

    python -m qudos_b200.profile_solve [--deck molecule_15] [--mg 7] [--prec mixed|fp64] [--solves 1] [--post]
    python -m qudos_b200.profile_solve --gradients-c4

One solve = H assembly (FP64, lower triangle) + the windowed eigensolve on
the device.  With QD_PROFILE=1 in the environment the dense->band reduction
is also broken down into its steps.  --post then runs twice (a first pass
with the one-time costs and a warm one), on the last solve's states, the
stages that follow it in the reference: Coulomb matrix elements (the deck's
CME setting and Coulomb cell), momentum matrix elements,
envelopes on a [001] line scan of 300 points, and the gradients of the
lowest 8 states with respect to the (upper) dot's height and composition.
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


def gradients_c4():
    """The C4 gradient call alone: the 11^3 pyramid deck with 8 + 8 window
    states, one FP64 solve, three warm calls of eigen_gradients_8_band for dot
    height, base width, composition, field, Ep and gamma_1, then one more
    call between cudaProfilerStart and cudaProfilerStop, so that
    `ncu --profile-from-start off` lists the launches of that call only."""
    import torch
    params = [(L.QD_GRAD_LENGTH, 1, 4), (L.QD_GRAD_BASE, 1, 0), (L.QD_GRAD_COMPOSITION, 1, 0),
              (L.QD_GRAD_FIELD, 0, 2), (L.QD_GRAD_EP, 0, 0), (L.QD_GRAD_GAMMA1, 0, 0)]
    with tempfile.TemporaryDirectory() as d:
        configs.write_deck(d, *configs.pyramid_11(mg=5, n_states=4, cme=0))
        pr = q.Problem(d)
        w, v = pr.solve(q.QD_PREC_FP64)
    for rep in range(3):
        t0 = time.perf_counter()
        pr.gradients(v, params)
        print("gradients, warm-up call %d: %.1f ms wall" % (rep, (time.perf_counter() - t0) * 1e3), flush=True)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    t0 = time.perf_counter()
    pr.gradients(v, params)
    print("gradients, listed call: %.1f ms wall" % ((time.perf_counter() - t0) * 1e3), flush=True)
    torch.cuda.cudart().cudaProfilerStop()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mg", type=int, default=7)
    ap.add_argument("--prec", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--solves", type=int, default=1)
    ap.add_argument("--post", action="store_true")
    ap.add_argument("--deck", choices=["molecule_15", "lens_7", "pyramid_11"], default="molecule_15")
    ap.add_argument("--xprod-curve", action="store_true",
                    help="print the X-product kernel's bandwidth per launch of the last solve, binned by m")
    ap.add_argument("--gradients-c4", action="store_true",
                    help="run only the C4 gradient call (profiled region: one warm call)")
    a = ap.parse_args(argv)
    if a.gradients_c4:
        gradients_c4()
        return
    with tempfile.TemporaryDirectory() as d:
        if a.deck == "molecule_15":
            deck = configs.molecule_15(mg=a.mg, cme=4 if a.post else 0)
        elif a.deck == "lens_7":
            deck = configs.lens_7(mg=a.mg)
        else:
            deck = configs.pyramid_11(mg=a.mg, cme=4 if a.post else 1)
        configs.write_deck(d, *deck)
        pr = q.Problem(d)
        pr.build_tables()
    n, lo, hi = pr.n_h, pr.lo, pr.hi
    m = hi - lo + 1
    prec = q.QD_PREC_MIXED if a.prec == "mixed" else q.QD_PREC_FP64
    H = L.DeviceBuffer(n * n * 16)
    Z = L.DeviceBuffer(n * m * 16)
    W = L.DeviceBuffer(m * 8)
    for s in range(a.solves):
        if s == a.solves - 1:  # per-launch timers cover the last solve only
            import ctypes
            cnt, ms_, wk_ = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
            for which in (0, 1):
                L.check(L.lib.qd_tc_kernel_stats(which, ctypes.byref(cnt), ctypes.byref(ms_), ctypes.byref(wk_)))
        t0 = time.perf_counter()
        L.check(L.lib.qd_problem_assemble_dev(pr.handle, H.ptr, n, 0, q.QD_PREC_FP64, None))
        L.check(L.lib.qd_eigh_window_dev(n, H.ptr, n, lo, hi, prec, W.ptr, Z.ptr, n, None))
        L.check(L.lib.qd_device_synchronize())
        t = (time.perf_counter() - t0) * 1e3
        st = L.last_timings()
        print("solve %d (%s %s, N_H = %d): %.1f ms wall; " % (s, a.deck, a.prec, n, t) +
              ", ".join("%s %.1f" % (k, v) for k, v in zip(STAGES[1:], st[1:7])))
        if os.environ.get("QD_PROFILE", "0") not in ("", "0"):
            pf = L.stage1_profile()
            print("    band reduction steps (ms): " + ", ".join("%s %.1f" % (k, v) for k, v in zip(STEPS, pf)))
    if a.xprod_curve and prec == q.QD_PREC_MIXED:
        import ctypes
        import numpy as np
        cap = 4 * n
        ms = np.zeros(cap)
        wk = np.zeros(cap)
        k = L.lib.qd_tc_kernel_launches(0, cap, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        wk.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if k < 0:
            L.check(-k)
        ms, wk = ms[:k], wk[:k]
        mm = np.sqrt(wk / 8.0)
        print("xprod per launch (m bins: launches, total ms, GB/s):")
        edges = [0, 2000, 5000, 10000, 15000, 20000, 25000, 10 ** 9]
        for lo_, hi_ in zip(edges[:-1], edges[1:]):
            sel = (mm >= lo_) & (mm < hi_)
            if sel.any():
                print("  m in [%d, %s): %d, %.1f ms, %.0f GB/s" %
                      (lo_, hi_ if hi_ < 10 ** 9 else "inf", sel.sum(), ms[sel].sum(),
                       wk[sel].sum() / (ms[sel].sum() * 1e-3) / 1e9))
        print("  all: %d, %.1f ms, %.0f GB/s" % (k, ms.sum(), wk.sum() / (ms.sum() * 1e-3) / 1e9))
    if a.post:
        import numpy as np
        w = np.empty(m)
        v = np.empty((n, m), dtype=np.complex128, order="F")
        W.download(w)
        Z.download(v)
        H.free()
        nv, nc = 2 * pr.n_vb, 2 * pr.n_cb
        geo = pr.geometry(pr.n_shape)[0]
        z = np.linspace(-0.5 * geo["L3"], 0.5 * geo["L3"], 300)
        dot, height = {"molecule_15": (2, 3), "lens_7": (1, 3), "pyramid_11": (1, 4)}[a.deck]
        # the first pass includes one-time costs (kernel loading, pool growth); the second is warm
        for rep in ("first", "warm"):
            t0 = time.perf_counter()
            pr.coulomb(v, nv, nc, 1)
            t1 = time.perf_counter()
            pr.momentum(v, nv, nc)
            t2 = time.perf_counter()
            pr.envelopes(v, np.zeros(300), np.zeros(300), z)
            t3 = time.perf_counter()
            pr.gradients(v[:, :8], [(L.QD_GRAD_LENGTH, dot, height), (L.QD_GRAD_COMPOSITION, dot, 0)])
            t4 = time.perf_counter()
            print("post, %s pass (ms wall): coulomb %.1f, momentum %.1f, envelopes %.1f, gradients %.1f" %
                  (rep, (t1 - t0) * 1e3, (t2 - t1) * 1e3, (t3 - t2) * 1e3, (t4 - t3) * 1e3))
    sys.stdout.flush()


if __name__ == "__main__":
    main()
