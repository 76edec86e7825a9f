"""Benchmark of the PWEM solve path: ms per solve (H assembly + 32 eigenpairs
nearest the gap) at 15^3 plane waves (N_H = 27000), mixed precision against
the all-FP64 GPU path, on the two-lens quantum-dot molecule deck
(qudos_b200.configs.molecule_15, synthetic inputs in the reference's format).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference]

One JSON line on stdout (rank 0).  N > 1 runs N independent replicas (the
solve does not shard), launched by torch.distributed.run; times are the max
over ranks.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "ms/solve (assembly+32 eigenpairs, 15^3 PW): mixed vs FP64 GPU at 1 ueV"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.out = None

    def __enter__(self):
        self.out = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.out.name).read().strip().splitlines() if r.strip()]
            sm = [float(r[0]) for r in rows]
            mx = float(rows[0][1])
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[3 + i] and "Not" not in r[3 + i]})
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(sm)}
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_sample(mg=4):
    """Oracle (numpy assembly + LAPACK zheevr from scipy's OpenBLAS, all host threads)
    on the same deck at 9^3 plane waves (N_H = 5832), scaled to N_H = 27000 by N^3."""
    from oracle import eigen, inputs, pipeline
    from qudos_b200 import configs
    with tempfile.TemporaryDirectory() as d:
        configs.write_deck(d, *configs.molecule_15(mg=mg))
        p, geo = inputs.load(d)
        t0 = time.time()
        pr = pipeline.prepare(p, geo)
        t1 = time.time()
        H = pipeline.assemble(pr)
        lo, hi = eigen.index_window(pr.n_pw, p["N_VB"], p["N_CB"])
        eigen.diagonalise(H, lo, hi)
        t2 = time.time()
    n = pr.n_h
    scale = (27000.0 / n) ** 3
    return (t2 - t1) * 1e3 * scale, n, t2 - t1


def run_reference(args, ws, rank):
    if rank != 0:
        return
    cores = os.cpu_count()
    times = []
    for i in range(args.warmup + args.steps):
        ms, n, raw = cpu_sample()
        if i >= args.warmup:
            times.append(ms)
    v = float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ms", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": "molecule_15: two stacked InGaAs lenses, 15^3 PW, N_H=27000, 32 eigenpairs",
                   "sample": "same deck at 9^3 PW (N_H=5832), scaled by (27000/5832)^3"},
        "cpu_baseline": {"value": v, "unit": "ms", "cores": cores, "kind": "port",
                         "sample": "oracle assembly + scipy/OpenBLAS zheevr at N_H=5832, x(27000/5832)^3"},
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# DRAM bytes per launch of xprod_kernel over its algorithmic bytes, from the ncu
# capture summarised in profiles/xprod_kernel_9cubed.md (one launch, m = 5480).
XPROD_TRAFFIC_RATIO = 1.083


def tc_stats(L, which):
    import ctypes as C
    n, ms, work = C.c_longlong(0), C.c_double(0), C.c_double(0)
    L.check(L.lib.qd_tc_kernel_stats(which, C.byref(n), C.byref(ms), C.byref(work)))
    return n.value, ms.value, work.value


def run_gpu(args, ws, rank, local):
    import ctypes as C
    import qudos_b200 as q
    from qudos_b200 import configs, lib as L
    if ws > 1:
        L.check(L.lib.qd_set_device(local))
    hbm_peak, bf16_peak, peak_src = peaks()
    with tempfile.TemporaryDirectory() as d:
        configs.write_deck(d, *configs.molecule_15(mg=args.mg))
        pr = q.Problem(d)
        pr.build_tables()
    n, lo, hi = pr.n_h, pr.lo, pr.hi
    M = hi - lo + 1
    # roofline denominators not in the measured-peak file: cuBLAS TF32 and FP64 GEMM throughput on this GPU
    tf32_peak, fp64_peak = C.c_double(0), C.c_double(0)
    L.check(L.lib.qd_gemm_peak(1, 8192, 10, C.byref(tf32_peak)))
    L.check(L.lib.qd_gemm_peak(0, 8192, 4, C.byref(fp64_peak)))
    tf32_peak, fp64_peak = tf32_peak.value, fp64_peak.value
    H = L.DeviceBuffer(n * n * 16)
    Z = L.DeviceBuffer(n * M * 16)
    W = L.DeviceBuffer(M * 8)
    e0, e1, ea0, ea1 = L.Event(), L.Event(), L.Event(), L.Event()

    def step(prec):
        L.check(L.lib.qd_problem_assemble_dev(pr.handle, H.ptr, n, 0, q.QD_PREC_FP64, None))
        L.check(L.lib.qd_eigh_window_dev(n, H.ptr, n, lo, hi, prec, W.ptr, Z.ptr, n, None))

    # FP64 comparator
    for _ in range(1):
        step(q.QD_PREC_FP64)
    w64 = np.empty(M)
    barrier(ws)
    L.check(L.lib.qd_device_synchronize())
    e0.record()
    for _ in range(args.fp64_steps):
        step(q.QD_PREC_FP64)
    e1.record()
    ms64 = allreduce_max(e0.elapsed_ms(e1) / args.fp64_steps, ws)
    t64 = L.last_timings()
    W.download(w64)
    # mixed path: warm-up, then the timed steps
    for _ in range(args.warmup):
        step(q.QD_PREC_MIXED)
    launches0 = int(L.lib.qd_launch_count())
    tc_stats(L, 0)
    tc_stats(L, 1)  # reset the per-kernel event timers
    barrier(ws)
    L.check(L.lib.qd_device_synchronize())
    with Clocks(local) as clk:
        e0.record()
        for _ in range(args.steps):
            step(q.QD_PREC_MIXED)
        e1.record()
        ms = e0.elapsed_ms(e1) / args.steps
    launches = (int(L.lib.qd_launch_count()) - launches0) // args.steps
    x_n, x_ms, x_bytes = tc_stats(L, 0)
    f_n, f_ms, f_flops = tc_stats(L, 1)
    ms = allreduce_max(ms, ws)
    tmx = L.last_timings()
    wmx = np.empty(M)
    W.download(wmx)
    dE = float(np.abs(wmx - w64).max()) * 1e6
    # assembly kernel alone (HBM roofline): lower triangle, complex128
    ea0.record()
    for _ in range(3):
        L.check(L.lib.qd_problem_assemble_dev(pr.handle, H.ptr, n, 0, q.QD_PREC_FP64, None))
    ea1.record()
    ms_asm = ea0.elapsed_ms(ea1) / 3
    asm_bytes = 16.0 * n * (n + 1) / 2
    # stage-1 reduction (tensor-bound): LAPACK flop count of the dense->band reduction
    flops_stage1 = 16.0 / 3.0 * n ** 3
    st1_ms = tmx[1]
    # e2e through the reference-named C-ABI with host buffers (eigenstates)
    e2e_ms, h2d, d2h = e2e_reference_call(pr, args, L)
    cpu = None
    if rank == 0 and not args.no_cpu:
        cms, cn, raw = cpu_sample()
        cpu = {"value": cms, "unit": "ms", "cores": os.cpu_count(), "kind": "port",
               "sample": "oracle assembly + scipy/OpenBLAS zheevr at N_H=%d (%.1f s), x(27000/%d)^3" % (cn, raw, cn)}
    value = ms  # per replica; every rank solves its own instance
    line = {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "c64+c128",
        "data": "synthetic",
        "config": {"workload": "molecule_15: two stacked InGaAs lenses, 15^3 PW, N_H=27000, 32 eigenpairs",
                   "n_h": n, "eigenpairs": M, "parallelism": "replicas" if ws > 1 else "single",
                   "l2": "inputs larger than L2 (H is %.1f GB)" % (n * n * 16 / 1e9)},
        "fp64_ms_per_solve": ms64, "speedup_vs_fp64": ms64 / ms, "max_dE_ueV_vs_fp64": dE,
        "stages_ms_mixed": {"band_reduction": tmx[1], "bulge_chasing": tmx[2], "bisection": tmx[3],
                            "inverse_iteration": tmx[4], "back_transform": tmx[5], "rayleigh_ritz": tmx[6]},
        "stages_ms_fp64": {"band_reduction": t64[1], "bulge_chasing": t64[2], "bisection": t64[3],
                           "inverse_iteration": t64[4], "back_transform": t64[5]},
        # the largest kernel with a bandwidth or throughput bound (the bulge chasing ahead of it is latency-bound)
        "roofline": {"bound": "hbm", "kernel": "xprod_kernel (X = A22 VT, tcgen05 3xTF32)",
                     "achieved": x_bytes / (x_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                     "frac": x_bytes / (x_ms * 1e-3) / 1e9 / hbm_peak,
                     "traffic": XPROD_TRAFFIC_RATIO * x_bytes / max(x_n, 1),
                     "launches_per_step": x_n / args.steps, "ms_per_step": x_ms / args.steps,
                     "note": "work = 8 m^2 bytes per launch (trailing matrix read once); peak = %s HBM copy; "
                             "traffic = dram bytes per launch scaled from one ncu capture" % peak_src},
        "roofline_flush": {"bound": "tensor", "kernel": "flush_kernel (Hermitian rank-2K update, tcgen05 3xTF32)",
                           "achieved": f_flops / (f_ms * 1e-3) / 1e12, "peak": tf32_peak / 3.0, "unit": "TFLOP/s",
                           "frac": f_flops / (f_ms * 1e-3) / 1e12 / (tf32_peak / 3.0), "traffic": None,
                           "issued_tf32_tflops": 3.0 * f_flops / (f_ms * 1e-3) / 1e12,
                           "launches_per_step": f_n / args.steps, "ms_per_step": f_ms / args.steps,
                           "note": "work = 8 mt (mt+1) K flops per launch; peak = measured cuBLAS TF32 GEMM / 3 "
                                   "(three TF32 products per FP32-accurate product)"},
        "reduction_fp64_vs_peak": {"achieved": flops_stage1 / (t64[1] * 1e-3) / 1e12, "peak": fp64_peak,
                                   "unit": "TFLOP/s", "frac": flops_stage1 / (t64[1] * 1e-3) / 1e12 / fp64_peak,
                                   "note": "FP64 dense->band reduction, 16/3 N^3 flop; peak = measured cuBLAS DGEMM"},
        "measured_gemm_peaks_tflops": {"tf32": tf32_peak, "fp64": fp64_peak, "bf16": bf16_peak},
        "roofline_assembly": {"bound": "hbm", "achieved": asm_bytes / (ms_asm * 1e-3) / 1e9, "peak": hbm_peak,
                              "unit": "GB/s", "frac": asm_bytes / (ms_asm * 1e-3) / 1e9 / hbm_peak,
                              "traffic": None, "ms": ms_asm},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def e2e_reference_call(pr, args, L):
    """eigenstates() (the reference's routine) with the tables in host memory,
    H assembled on the device, eigenvectors copied back: timed on the host."""
    import ctypes as C
    from qudos_b200 import pwem
    os.environ["QD_PRECISION"] = "mixed"
    ns = pr.n_shape
    shp = None
    geo = pr.geometry(ns)
    mat = pr.materials(ns)
    n_pw = pr.n_pw
    N = round(n_pw ** (1.0 / 3.0))
    NT = 2 * N - 1
    shp = (NT, NT, NT)
    nT = NT ** 3
    chi = [None] + [pr.table(0, s, 0, shp) for s in range(1, ns)]
    eps = [pr.table(1, c, 0, shp) for c in range(6)]
    phi = pr.table(2, 0, 0, shp)
    conv = [None] + [[pr.table(3, s, c, shp) for c in range(8)] for s in range(1, ns)]
    keep = []

    class CF(C.Structure):
        _fields_ = [("chi", C.c_void_p)]

    class ST(C.Structure):
        _fields_ = [(k, C.c_void_p) for k in ("xx", "yy", "zz", "yz", "xz", "xy")]

    class CV(C.Structure):
        _fields_ = [(k, C.c_void_p) for k in ("char_xx", "char_yy", "char_zz", "char_yz", "char_xz", "char_xy",
                                              "char_hydrostatic", "char_biaxial")] + [("rest%d" % i, C.c_void_p)
                                                                                       for i in range(24)]
    cf = (CF * ns)()
    for s in range(1, ns):
        cf[s].chi = chi[s].ctypes.data
    cv = (CV * ns)()
    for s in range(1, ns):
        for c, k in enumerate(("char_xx", "char_yy", "char_zz", "char_yz", "char_xz", "char_xy", "char_hydrostatic",
                               "char_biaxial")):
            setattr(cv[s], k, conv[s][c].ctypes.data)
    st = ST(*[e.ctypes.data for e in eps])
    C.c_void_p.in_dll(L.lib, "characteristic_function_G").value = C.addressof(cf)
    C.c_void_p.in_dll(L.lib, "convolutions_char_strain").value = C.addressof(cv)
    C.memmove(C.addressof(ST.in_dll(L.lib, "strain_G")), C.addressof(st), C.sizeof(ST))
    C.c_void_p.in_dll(L.lib, "phi_piezo_G").value = phi.ctypes.data
    C.c_int.in_dll(L.lib, "include_strain").value = 1
    C.c_int.in_dll(L.lib, "include_piezo").value = 1
    C.c_int64.in_dll(L.lib, "N_H").value = pr.n_h
    C.c_int64.in_dll(L.lib, "na_rows").value = pr.n_h
    grids = [np.ascontiguousarray(((2 * np.pi) / L_) * (0.5 * (1.0 - NT) + np.arange(NT))) for L_ in
             (geo[0]["L1"], geo[0]["L2"], geo[0]["L3"])]
    basis = L.WaveVectors(N, N, N, NT, NT, NT, *[g.ctypes.data_as(C.POINTER(C.c_double)) for g in grids], 0.0, 0.0,
                          0.0)
    gstruct = (L.SupercellGeometry * ns)(*[L.SupercellGeometry(**g) for g in geo])
    mstruct = (L.MaterialParams * ns)(*[L.MaterialParams(**m) for m in mat])
    nstates = (C.c_int * 2)(pr.n_vb, pr.n_cb)
    vb = (L.Eigenstate * (2 * pr.n_vb))()
    cb = (L.Eigenstate * (2 * pr.n_cb))()
    bufs = [np.zeros(pr.n_h, dtype=np.complex128) for _ in range(2 * pr.n_vb + 2 * pr.n_cb)]
    for i in range(2 * pr.n_vb):
        vb[i].fourier = bufs[i].ctypes.data
    for i in range(2 * pr.n_cb):
        cb[i].fourier = bufs[2 * pr.n_vb + i].ctypes.data
    F = L.Vector(0.0, 0.0, 0.0)
    times = []
    for i in range(2):
        t0 = time.perf_counter()
        L.lib.eigenstates(ns, nstates, F, basis, gstruct, mstruct, vb, cb)
        times.append(time.perf_counter() - t0)
    h2d = 16 * nT * ((ns - 1) + 6 + 1 + 8 * (ns - 1))
    d2h = 16 * pr.n_h * len(bufs) + 8 * len(bufs)
    keep.append((cf, cv, st, grids, bufs))
    return times[-1] * 1e3, h2d, d2h


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--mg", type=int, default=7)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    ws, rank, local = dist_setup()
    if args.impl == "gpu":
        import qudos_b200  # noqa: F401  (before torch: the toolkit cuBLAS must be the one loaded)
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_gpu(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
