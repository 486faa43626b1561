#!/usr/bin/env python
"""Benchmark of the spectrum-slicing hot path on B200.

Workload (default, "lap3d-slice"): one polynomial-filtered Lanczos slice solve
(ChebLanNr, FP64, tol 1e-8) on the 3-D 7-point Dirichlet Laplacian 100^3
(n = 1,000,000, nnz = 6,940,000, spectrum bounds [0, 12]) -- the config-2
matrix -- over an interval that holds 100 eigenvalues just above 0.6, with
both end points at midpoints of gaps of the analytic spectrum (the
serving-size slice request of the mixed request stream).  The filter is
designed by find_pol with damping 2, thresholds 0.8 / 0.2, max degree 3000.
One step = one complete slice solve; every step checks the eigenvalue count
against the analytic spectrum and the residuals against tol.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (launched by torch.distributed.run): every rank solves its own slice of
the same matrix (independent units, no data-path collective, weak scaling);
rank 0 prints the aggregate.  --impl reference times the reference EVSL CPU
build (oracle/_ref) on the same request with all host threads.
"""
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

NX = NY = NZ = 100
LMIN, LMAX = 0.0, 12.0
COUNT = 100
TOL = 1e-8
MAXIT = 2000
SEED = 1234
METRIC = "eigenpairs/sec + p50/p99 slice latency at resid<=1e-8; filter SpMV GB/s vs HBM"
UNIT = "eigenpairs/s"
# Random sparse SPD matrix of the mixed-precision configuration: 2,000,000
# rows, 16 seeded off-diagonal columns per row, symmetrised (~66M nonzeros).
RSPD_N = 2_000_000
RSPD_SEED = 3
# Lanczos dimension of this request, as the GPU arm measures it (used only to
# scale the CPU sample to a whole request; the recurrence is the same).
REQUEST_LANCZOS_STEPS = 451


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--count", type=int, default=COUNT)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", choices=["lap3d-slice", "lap3d-filter", "lap3d-batch", "serve", "lap3d-multifilter",
                                          "lap3d-reorth", "lap3d-kpm", "rspd-filter", "dgemm", "batch-uneven", "rspd-kpm",
                                          "block-cgs", "lap3d-pipeline"],
                   default="lap3d-slice",
                   help="lap3d-filter: only the filter p(A)v of the same request (kernel micro-benchmark); "
                        "lap3d-batch: several slices through the request engine; serve: a Poisson request stream")
    p.add_argument("--slices", type=int, default=4, help="lap3d-batch: slices solved together")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="mixed",
                   help="lap3d-batch / serve: filter precision of the engine")
    p.add_argument("--rate", type=float, default=2.0, help="serve: mean arrivals per second")
    p.add_argument("--duration", type=float, default=20.0, help="serve: seconds of arrivals")
    p.add_argument("--slots", type=int, default=16, help="serve: slice solves in flight")
    p.add_argument("--budget-gb", type=float, default=150.0, help="serve: HBM budget of the engine")
    p.add_argument("--max-count", type=int, default=150, help="serve: most eigenvalues in a slice request")
    p.add_argument("--compare-sequential", action="store_true",
                   help="lap3d-batch: also time ChebLanNr on the same slices one after another")
    p.add_argument("--serve-mix", choices=["default", "small"], default="default",
                   help="serve: 'small' draws the large-matrix requests on the 2-D 100x100 Laplacian only")
    p.add_argument("--rspd-n", type=int, default=RSPD_N, help="rspd-filter: rows of the random SPD matrix")
    p.add_argument("--dgemm-kernel", type=int, choices=[-1, 0, 1, 2], default=-1,
                   help="dgemm, block-cgs: 0 the 64x64 kernel, 1 the 128x128 DFMA kernel, 2 the mma.sync f64 kernel "
                        "(-1: library default)")
    p.add_argument("--grid", type=int, default=50,
                   help="lap3d-pipeline: the 3-D Laplacian's grid points per side")
    p.add_argument("--kpm-prefetch", type=int, choices=[-1, 0, 1], default=-1,
                   help="lap3d-kpm / rspd-kpm: the KPM step's own-row prefetch form (-1: library default)")
    p.add_argument("--kpm-split", type=int, choices=[-1, 0, 1], default=-1,
                   help="rspd-kpm: KPM block step on the column-split copy: -1 automatic, 0 off, 1 on")
    p.add_argument("--split-range-mb", type=float, default=0.0,
                   help="rspd-filter / rspd-kpm: MiB of block rows one column range of the column-split copy "
                        "gathers from (0: the library default)")
    p.add_argument("--rspd-ncols", default="1",
                   help="rspd-filter: columns filtered together (> 1: the multi-column block filter, "
                        "FP64 or FP32 by --precision); a comma-separated list prints one line per width")
    p.add_argument("--sigma", type=int, default=-1,
                   help="rspd-filter: SELL-C-sigma sort window (-1 automatic, 0 unsorted SELL-32)")
    p.add_argument("--instances", type=int, default=128, help="batch-uneven: independent Laplacians")
    p.add_argument("--batch-persistent", type=int, choices=[0, 1], default=0,
                   help="batch-uneven: the batched filter as one persistent launch (1) or one launch per degree (0)")
    p.add_argument("--gemm", default="1000000,1000,256",
                   help="dgemm: n,K,m of the Ritz product V(n x K) Y(K x m)")
    p.add_argument("--ncols", type=int, default=16, help="lap3d-multifilter: columns")
    p.add_argument("--variant", type=int, default=-1, help="lap3d-multifilter: kernel variant (-1 autotuned)")
    p.add_argument("--sweep", action="store_true", help="lap3d-multifilter: every variant/width/precision once")
    p.add_argument("--low-degree", action="store_true", help="lap3d-multifilter: only the degree-7 filter")
    p.add_argument("--l2-resident", action="store_true",
                   help="keep the stored matrix persisting in L2 (comparison runs)")
    p.add_argument("--maxit-reorth", type=int, default=600, help="lap3d-reorth: Lanczos steps")
    p.add_argument("--kpm-probes", type=int, default=30, help="lap3d-kpm: probe vectors")
    p.add_argument("--kpm-moments", type=int, default=300, help="lap3d-kpm: Chebyshev moments")
    p.add_argument("--kpm-direct", action="store_true",
                   help="lap3d-kpm: one dot with the probe per degree instead of the product identities")
    p.add_argument("--filter-mode", choices=["per-degree", "wave"], default="per-degree",
                   help="filter execution: one launch per degree or one pipelined launch")
    p.add_argument("--row-patterns", choices=["on", "off"], default="on",
                   help="row-pattern dictionary of the stored matrix (on: used when the rows allow it)")
    p.add_argument("--filter-kernel", default="auto",
                   help="single-vector FP64 filter kernel: auto (timed choice per matrix) or one of "
                        "sell-loop, sell-unrolled, pattern-global-unrolled, pattern-global-loop, "
                        "pattern-constant-loop, pattern-constant-unrolled, pattern-constant-rowdesc (profiling runs)")
    return p.parse_args()


def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def slice_interval(ev, rank, count):
    from evsl_b200 import workloads as W

    lo = 0.6 + 0.01 * rank  # every rank gets its own slice
    a, b, cnt = W.gap_interval(ev, lo, count)
    return [a, b, LMIN, LMAX], cnt


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, maxs, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                maxs = max(maxs, float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sms:
            return None
        loaded = [s for s in sms if s > 0.5 * maxs] or sms
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": maxs, "reasons": sorted(reasons),
                "samples": len(sms)}


def sm_count():
    try:
        import torch

        return torch.cuda.get_device_properties(0).multi_processor_count
    except Exception:
        return 148


def measured_peak_hbm():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel, workload="lap3d-slice"):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 3 and not line.startswith("#") and f[0] == workload and f[1] == kernel:
            return float(f[2])
    return None


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    import evsl_b200
    from evsl_b200 import workloads as W

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    lib = evsl_b200.Library()
    if args.l2_resident:
        lib.set_l2_resident(True)
    lib.set_filter_wave(args.filter_mode == "wave")
    lib.set_row_patterns(args.row_patterns == "on")
    lib.set_filter_kernel(None if args.filter_kernel == "auto" else args.filter_kernel)
    ia, ja, a = W.laplacian_csr(NX, NY, NZ)
    ev = W.laplacian_eigenvalues(NX, NY, NZ)
    lib.set_csr(ia, ja, a)
    intv, expected = slice_interval(ev, rank, args.count)
    exact = ev[(ev >= intv[0]) & (ev <= intv[1])]
    pol = lib.find_pol(intv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    rng = np.random.default_rng(SEED + rank)
    v0 = rng.standard_normal(NX * NY * NZ)
    v0 /= np.linalg.norm(v0)
    dv = evsl_b200.DeviceBuffer.from_host(lib.lib, v0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    lstream = torch.cuda.ExternalStream(lib.stream_handle())
    import ctypes as C

    def solve_device():
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        nev = C.c_int()
        lam, res = C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
        Wp = C.c_void_p()
        rc = lib.lib.ChebLanNr(iv.ctypes.data_as(C.POINTER(C.c_double)), MAXIT, TOL, dv.ptr, C.byref(pol),
                               C.byref(nev), C.byref(lam), C.byref(Wp), C.byref(res), None)
        if rc != 0:
            raise RuntimeError(f"ChebLanNr returned {rc}: {lib.last_error()}")
        m = nev.value
        lam_h = np.ctypeslib.as_array(lam, (m,)).copy() if m else np.zeros(0)
        res_h = np.ctypeslib.as_array(res, (m,)).copy() if m else np.zeros(0)
        lib.lib._evsl_Free(C.cast(lam, C.c_void_p))
        lib.lib._evsl_Free(C.cast(res, C.c_void_p))
        return lam_h, res_h, Wp.value

    def check(lam, res):
        ok = len(lam) == len(exact)
        err = float(np.max(np.abs(np.sort(lam) - exact))) if ok and len(lam) else float("inf")
        return {"count": int(len(lam)), "exact": int(len(exact)), "max_res": float(np.max(res)) if len(res) else 0.0,
                "max_err": err, "ok": bool(ok and err <= 1e-10 * (LMAX - LMIN) and (len(res) == 0 or res.max() < TOL))}

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up
    for _ in range(args.warmup):
        lam, res, Wp = solve_device()
        lib.lib._evsl_Free_device(Wp)
    kdim, cand = lib.last_solve_info()
    # timed region: device-resident inputs
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    lib.filter_profile(True)
    launches0 = lib.launch_count()
    ev_start = torch.cuda.Event(enable_timing=True)
    ev_end = torch.cuda.Event(enable_timing=True)
    lat = []
    found = 0
    checks = []
    ev_start.record(lstream)
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        lam, res, Wp = solve_device()
        e1.record(lstream)
        e1.synchronize()
        lat.append(e0.elapsed_time(e1))
        lib.lib._evsl_Free_device(Wp)
        found += len(lam)
        checks.append(check(lam, res))
    ev_end.record(lstream)
    ev_end.synchronize()
    launches = lib.launch_count() - launches0
    f_sec, f_bytes, f_launch, f_calls = lib.filter_stats()
    lib.filter_profile(False)
    clocks = sampler.stop()
    t_dev = sum(lat) / 1e3  # seconds of device time in the solves (flushes excluded)
    barrier()

    # e2e through the C ABI with host buffers: vinit H2D and eigenpairs D2H each step
    pinned_in = torch.from_numpy(v0).pin_memory()
    pinned_out = torch.empty((len(exact) + 16, NX * NY * NZ), dtype=torch.float64).pin_memory()
    e2e_times, e2e_found, h2d, d2h = [], 0, 0, 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lib.lib.evsl_memcpy_host_to_device(dv.ptr, pinned_in.data_ptr(), v0.nbytes)
        lam, res, Wp = solve_device()
        m = len(lam)
        if m and m <= pinned_out.shape[0]:
            lib.lib.evsl_memcpy_device_to_host(pinned_out.data_ptr(), Wp, m * NX * NY * NZ * 8)
        lib.lib._evsl_Free_device(Wp)
        e2e_times.append(time.perf_counter() - t0)
        e2e_found += m
        h2d = v0.nbytes
        d2h = m * NX * NY * NZ * 8 + 2 * m * 8

    # the slice matrix's storage and filter kernel, read before config 1 replaces the matrix
    storage = storage_desc(lib)
    v_chosen, _ = lib.filter_kernel()
    kname = lib.FILTER_KERNELS[v_chosen] if v_chosen >= 0 else "sell-loop"
    config1 = run_config1_ours(lib, lstream) if world == 1 else None

    # aggregate over ranks
    stats = torch.tensor([t_dev, float(found), sum(e2e_times), float(e2e_found)], dtype=torch.float64,
                         device="cuda")
    if dist is not None:
        tmax = stats.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        tsum = stats.clone()
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        t_all, found_all, e2e_t, e2e_f = tmax[0].item(), tsum[1].item(), tmax[2].item(), tsum[3].item()
    else:
        t_all, found_all, e2e_t, e2e_f = t_dev, float(found), sum(e2e_times), float(e2e_found)

    result = None
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        achieved = f_bytes / f_sec / 1e9 if f_sec > 0 else 0.0
        traffic = profiled_traffic("k_cheb:" + kname)
        avg_launch = f_sec / f_launch if f_launch else None
        result = {
            "metric": METRIC,
            "value": found_all / t_all,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": 1e3 * t_all / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (3-D Dirichlet Laplacian, seeded start vector)",
            "config": {
                "workload": "lap3d-slice: ChebLanNr FP64 tol 1e-8 on the 3-D 7-point Laplacian 100^3 "
                            "(n=1e6, nnz=6.94e6, bounds [0,12]), one slice of %d eigenvalues above 0.6 per rank "
                            "(end points at spectral gap midpoints), find_pol damping 2, thresholds 0.8/0.2, "
                            "max_deg 3000, maxit %d" % (args.count, MAXIT),
                "interval": intv[:2],
                "filter_degree": int(pol.deg),
                "lanczos_steps": int(kdim),
                "parallelism": f"replicas x{world} (independent slices)",
                "l2": "256 MB buffer written between steps; per-step working set (A + basis) > L2",
                "storage": storage,
            },
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "per_step": lat},
            "check": checks[-1],
            "all_steps_ok": all(c["ok"] for c in checks),
            "roofline": {
                "kernel": "k_cheb (fused FP64 SpMV + Chebyshev step; storage and variant in config.storage)",
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "peak_kind": peak_kind,
                "unit": "GB/s",
                "frac": achieved / peak if peak else None,
                "frac_algorithmic": achieved / peak if peak else None,
                "frac_dram": (traffic / avg_launch / 1e9 / peak) if (traffic and avg_launch and peak) else None,
                "frac_note": "frac = frac_algorithmic: the formula's bytes (12 B per stored entry + vectors) over the "
                             "kernel time; the row-pattern dictionary stores 2-byte ids and the per-degree working set "
                             "stays in L2, so it exceeds 1; frac_dram = the DRAM bytes ncu measured per launch of this "
                             "kernel variant (cold caches) over the same time",
                "traffic": traffic,
                "traffic_kernel": "k_cheb:" + kname,
                "algorithmic_bytes_per_launch": f_bytes / f_launch if f_launch else None,
                "avg_launch_us": 1e6 * f_sec / f_launch if f_launch else None,
                "launches": f_launch,
                "share_of_step": f_sec / t_dev if t_dev else None,
            },
            "e2e": {"value": e2e_f / e2e_t if e2e_t else None, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if config1 is not None:
            result["config1"] = config1
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(pol.deg, kdim, intv, found / args.steps, v0, nthreads=1)
    lib.free_pol(pol)
    dv.free()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


# ---------------------------------------------------------------------------
# config 1, run to completion by both arms: ChebLanNr over [0.6, 0.9] of the
# 2-D Laplacian 100x100 (260 eigenpairs), find_pol damping 2, thresholds
# 0.8 / 0.2, tol 1e-8, maxit 2000, seeded normal start vector
# ---------------------------------------------------------------------------
C1_DIMS = (100, 100, 1)
C1_INTV = [0.6, 0.9, 0.0, 8.0]
C1_SEED = 1234
C1_STEPS = 3


def run_config1_ours(lib, lstream):
    """Config 1 on the GPU through ChebLanNr (the drop-in entry point):
    device time of each complete solve (CUDA events on the library stream),
    eigenpairs/s = 260 / median solve time; e2e adds the start vector's copy
    in and the eigenvectors' copy out."""
    import ctypes as C

    import torch

    from evsl_b200 import workloads as W

    ia, ja, a = W.laplacian_csr(*C1_DIMS)
    ev = W.laplacian_eigenvalues(*C1_DIMS)
    exact = ev[(ev >= C1_INTV[0]) & (ev <= C1_INTV[1])]
    lib.set_csr(ia, ja, a)
    pol = lib.find_pol(C1_INTV, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    v = np.random.default_rng(C1_SEED).standard_normal(len(ia) - 1)
    v /= np.linalg.norm(v)
    out = {"workload": "config 1: ChebLanNr FP64 over [0.6, 0.9] of the 2-D Laplacian 100x100, tol 1e-8, "
                       "maxit 2000, complete solve per step", "steps": C1_STEPS, "filter_degree": int(pol.deg)}
    times, e2e, oks = [], [], []
    for i in range(1 + C1_STEPS):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        lam, Y, res = lib.cheblan_nr(C1_INTV, 2000, TOL, v, pol, want_vectors=True)
        e1.record(lstream)
        e1.synchronize()
        t1 = time.perf_counter()
        if i == 0:
            continue  # warm-up (kernel choice by timing, workspace)
        times.append(e0.elapsed_time(e1) / 1e3)
        e2e.append(t1 - t0)
        lam = np.sort(lam)
        ok = len(lam) == len(exact) and np.max(np.abs(lam - exact)) <= 1e-10 * 8.0 and np.all(res < TOL)
        oks.append(bool(ok))
    lib.free_pol(pol)
    t = statistics.median(times)
    out.update({"value": len(exact) / t, "unit": UNIT, "ms_per_step": 1e3 * t, "eigenpairs": int(len(exact)),
                "e2e": {"value": len(exact) / statistics.median(e2e), "unit": UNIT,
                        "h2d_bytes_per_step": int(v.nbytes), "d2h_bytes_per_step": int(len(exact) * (v.nbytes + 16))},
                "all_steps_ok": all(oks), "timing": "device time per complete solve (CUDA events), median"})
    return out


def run_config1_reference(nthreads):
    """Config 1 by the reference CPU build, to completion, with all host
    threads in the reference's own parallel pattern (TESTS/PLanR/
    MMPLanR_omp.c:183-241: the interval cut into slices, one ChebLanNr per
    slice per OpenMP thread).  Slices hold about equal numbers of
    eigenvalues, with end points at gap midpoints of the analytic spectrum
    (at least 10 eigenvalues per slice)."""
    from evsl_b200 import workloads as W
    from oracle import evsl_oracle as O

    R = O.RefLib()
    ia, ja, a = R.lap_csr(*C1_DIMS)
    R.set_csr(ia, ja, a)
    ev = W.laplacian_eigenvalues(*C1_DIMS)
    inside = ev[(ev >= C1_INTV[0]) & (ev <= C1_INTV[1])]
    ns = max(1, min(nthreads, len(inside) // 10))
    cuts = [C1_INTV[0]]
    for k in range(1, ns):
        i = round(k * len(inside) / ns)
        while i < len(inside) and inside[i] - inside[i - 1] < 1e-10:
            i += 1
        cuts.append(0.5 * (inside[i - 1] + inside[i]))
    cuts.append(C1_INTV[1])
    v = np.random.default_rng(C1_SEED).standard_normal(len(ia) - 1)
    v /= np.linalg.norm(v)
    r = R.slices_nr(np.array(cuts), C1_INTV[2], C1_INTV[3], 2000, TOL, v, damping=2, thresh_int=0.8,
                    thresh_ext=0.2, max_deg=3000, nthreads=nthreads)
    lam = np.sort(np.concatenate(r["evals"]))
    ok = len(lam) == len(inside) and np.max(np.abs(lam - inside)) <= 1e-10 * 8.0
    return {"workload": "config 1: ChebLanNr over [0.6, 0.9] of the 2-D Laplacian 100x100, tol 1e-8, complete "
                        "solve", "value": len(lam) / r["wall"], "unit": UNIT, "wall_s": r["wall"],
            "eigenpairs": int(len(lam)), "exact": int(len(inside)), "ok": bool(ok), "threads": nthreads,
            "slices": ns, "slice_degrees": [int(d) for d in r["deg"]],
            "sample": "one complete run (measured, not extrapolated): %d slices on %d OpenMP threads" % (ns, nthreads)}


# ---------------------------------------------------------------------------
# reference CPU build (oracle/_ref): the CPU baseline and the reference arm
# ---------------------------------------------------------------------------
SAMPLE_DEG = 96


def _ref_setup():
    from oracle import evsl_oracle as O

    R = O.RefLib()
    ia, ja, a = R.lap_csr(NX, NY, NZ)  # the reference's own generator
    R.set_csr(ia, ja, a)
    return R, (ia, ja, a)


def cpu_baseline(deg, kdim, intv, pairs_per_request, v0, nthreads=1):
    """Reference ChebAv on the same matrix and filter, truncated to SAMPLE_DEG
    degrees, run by `nthreads` concurrent threads; scaled to the request:
    request time = (kdim + 1) filter applications of degree `deg` (the
    filter is >97% of a request's cost at this size)."""
    try:
        R, keep = _ref_setup()
    except Exception as e:
        return {"value": None, "unit": UNIT, "cores": nthreads, "kind": "reference", "sample": f"unavailable: {e}"}
    rc, rpol = R.find_pol(intv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    wall = R.chebav_multi(rpol, SAMPLE_DEG, v0, nthreads)
    per_degree = wall / SAMPLE_DEG  # per thread
    request_s = (kdim + 1) * rpol.deg * per_degree
    R.free_pol(rpol)
    return {"value": nthreads * pairs_per_request / request_s, "unit": UNIT, "cores": nthreads, "kind": "reference",
            "extrapolated": True,
            "sample": f"{nthreads} thread(s) x reference ChebAv truncated to {SAMPLE_DEG} of {deg} degrees on the "
                      f"same matrix and filter ({wall:.2f} s); request = ({kdim}+1) x degree-{deg} filter "
                      f"applications, extrapolated"}


def run_reference(args):
    rank, world, local = rank_info()
    if rank != 0:
        return
    from evsl_b200 import workloads as W

    nthreads = os.cpu_count() or 1
    ev = W.laplacian_eigenvalues(NX, NY, NZ)
    intv, expected = slice_interval(ev, 0, args.count)
    try:
        R, keep = _ref_setup()
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference build missing: {e}"}))
        return
    rc, rpol = R.find_pol(intv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    rng = np.random.default_rng(SEED)
    v0 = rng.standard_normal(NX * NY * NZ)
    v0 /= np.linalg.norm(v0)
    kdim = REQUEST_LANCZOS_STEPS or int(os.environ.get("EVSL_BENCH_KDIM", "0")) or 330
    for _ in range(args.warmup):
        R.chebav_multi(rpol, SAMPLE_DEG, v0, nthreads)
    walls = [R.chebav_multi(rpol, SAMPLE_DEG, v0, nthreads) for _ in range(args.steps)]
    per_degree = statistics.median(walls) / SAMPLE_DEG
    request_s = (kdim + 1) * rpol.deg * per_degree
    value = nthreads * expected / request_s
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * request_s,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (3-D Dirichlet Laplacian, seeded start vector)",
        "config": {"workload": "lap3d-slice (same request as the GPU arm)", "interval": intv[:2],
                   "filter_degree": int(rpol.deg), "lanczos_steps": kdim,
                   "parallelism": f"{nthreads} concurrent requests (one per host thread)"},
        "extrapolated": True,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "reference", "extrapolated": True,
                         "sample": f"{nthreads} threads x reference ChebAv truncated to {SAMPLE_DEG} of "
                                   f"{rpol.deg} degrees per step; request = ({kdim}+1) filter applications"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    R.free_pol(rpol)
    try:
        out["config1"] = run_config1_reference(nthreads)
    except Exception as e:  # the main line stands without it
        out["config1"] = {"unavailable": str(e)}
    print(json.dumps(out))


def storage_desc(lib):
    """How the registered matrix is stored for the FP64 filter, and which
    single-vector filter kernel the timing-based selection chose."""
    npat = lib.row_pattern_count()
    vb, ib = lib.matrix_storage()
    desc = "SELL-32: %d-byte values, %d-byte column indices" % (vb, ib)
    if npat:
        desc += "; row-pattern dictionary: %d patterns, 2-byte pattern id per row" % npat
    v, us = lib.filter_kernel()
    return {"matrix": desc, "filter_kernel": lib.FILTER_KERNELS[v] if v >= 0 else None,
            "filter_grid_blocks": lib.filter_kernel_grid() or "one row per thread",
            "us_per_degree_step_by_kernel": {k: round(t, 3) for k, t in us.items()}}


def run_filter(args):
    """The dominant kernel alone: W + K applications of the request's filter
    p(A)v (ChebAv, degree ~1440) on the 3-D Laplacian 100^3."""
    import ctypes as C

    import torch

    import evsl_b200
    from evsl_b200 import workloads as W

    lib = evsl_b200.Library()
    if args.l2_resident:
        lib.set_l2_resident(True)
    lib.set_filter_wave(args.filter_mode == "wave")
    lib.set_row_patterns(args.row_patterns == "on")
    lib.set_filter_kernel(None if args.filter_kernel == "auto" else args.filter_kernel)
    ia, ja, a = W.laplacian_csr(NX, NY, NZ)
    ev = W.laplacian_eigenvalues(NX, NY, NZ)
    lib.set_csr(ia, ja, a)
    intv, _ = slice_interval(ev, 0, args.count)
    pol = lib.find_pol(intv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    n = NX * NY * NZ
    v0 = np.random.default_rng(SEED).standard_normal(n)
    dv = evsl_b200.DeviceBuffer.from_host(lib.lib, v0)
    dy = evsl_b200.DeviceBuffer(lib.lib, 8 * n)
    dw = evsl_b200.DeviceBuffer(lib.lib, 24 * n)
    for _ in range(args.warmup):
        lib._check(lib.lib.ChebAv(C.byref(pol), dv.ptr, dy.ptr, dw.ptr), "ChebAv")
    lib.filter_profile(True)
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    for _ in range(args.steps):
        lib._check(lib.lib.ChebAv(C.byref(pol), dv.ptr, dy.ptr, dw.ptr), "ChebAv")
    sec, byt, launches, calls = lib.filter_stats()
    clocks = sampler.stop()
    peak, kind = measured_peak_hbm()
    gbs = byt / sec / 1e9
    print(json.dumps({"metric": "filter SpMV GB/s", "value": gbs, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": "lap3d-filter: ChebAv degree %d on the 3-D Laplacian 100^3" % pol.deg,
                                 "storage": storage_desc(lib)},
                      "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "peak_kind": kind, "unit": "GB/s",
                                   "frac": gbs / peak, "traffic": profiled_traffic("k_cheb", "lap3d-filter"),
                                   "avg_launch_us": 1e6 * sec / launches},
                      "gpu_launches": launches, "clocks": clocks}))
    lib.free_pol(pol)


def run_rspd_filter(args):
    """rspd-filter: the filter kernel alone on the random sparse SPD matrix of
    the mixed-precision configuration (n = 2,000,000, 16 seeded off-diagonal
    columns per row, symmetrised: ~66M nonzeros of unequal row lengths, no
    stencil structure, far larger than L2), stored as SELL-C-sigma.

    --precision mixed: the FP32 filter (values and recurrence in float, FMA
    accumulation; the multi-column kernel with one column).  Per-degree
    device time = (time of a degree-400 filter - time of a degree-40 filter)
    / 360, CUDA events on the library stream around evslx_chebav_multi on
    device-resident vectors, median of K steps.
    --precision fp64: ChebAv (the drop-in FP64 single-vector filter),
    device time of every filter application from CUDA events, averaged over
    its degree launches.

    --rspd-ncols B > 1: the block filter (evslx_chebav_multi with B columns,
    each with the same degree-400 polynomial; FP64 or FP32 by --precision),
    per-degree time from the same degree-400 minus degree-40 difference.

    Algorithmic bytes per degree (the SpMV + Chebyshev update, no padding,
    no chunk tables, no gathers counted): nnz (s_v + 4) + 4 (n + 1) + 5 B n s_x
    with s_v = s_x = 4 (FP32) or 8 (FP64)."""
    import ctypes as C

    import torch

    import evsl_b200 as E
    from evsl_b200 import workloads as W

    n = args.rspd_n
    t0 = time.time()
    ia, ja, a = W.random_spd_csr(n, 16, RSPD_SEED)
    glo, ghi = W.gershgorin_bounds(ia, ja, a)
    gen_s = time.time() - t0
    nnz = int(ia[-1])
    lib = E.Library()
    lib.set_sell_sigma(args.sigma)
    lib.set_filter_kernel(None if args.filter_kernel == "auto" else args.filter_kernel)
    lib.set_filter_variant(args.variant)
    lib.set_split_range_bytes(int(args.split_range_mb * (1 << 20)))
    lib.set_csr(ia, ja, a)
    del ja, a
    sigma, stored, stored_plain = lib.matrix_sell_layout()
    iv = [glo + 0.3 * (ghi - glo), glo + 0.32 * (ghi - glo), glo, ghi]
    for B in [max(1, int(b)) for b in str(args.rspd_ncols).split(",")]:
        _rspd_filter_width(args, lib, B, n, nnz, iv, (sigma, stored, stored_plain), gen_s, glo, ghi)


def _rspd_filter_width(args, lib, B, n, nnz, iv, layout, gen_s, glo, ghi):
    """One rspd-filter line: the filter of B columns on the registered matrix."""
    import ctypes as C

    import torch

    import evsl_b200 as E

    sigma, stored, stored_plain = layout
    fp32 = args.precision == "mixed"
    sx = 4 if fp32 else 8
    abytes = nnz * (sx + 4) + 4.0 * (n + 1) + 5.0 * B * n * sx
    v0 = np.random.default_rng(RSPD_SEED).standard_normal((B, n))
    dv = E.DeviceBuffer.from_host(lib.lib, v0)
    dy = E.DeviceBuffer(lib.lib, 8 * n * B)
    lstream = torch.cuda.ExternalStream(lib.stream_handle())
    sampler = ClockSampler(rank_info()[2])
    if fp32 or B > 1:
        p_hi = lib.find_pol(iv, deg=400)
        p_lo = lib.find_pol(iv, deg=40)
        prec = E.PREC_MIXED if fp32 else E.PREC_FP64

        def timed(pol):
            arr = (E.PolParams * B)(*([pol] * B))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(lstream)
            lib._check(lib.lib.evslx_chebav_multi(B, arr, dv.ptr, dy.ptr, prec), "evslx_chebav_multi")
            e1.record(lstream)
            e1.synchronize()
            return e0.elapsed_time(e1) / 1e3

        for _ in range(args.warmup):
            timed(p_hi)
            timed(p_lo)
        sampler.start()
        per = []
        for _ in range(args.steps):
            per.append((timed(p_hi) - timed(p_lo)) / (p_hi.deg - p_lo.deg))
        clocks = sampler.stop()
        t = statistics.median(per)
        launches = args.steps * (p_hi.deg + p_lo.deg + 4)
        bw = 1
        while bw < B:
            bw *= 2
        kernel = ("k_mf_panel<float>" if fp32 and B == 1 and lib.tuned_filter_variant(E.PREC_MIXED, 1) == 6
                  else "k_mf_step<%s,%d>" % ("float" if fp32 else "double", bw))
        lib.free_pol(p_lo)
    else:
        p_hi = lib.find_pol(iv, deg=400)
        dw = E.DeviceBuffer(lib.lib, 16 * n)
        for _ in range(args.warmup):
            lib._check(lib.lib.ChebAv(C.byref(p_hi), dv.ptr, dy.ptr, dw.ptr), "ChebAv")
        lib.filter_profile(True)
        sampler.start()
        for _ in range(args.steps):
            lib._check(lib.lib.ChebAv(C.byref(p_hi), dv.ptr, dy.ptr, dw.ptr), "ChebAv")
        sec, byt, launches, calls = lib.filter_stats()
        clocks = sampler.stop()
        lib.filter_profile(False)
        t = sec / launches
        kernel = "k_cheb_panel" if lib.filter_kernel()[0] == 7 else "k_cheb"
    peak, kind = measured_peak_hbm()
    gbs = abytes / t / 1e9
    traffic = profiled_traffic(kernel, "rspd-filter-" + ("fp32" if fp32 else "fp64"))
    if traffic:
        traffic *= nnz / 33.0e6  # captured at n = 10^6 (33M stored entries); traffic grows with the entries
    # one gather per stored entry brings B * s_x bytes; a 128-byte line carries up to 128 of them
    gathers_per_entry = max(1.0, B * sx / 128.0)
    gather_us = nnz * gathers_per_entry / (sm_count() * 1.965e9) * 1e6
    print(json.dumps({
        "metric": "filter SpMV GB/s", "value": gbs, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t * p_hi.deg, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if fp32 else "f64",
        "data": "synthetic (random sparse SPD, seeded; inputs larger than L2)",
        "config": {"workload": "rspd-filter: %s filter, %d column%s, degree %d, random sparse SPD n=%d, nnz=%d"
                               % ("FP32" if fp32 else "FP64", B, "" if B == 1 else "s", p_hi.deg, n, nnz),
                   "columns": B, "us_per_column_degree": 1e6 * t / B,
                   "tuned_variant": lib.tuned_filter_variant(E.PREC_MIXED if fp32 else E.PREC_FP64, B),
                   "storage": {"sigma": sigma, "stored_slots": stored, "stored_slots_unsorted": stored_plain,
                               "padding": stored / nnz - 1.0,
                               "panel_layout": dict(zip(("rows_per_block", "panel_width", "bytes"),
                                                        lib.matrix_panel_layout(fp32)))},
                   "kernel_times_us": (lib.filter_kernel()[1] if not fp32 and B == 1 else None),
                   "us_per_degree": 1e6 * t, "algorithmic_bytes_per_degree": abytes,
                   "generate_s": round(gen_s, 1), "bounds": [glo, ghi]},
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": gbs, "peak": peak, "peak_kind": kind,
                     "unit": "GB/s", "frac": gbs / peak, "traffic": traffic,
                     "frac_dram": (traffic / t / 1e9 / peak) if traffic else None,
                     "gather_bound_us": gather_us,
                     "hbm_bound_us": abytes / (peak * 1e9) * 1e6,
                     "frac_of_gather_bound": gather_us / 1e6 / t,
                     "note": "every stored entry gathers x[col] (B values) from its own cache line (random "
                             "columns, x far larger than L1): one L1TEX wavefront per entry and 128 bytes; ncu "
                             "shows L1TEX at 90-94% of peak and DRAM at 24-33% for one column, so the gather "
                             "rate (one line per clock per SM), not HBM, bounds the single-vector kernel; "
                             "gather_bound_us = nnz x max(1, B s_x / 128) / (SMs x 1.965 GHz); with B columns "
                             "each line carries B values and the bound moves to HBM once hbm_bound_us exceeds it"},
        "gpu_launches": launches, "clocks": clocks}))
    lib.free_pol(p_hi)


def run_dgemm(args):
    """dgemm: the FP64 Ritz product U = V(:, 1:K) Y of ChebLanNr
    (SRC/cheblanNr.c:333-399) through evsl_dgemm_device, V n x K and Y K x m
    column-major, device-resident seeded operands.  Device time per GEMM from
    CUDA events on the library stream, median of K steps; FP64 TFLOP/s =
    2 n K m / time, against the FP64 peak measured on this GPU by the
    library's probe (FMA chains and mma.sync f64 chains in registers)."""
    import ctypes as C

    import torch

    import evsl_b200 as E

    n, K, m = (int(x) for x in args.gemm.split(","))
    lib = E.Library()
    if args.dgemm_kernel >= 0:
        lib.lib.evslcu_set_dgemm_tiled(args.dgemm_kernel)
    lib.lib.evslcu_fp64_probe.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
    dfma, dmma = C.c_double(), C.c_double()
    lib._check(lib.lib.evslcu_fp64_probe(C.byref(dfma), C.byref(dmma)), "evslcu_fp64_probe")
    peak = max(dfma.value, dmma.value)
    g = torch.Generator(device="cuda").manual_seed(SEED)
    V = torch.randn(K, n, dtype=torch.float64, device="cuda", generator=g)  # column-major n x K
    Y = torch.randn(m, K, dtype=torch.float64, device="cuda", generator=g)  # column-major K x m
    U = torch.zeros(m, n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    lstream = torch.cuda.ExternalStream(lib.stream_handle())
    ci = lambda v: C.byref(C.c_int(v))  # noqa: E731
    cd = lambda v: C.byref(C.c_double(v))  # noqa: E731

    def gemm():
        lib.lib.evsl_dgemm_device(b"N", b"N", ci(n), ci(m), ci(K), cd(1.0), C.c_void_p(V.data_ptr()), ci(n),
                                  C.c_void_p(Y.data_ptr()), ci(K), cd(0.0), C.c_void_p(U.data_ptr()), ci(n))

    for _ in range(args.warmup):
        gemm()
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    times = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        gemm()
        e1.record(lstream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    clocks = sampler.stop()
    t = statistics.median(times)
    tf = 2.0 * n * K * m / t / 1e12
    # spot check of one output column against torch
    j = m // 2
    err = (U[j] - V.t() @ Y[j]).abs().max().item() / max(1e-300, (V.t() @ Y[j]).abs().max().item())
    print(json.dumps({
        "metric": "FP64 GEMM TFLOP/s (Ritz product)", "value": tf, "unit": "TFLOP/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded normal operands)",
        "config": {"workload": "dgemm: U = V(:,1:K) Y, n=%d K=%d m=%d" % (n, K, m), "check_rel_err": err},
        "roofline": {"bound": "fp64", "kernel": {0: "k_dgemm", 1: "k_dgemm_nn128"}.get(args.dgemm_kernel,
                                                                                   "k_dgemm_mma"),
                     "achieved": tf, "peak": peak,
                     "peak_kind": "measured on this GPU (FMA %.1f, mma.sync f64 %.1f TFLOP/s)" % (dfma.value,
                                                                                               dmma.value),
                     "unit": "TFLOP/s", "frac": tf / peak},
        "clocks": clocks}))


def run_pipeline(args):
    """lap3d-pipeline: the drop-in slicing pipeline of the reference's
    Laplacian driver (TESTS/PLanN/LapPLanN.c:10-283) with the drop-in slicing
    configuration's settings on a `--grid`^3 3-D Laplacian (default 50^3 =
    125,000 rows; the configuration's 100^3 takes about half an hour): kpmdos over
    [0.6, 1.2] (300 moments, Jackson damping, 30 seeded Rademacher probes),
    spslicer into 8 slices (npts = 10 ecount), then per slice find_pol
    (damping 2, thresholds 0.8 / 0.2) and ChebLanNr (tol 1e-8) from a seeded
    normal start vector.  One step = the whole pipeline; every slice's count
    is checked against the analytic spectrum and every residual against tol.
    Device time per stage from CUDA events on the library stream (the
    slicer's host time by the wall clock); within a slice, the filter's
    device time (events around each filter call) and the solver's own
    timers for the tridiagonal eigenproblems and the Ritz step."""
    import torch

    import evsl_b200 as E
    from evsl_b200 import workloads as W

    nx = args.grid
    lib = E.Library()
    ia, ja, a = W.laplacian_csr(nx, nx, nx)
    n = len(ia) - 1
    lib.set_csr(ia, ja, a)
    ev = W.laplacian_eigenvalues(nx, nx, nx)
    intv = [0.6, 1.2, 0.0, 12.0]
    probes = np.random.default_rng(SEED).choice(np.array([-1.0, 1.0]), size=(30, n))
    v0 = np.random.default_rng(SEED + 1).standard_normal(n)
    v0 /= np.linalg.norm(v0)
    lstream = torch.cuda.ExternalStream(lib.stream_handle())
    nexact_total = int(np.count_nonzero((ev >= intv[0]) & (ev <= intv[1])))

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        out = fn()
        e1.record(lstream)
        e1.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    def pipeline():
        (mu, ecnt), t_kpm = timed(lambda: lib.kpmdos_probes(300, 1, probes, intv))
        w0 = time.time()
        rc, sli = lib.spslicer(mu, intv, 8, int(10 * ecnt))
        t_sli = time.time() - w0
        if rc != 0:
            raise RuntimeError("spslicer returned %d" % rc)
        slices = []
        for i in range(8):
            iv = [float(sli[i]), float(sli[i + 1]), 0.0, 12.0]
            exact = int(np.count_nonzero((ev >= iv[0]) & (ev <= iv[1])))
            pol = lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2)
            maxit = max(2000, 5 * exact)  # about 4 Lanczos steps per eigenvalue are needed
            lib.stats_reset()
            lib.filter_profile(True)
            (lam, _, res), t = timed(lambda: lib.cheblan_nr(iv, maxit, TOL, v0, pol, want_vectors=False))
            t_filter, _, _, _ = lib.filter_stats()
            lib.filter_profile(False)
            st = lib.stats()
            kdim, ncand = lib.last_solve_info()
            # phases: filter (CUDA events around every filter call), the
            # tridiagonal eigenproblems (convergence tests and Ritz), the Ritz
            # step (GEMM V(:,1:K) Y, residuals, gather), and the rest of the
            # Lanczos loop (reorthogonalisation, norms, scalar reads)
            t_rest = st["t_iter"] - t_filter - st["t_eig"] - st["t_ritz"]
            slices.append({"interval": iv[:2], "degree": int(pol.deg), "found": int(len(lam)), "exact": exact,
                           "max_res": float(np.max(res)) if len(res) else 0.0, "seconds": t,
                           "lanczos_steps": int(kdim), "ritz_candidates": int(ncand),
                           "phase_s": {"filter": t_filter, "tridiag_eig": st["t_eig"], "ritz": st["t_ritz"],
                                       "reorth_and_rest": t_rest},
                           "ritz_gemm_tflop": 2e-12 * n * kdim * ncand})
            print("slice %d: %s" % (i, json.dumps(slices[-1])), file=sys.stderr, flush=True)
            lib.free_pol(pol)
        return {"kpm_s": t_kpm, "ecount": float(ecnt), "slicer_s": t_sli, "slices": slices}

    for _ in range(args.warmup):
        pipeline()
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    runs = [pipeline() for _ in range(args.steps)]
    clocks = sampler.stop()
    tot = [r["kpm_s"] + r["slicer_s"] + sum(x["seconds"] for x in r["slices"]) for r in runs]
    found = [sum(x["found"] for x in r["slices"]) for r in runs]
    ok = all(all(x["found"] == x["exact"] and x["max_res"] < TOL for x in r["slices"]) for r in runs)
    t = statistics.median(tot)
    last = runs[-1]
    print(json.dumps({
        "metric": METRIC, "value": found[-1] / tot[-1], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (3-D Dirichlet Laplacian, seeded probes and start)",
        "config": {"workload": "lap3d-pipeline: kpmdos (300 moments, 30 Rademacher probes) + spslicer (8 slices) + "
                               "8 x ChebLanNr over [0.6, 1.2] of the 3-D Laplacian %d^3 (n=%d)" % (nx, n, ),
                   "eigenvalues_in_interval": nexact_total, "kpm_s": last["kpm_s"], "ecount": last["ecount"],
                   "slicer_s": last["slicer_s"], "slices": last["slices"]},
        "all_steps_ok": bool(ok), "clocks": clocks}))


def run_block_cgs(args):
    """block-cgs: the blocked Gram-Schmidt of the mixed-precision refinement
    (evslcu_block_cgs2: two passes of GEMM projections against the earlier
    blocks, CGS + DGKS inside each block of b columns) on a seeded n x m
    block, `--gemm n,m,b`.  Device time per call from CUDA events on the
    library stream, median of K steps (the block is re-seeded between calls,
    outside the timed region).  FP64 flops counted: the GEMMs, 8 n c0 nb per
    block (two passes of W_prev^T W_b and W_b -= W_prev H), against the FP64
    peak measured by the library's probe."""
    import ctypes as C

    import torch

    import evsl_b200 as E

    n, m, b = (int(x) for x in args.gemm.split(","))
    lib = E.Library()
    if args.dgemm_kernel >= 0:
        lib.lib.evslcu_set_dgemm_tiled(args.dgemm_kernel)
    lib.lib.evslcu_fp64_probe.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
    dfma, dmma = C.c_double(), C.c_double()
    lib._check(lib.lib.evslcu_fp64_probe(C.byref(dfma), C.byref(dmma)), "evslcu_fp64_probe")
    peak = max(dfma.value, dmma.value)
    g = torch.Generator(device="cuda").manual_seed(SEED)
    W0 = torch.randn(m, n, dtype=torch.float64, device="cuda", generator=g)  # column-major n x m
    W = torch.empty_like(W0)
    H = torch.empty(m * b, dtype=torch.float64, device="cuda")
    nrm = torch.empty(1, dtype=torch.float64, device="cuda")
    lib.lib.evslcu_cgs_work_size.restype = C.c_size_t
    lib.lib.evslcu_cgs_work_size.argtypes = [C.c_int, C.c_int]
    work = torch.empty(int(lib.lib.evslcu_cgs_work_size(n, b)), dtype=torch.float64, device="cuda")
    fn = lib.lib.evslcu_block_cgs2
    fn.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    lstream = torch.cuda.ExternalStream(lib.stream_handle())

    def once():
        W.copy_(W0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        lib._check(fn(n, m, C.c_void_p(W.data_ptr()), b, C.c_void_p(H.data_ptr()), C.c_void_p(nrm.data_ptr()),
                      C.c_void_p(work.data_ptr())), "evslcu_block_cgs2")
        e1.record(lstream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    for _ in range(args.warmup):
        once()
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    times = [once() for _ in range(args.steps)]
    clocks = sampler.stop()
    t = statistics.median(times)
    flops = sum(8.0 * n * c0 * min(b, m - c0) for c0 in range(0, m, b))
    print(json.dumps({
        "metric": "blocked CGS2 FP64 TFLOP/s", "value": flops / t / 1e12, "unit": "TFLOP/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded normal block)",
        "config": {"workload": "block-cgs: n=%d m=%d block %d" % (n, m, b), "gemm_flops": flops},
        "roofline": {"bound": "fp64", "achieved": flops / t / 1e12, "peak": peak, "unit": "TFLOP/s",
                     "frac": flops / t / 1e12 / peak,
                     "peak_kind": "measured on this GPU (FMA %.1f, mma.sync f64 %.1f TFLOP/s)" % (dfma.value,
                                                                                               dmma.value)},
        "clocks": clocks}))


def run_multifilter(args):
    """lap3d-multifilter: the multi-column filter kernel alone on the 3-D
    Laplacian 100^3, `--ncols` columns with the slice request's polynomial
    (degree 1440).  Per-degree device time = (time of the degree-1440 filter
    - time of a degree-7 filter) / 1433, CUDA events on the library stream
    around evslx_chebav_multi, median of K steps.  Algorithmic bytes per
    degree = stored matrix (values + column indices + chunk tables) + 5 n B
    vector accesses.  `--sweep`: every kernel variant, width and precision
    once with the degree-7 filter (a launch list for ncu); `--low-degree`:
    only the degree-7 filter (a small capture)."""
    import torch

    import evsl_b200 as E
    from evsl_b200 import workloads as W

    lib = E.Library()
    ia, ja, a = W.laplacian_csr(NX, NY, NZ)
    ev = W.laplacian_eigenvalues(NX, NY, NZ)
    lib.set_csr(ia, ja, a)
    n = NX * NY * NZ
    intv, _ = slice_interval(ev, 0, args.count)
    p_hi = lib.find_pol(intv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    p_lo = lib.find_pol([1.0, 3.0, LMIN, LMAX], damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    prec = E.PREC_MIXED if args.precision == "mixed" else E.PREC_FP64
    lstream = torch.cuda.ExternalStream(lib.stream_handle())
    if args.sweep or args.low_degree:
        combos = [(v, pr, b) for v in range(6) for pr in (E.PREC_FP64, E.PREC_MIXED) for b in (1, 2, 4, 8, 16)] \
            if args.sweep else [(args.variant, prec, args.ncols)]
        for v, pr, b in combos:
            lib.set_filter_variant(v)
            X = np.random.default_rng(b).standard_normal((b, n))
            lib.chebav_multi([p_lo] * b, X, pr)
        print(json.dumps({"workload": "lap3d-multifilter " + ("sweep" if args.sweep else "low-degree"),
                          "launch_sets": len(combos), "degree": int(p_lo.deg)}))
        return
    lib.set_filter_variant(args.variant)
    B = args.ncols
    X = np.random.default_rng(B).standard_normal((B, n))

    def timed(pol):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        lib.chebav_multi([pol] * B, X, prec)
        e1.record(lstream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    for _ in range(args.warmup):
        timed(p_hi)
        timed(p_lo)
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    per = []
    for _ in range(args.steps):
        per.append((timed(p_hi) - timed(p_lo)) / (p_hi.deg - p_lo.deg))
    clocks = sampler.stop()
    t = statistics.median(per)
    vb, ib = lib.matrix_storage()
    _, nnz, stored = lib.problem_info()
    sx = 4 if prec == E.PREC_MIXED else 8
    abytes = stored * ((4 if prec == E.PREC_MIXED else vb) + ib) + 12 * ((n + 31) // 32) + 5 * n * B * sx
    peak, kind = measured_peak_hbm()
    gbs = abytes / t / 1e9
    print(json.dumps({
        "metric": "filter SpMV GB/s", "value": gbs, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t * p_hi.deg, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if prec == E.PREC_MIXED else "f64", "data": "synthetic",
        "config": {"workload": "lap3d-multifilter: %d columns, degree %d, 3-D Laplacian 100^3" % (B, p_hi.deg),
                   "variant": args.variant, "tuned_variant": lib.tuned_filter_variant(prec, B),
                   "us_per_degree": 1e6 * t, "us_per_column_degree": 1e6 * t / B,
                   "algorithmic_bytes_per_degree": abytes},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "peak_kind": kind, "unit": "GB/s",
                     "frac": gbs / peak, "traffic": None},
        "clocks": clocks}))
    lib.free_pol(p_hi)
    lib.free_pol(p_lo)


def run_reorth(args):
    """lap3d-reorth: ChebLanNr FP64 on the 3-D Laplacian 100^3 over [0.6, 0.9]
    (thousands of eigenvalues, so the restricted-trace test does not stop it)
    with maxit = `--maxit-reorth` (default 600): a run where the full
    reorthogonalisation (classical Gram-Schmidt + DGKS against the whole
    basis, 16 n k bytes per pass at step k) is a large share of the time.
    Reports the time per Lanczos step; the CGS kernels' own numbers come from
    ncu on this command."""
    import torch

    import evsl_b200
    from evsl_b200 import workloads as W

    lib = evsl_b200.Library()
    ia, ja, a = W.laplacian_csr(NX, NY, NZ)
    lib.set_csr(ia, ja, a)
    iv = [0.6, 0.9, LMIN, LMAX]
    pol = lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    n = NX * NY * NZ
    v0 = np.random.default_rng(SEED).standard_normal(n)
    v0 /= np.linalg.norm(v0)
    lstream = torch.cuda.ExternalStream(lib.stream_handle())
    k = args.maxit_reorth
    times = []
    for step in range(args.warmup + args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        lam, Y, res = lib.cheblan_nr(iv, k, TOL, v0, pol, want_vectors=False)
        e1.record(lstream)
        e1.synchronize()
        if step >= args.warmup:
            times.append(e0.elapsed_time(e1) / 1e3)
    t = statistics.median(times)
    kdim, _ = lib.last_solve_info()
    cgs_bytes = 2 * 16.0 * n * kdim * (kdim + 1) / 2  # two passes over V^T and V per step
    print(json.dumps({"workload": "lap3d-reorth: ChebLanNr FP64, [0.6, 0.9], maxit %d, filter degree %d" % (k, pol.deg),
                      "seconds_per_solve": t, "ms_per_lanczos_step": 1e3 * t / max(kdim, 1),
                      "lanczos_steps": int(kdim), "cgs_bytes_two_passes": cgs_bytes,
                      "eigenpairs": int(len(lam))}))
    lib.free_pol(pol)


def run_rspd_kpm(args):
    """rspd-kpm: kpmdos on the 2-million-row random sparse SPD matrix with the
    mixed-precision configuration's settings: 64 seeded Gaussian probes (drawn
    on the host, normalised inside as the reference does), 500 moments,
    Jackson damping, Gershgorin bounds; device time of the block recurrence
    (CUDA events around the KPM kernels).  Algorithmic bytes per block step
    as in lap3d-kpm (CSR 12 B per nonzero + 4 B per row, 3 probe vectors)."""
    import ctypes as C

    import evsl_b200
    from evsl_b200 import workloads as W

    n = args.rspd_n
    ia, ja, a = W.random_spd_csr(n, 16, RSPD_SEED)
    glo, ghi = W.gershgorin_bounds(ia, ja, a)
    nnz = int(ia[-1])
    lib = evsl_b200.Library()
    lib.lib.evslx_last_kpm_seconds.restype = C.c_double
    lib.set_split_range_bytes(int(args.split_range_mb * (1 << 20)))
    lib.lib.evslcu_set_kpm_split.argtypes = [C.c_int]
    lib.lib.evslcu_set_kpm_split(args.kpm_split)
    lib.set_csr(ia, ja, a)
    del ja, a
    B = args.kpm_probes if args.kpm_probes != 30 else 64
    M = args.kpm_moments if args.kpm_moments != 300 else 500
    probes = np.random.default_rng(RSPD_SEED).standard_normal((B, n))
    iv = [glo + 0.3 * (ghi - glo), glo + 0.35 * (ghi - glo), glo, ghi]
    for _ in range(args.warmup):
        lib.kpmdos_probes(M, 1, probes, iv)
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    secs = []
    for _ in range(args.steps):
        mu, ec = lib.kpmdos_probes(M, 1, probes, iv)
        secs.append(lib.lib.evslx_last_kpm_seconds())
    clocks = sampler.stop()
    t = statistics.median(secs)
    steps = (M + 1) // 2
    abytes = steps * (12.0 * nnz + 4.0 * (n + 1) + 3 * 8.0 * n * B)
    peak, kind = measured_peak_hbm()
    gbs = abytes / t / 1e9
    print(json.dumps({
        "metric": "KPM moments/s", "value": M / t, "unit": "moments/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (random sparse SPD, seeded Gaussian probes)",
        "config": {"workload": "rspd-kpm: kpmdos, %d probes, %d moments, random sparse SPD n=%d nnz=%d"
                               % (B, M, n, nnz), "block_steps": steps, "us_per_block_step": 1e6 * t / steps,
                   "kpm_split": args.kpm_split, "split_range_mb": args.split_range_mb,
                   "ecount": ec},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "peak_kind": kind, "unit": "GB/s",
                     "frac": gbs / peak, "algorithmic_bytes": abytes,
                     "note": "every stored entry gathers 8 B per probe from a random row of the probe block "
                             "(n x 32 x 8 B per launch = 512 MB, larger than L2): nnz x probes x 8 B of gather "
                             "traffic per step on top of the formula's bytes"},
        "clocks": clocks}))


def run_kpm(args):
    """lap3d-kpm: kpmdos on the 3-D Laplacian 100^3 with the config-2
    settings (30 Rademacher probes, 300 moments, Jackson damping; `--kpm-probes`,
    `--kpm-moments`), device time of the block recurrence (CUDA events around
    the KPM kernels).  Algorithmic bytes per block step: the CSR matrix
    (12 B per nonzero + 4 B per row) and 8 bytes per probe entry of each
    vector the step touches (read v_k, v_k-1; write v_k+1: 3 vectors with the
    product identities, 4 with a dot against the probe per degree); the
    identities need ceil(M/2) steps for M moments, the direct form M."""
    import ctypes as C

    import evsl_b200
    from evsl_b200 import workloads as W

    lib = evsl_b200.Library()
    lib.lib.evslx_last_kpm_seconds.restype = C.c_double
    lib.lib.evslcu_set_kpm_doubling(0 if args.kpm_direct else 1)
    if args.kpm_prefetch >= 0:
        lib.lib.evslcu_set_kpm_prefetch(args.kpm_prefetch)
    ia, ja, a = W.laplacian_csr(NX, NY, NZ)
    lib.set_csr(ia, ja, a)
    n, nnz = NX * NY * NZ, int(ia[-1])
    B, M = args.kpm_probes, args.kpm_moments
    iv = [0.6, 1.2, LMIN, LMAX]
    for _ in range(args.warmup):
        lib.kpmdos(M, 1, B, iv)
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    secs = []
    for _ in range(args.steps):
        lib.kpmdos(M, 1, B, iv)
        secs.append(lib.lib.evslx_last_kpm_seconds())
    clocks = sampler.stop()
    t = statistics.median(secs)
    steps = M if args.kpm_direct else (M + 1) // 2
    nvec_bytes = (4 if args.kpm_direct else 3) * 8.0 * n * B
    abytes = steps * (12.0 * nnz + 4.0 * (n + 1) + nvec_bytes)
    peak, kind = measured_peak_hbm()
    gbs = abytes / t / 1e9
    print(json.dumps({
        "metric": "KPM moments/s", "value": M / t, "unit": "moments/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (3-D Laplacian, device Rademacher probes)",
        "config": {"workload": "lap3d-kpm: kpmdos, %d probes, %d moments, 3-D Laplacian 100^3" % (B, M),
                   "method": "direct dots" if args.kpm_direct else "product identities",
                   "block_steps": steps, "us_per_block_step": 1e6 * t / steps},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "peak_kind": kind, "unit": "GB/s",
                     "frac": gbs / peak, "algorithmic_bytes": abytes},
        "clocks": clocks}))
    lib.lib.evslcu_set_kpm_doubling(1)


def _slice_plan(ev, start, nslices, count):
    """Consecutive gap-midpoint intervals of `count` eigenvalues from `start`."""
    from evsl_b200 import workloads as W

    out, lo = [], start
    for _ in range(nslices):
        a0, b0, c = W.gap_interval(ev, lo, count)
        out.append(([a0, b0, LMIN, LMAX], c))
        lo = b0 + 1e-12
    return out


def uneven_instances(count, seed=4, nmin=1e3, nmax=2e5):
    """The batched-instances configuration: `count` independent 2-D / 3-D
    Dirichlet Laplacians with n log-uniform in [nmin, nmax] (grid dims from
    the seed), each with an interval of 20-80 eigenvalues of its analytic
    spectrum starting at a seeded point of [0.3, 1.5], end points at gap
    midpoints.  Returns a list of (dims, intv, exact eigenvalues)."""
    from evsl_b200 import workloads as W

    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nn = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        if i % 2 == 0:
            s = max(int(round(np.sqrt(nn))), 10)
            dims, hi = (s, s + i % 3, 1), 8.0
        else:
            s = max(int(round(nn ** (1 / 3))), 8)
            dims, hi = (s, s + 1, s), 12.0
        ev = W.laplacian_eigenvalues(*dims)
        a0, b0, cnt = W.gap_interval(ev, float(rng.uniform(0.3, 1.5)), int(rng.integers(20, 81)))
        out.append((dims, [a0, b0, 0.0, hi], ev[(ev >= a0) & (ev <= b0)]))
    return out


def run_batch_uneven(args):
    """batch-uneven: `--instances` (default 128) independent Laplacians of
    uneven size (n log-uniform in [10^3, 2*10^5]), each with its own interval
    of 20-80 eigenvalues and its own find_pol degree, all submitted to one
    request engine (one slot per instance: every tick filters all slots --
    the slots of one matrix share multi-column launches, captured as CUDA
    graphs -- and advances every slot's Lanczos step).  One step = the whole
    batch; counts checked against the analytic spectra, residuals < tol.
    --compare-sequential also times the FP64 drop-in ChebLanNr on the same
    instances one after another."""
    import torch

    import evsl_b200 as E
    from evsl_b200 import workloads as W

    lib = E.Library()
    lib.set_batch_persistent(bool(args.batch_persistent))
    inst = uneven_instances(args.instances)
    mats, pols, vs = [], [], []
    for i, (dims, iv, _) in enumerate(inst):
        ia, ja, a = W.laplacian_csr(*dims)
        mats.append(lib.matrix(ia, ja, a))
        lib.set_csr(ia, ja, a)
        pols.append(lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000))
        v = np.random.default_rng(SEED + i).standard_normal(len(ia) - 1)
        vs.append(v / np.linalg.norm(v))
    prec = E.PREC_MIXED if args.precision == "mixed" else E.PREC_FP64
    lstream = torch.cuda.ExternalStream(lib.stream_handle())
    maxit = 1000
    phases = []

    def one_batch():
        eng = lib.engine(len(inst), precision=prec)
        for i, (dims, iv, _) in enumerate(inst):
            eng.submit_slice(mats[i], iv, pols[i], maxit, TOL, vs[i], i)
        eng.run()
        out = {}
        while True:
            r = eng.pop()
            if r is None:
                break
            out[int(r["tag"])] = r
        phases.append(eng.phase_times())
        eng.free()
        return out

    for _ in range(args.warmup):
        one_batch()
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    launches0 = lib.launch_count()
    times, found, ok, lat, max_err, max_res, bad = [], 0, True, [], 0.0, 0.0, []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        res = one_batch()
        e1.record(lstream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
        for i, (dims, iv, exact) in enumerate(inst):
            r = res[i]
            good = r["rc"] == 0 and r["nev"] == len(exact) and bool(np.all(r["res"] < TOL))
            if good:
                err = float(np.max(np.abs(np.sort(r["lam"]) - exact)))
                max_err = max(max_err, err)
                max_res = max(max_res, float(np.max(r["res"])))
                good = err <= 1e-8 * iv[3]
            if not good:
                bad.append({"instance": i, "dims": dims, "found": int(r["nev"]), "exact": int(len(exact))})
            ok = ok and good
            found += r["nev"]
            lat.append(1e3 * (r["t_finish"] - r["t_submit"]))
    launches = lib.launch_count() - launches0
    clocks = sampler.stop()
    t = sum(times)
    seq = None
    if args.compare_sequential:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        nseq, tseq = 0, 0.0
        for i, (dims, iv, _) in enumerate(inst):
            ia, ja, a = W.laplacian_csr(*dims)
            lib.set_csr(ia, ja, a)
            e0.record(lstream)
            lam, _, _ = lib.cheblan_nr(iv, maxit, TOL, vs[i], pols[i], want_vectors=False)
            e1.record(lstream)
            e1.synchronize()
            tseq += e0.elapsed_time(e1) / 1e3
            nseq += len(lam)
        seq = {"eigenpairs": nseq, "seconds": tseq, "eigenpairs_per_s": nseq / tseq,
               "engine_speedup": (found / t) / (nseq / tseq)}
    sizes = [int(np.prod(d)) for d, _, _ in inst]
    print(json.dumps({
        "metric": METRIC, "value": found / t, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 filter + f64" if prec == E.PREC_MIXED else "f64",
        "data": "synthetic (2-D/3-D Dirichlet Laplacians, seeded sizes, intervals and start vectors)",
        "config": {"workload": "batch-uneven: %d Laplacians, n log-uniform in [1e3, 2e5] (sum %d rows), 20-80 "
                               "eigenvalues each, one engine, %s" % (len(inst), sum(sizes), args.precision),
                   "batched_filter": "persistent" if args.batch_persistent else "one launch per degree",
                   "filter_degrees": [int(p.deg) for p in pols], "n": sizes, "tol": TOL, "maxit": maxit},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "sequential_chebLanNr_same_instances": seq,
        "engine_phase_seconds_last_step": phases[-1] if phases else None,
        "accuracy": {"max_abs_eig_err_vs_analytic": max_err, "max_residual": max_res,
                     "bar": "counts exact, |err| <= 1e-8 x width, residual < 1e-8", "failures": bad[:10]},
        "all_steps_ok": bool(ok), "gpu_launches": int(launches), "clocks": clocks}))
    for p in pols:
        lib.free_pol(p)
    for M in mats:
        M.free()


def run_batch(args):
    """lap3d-batch: `--slices` slices of `--count` eigenvalues above 0.6 on the
    3-D Laplacian 100^3 solved together by the request engine (one Lanczos
    step per tick for every slice, the filters of all slices sharing one
    multi-column launch per degree, captured as CUDA graphs), in FP64 or
    mixed precision (FP32 filter, FP64 Lanczos/orthogonalisation/Ritz, FP64
    refinement).  One step = the whole batch; checks exact counts and
    residuals <= tol."""
    import torch

    import evsl_b200 as E
    from evsl_b200 import workloads as W

    lib = E.Library()
    ia, ja, a = W.laplacian_csr(NX, NY, NZ)
    ev = W.laplacian_eigenvalues(NX, NY, NZ)
    lib.set_csr(ia, ja, a)
    M = lib.matrix(ia, ja, a)
    plan = _slice_plan(ev, 0.6, args.slices, args.count)
    pols = [lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000) for iv, _ in plan]
    prec = E.PREC_MIXED if args.precision == "mixed" else E.PREC_FP64
    n = NX * NY * NZ
    v0 = np.random.default_rng(SEED).standard_normal(n)
    v0 /= np.linalg.norm(v0)
    lstream = torch.cuda.ExternalStream(lib.stream_handle())
    widths = []

    def one_batch():
        eng = lib.engine(args.slices, precision=prec)
        for s, (iv, _) in enumerate(plan):
            eng.submit_slice(M, iv, pols[s], MAXIT, TOL, v0, s)
        eng.run()
        out = {}
        while True:
            r = eng.pop()
            if r is None:
                break
            out[int(r["tag"])] = r
        widths.append(eng.group_widths())
        eng.free()
        return out

    for _ in range(args.warmup):
        one_batch()
    sampler = ClockSampler(rank_info()[2])
    sampler.start()
    launches0 = lib.launch_count()
    times, found, ok, lat, max_err, max_res = [], 0, True, [], 0.0, 0.0
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        res = one_batch()
        e1.record(lstream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
        for s, (iv, cnt) in enumerate(plan):
            r = res[s]
            exact = ev[(ev >= iv[0]) & (ev <= iv[1])]
            good = r["rc"] == 0 and r["nev"] == cnt == len(exact) and bool(np.all(r["res"] < TOL))
            if good:
                err = float(np.max(np.abs(np.sort(r["lam"]) - exact)))
                max_err = max(max_err, err)
                max_res = max(max_res, float(np.max(r["res"])))
                good = err <= 1e-8 * (LMAX - LMIN)
            ok = ok and good
            found += r["nev"]
            lat.append(1e3 * (r["t_finish"] - r["t_submit"]))
    launches = lib.launch_count() - launches0
    clocks = sampler.stop()
    t = sum(times)
    seq = None
    if args.compare_sequential:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lstream)
        nseq = 0
        for s_, (iv, _) in enumerate(plan):
            lam, _, _ = lib.cheblan_nr(iv, MAXIT, TOL, v0, pols[s_], want_vectors=False)
            nseq += len(lam)
        e1.record(lstream)
        e1.synchronize()
        tseq = e0.elapsed_time(e1) / 1e3
        seq = {"eigenpairs": nseq, "seconds": tseq, "eigenpairs_per_s": nseq / tseq,
               "engine_speedup": (found / t) / (nseq / tseq)}
    print(json.dumps({
        "metric": METRIC, "value": found / t, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 filter + f64" if prec == E.PREC_MIXED else "f64",
        "data": "synthetic (3-D Dirichlet Laplacian, seeded start vector)",
        "config": {"workload": "lap3d-batch: %d slices of %d eigenvalues above 0.6 on the 3-D Laplacian 100^3, "
                               "solved together by the request engine, %s" % (args.slices, args.count,
                                                                              args.precision),
                   "filter_degrees": [int(p.deg) for p in pols], "tol": TOL, "maxit": MAXIT},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "filter_groups_by_width": widths[-1] if widths else None,
        "sequential_chebLanNr_same_slices": seq,
        "accuracy": {"max_abs_eig_err_vs_analytic": max_err, "max_residual": max_res,
                     "bar": "counts exact, |err| <= 1e-8 x width, residual < 1e-8"},
        "all_steps_ok": bool(ok), "gpu_launches": int(launches), "clocks": clocks}))
    for p in pols:
        lib.free_pol(p)
    M.free()


def run_serve(args):
    """serve: a seeded Poisson stream of requests at `--rate` per second for
    `--duration` seconds, served by the request engine under an HBM budget:
    50% slice solves (2-D 100x100 or 3-D 100^3 Laplacian, a random interval
    of 10-`--max-count` eigenvalues with end points at gap midpoints), 30%
    DOS estimates (kpmdos, 100-500 moments, 8-64 probes), 20% slice solves
    on small 2-D/3-D Laplacians (n log-uniform in [1e3, 2e5], 20-80
    eigenvalues).  Matrices stay resident.  Latency = submit to result
    (host clock of the engine); value = eigenpairs delivered per second of
    the run; every slice result is checked against the analytic spectrum."""
    import evsl_b200 as E
    from evsl_b200 import workloads as W

    lib = E.Library()
    rng = np.random.default_rng(SEED)
    prec = E.PREC_MIXED if args.precision == "mixed" else E.PREC_FP64
    mats = {}

    def matrix(dims):
        if dims not in mats:
            ia, ja, a = W.laplacian_csr(*dims)
            mats[dims] = (lib.matrix(ia, ja, a), np.sort(W.laplacian_eigenvalues(*dims)))
        return mats[dims]

    big = [(100, 100, 1), (NX, NY, NZ)] if args.serve_mix == "default" else [(100, 100, 1), (100, 100, 1)]
    for d in big:
        matrix(d)
    # the arrival schedule and the requests, all drawn before the run
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, size=int(args.rate * args.duration * 2) + 8))
    arrivals = arrivals[arrivals < args.duration]
    reqs = []
    for t in arrivals:
        u = rng.random()
        if u < 0.5 or u >= 0.8:
            if u < 0.5:
                dims = big[rng.integers(0, 2)]
                cnt = int(rng.integers(10, args.max_count + 1))
            else:
                nn = int(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
                if rng.random() < 0.5:
                    s = max(int(round(np.sqrt(nn))), 8)
                    dims = (s, s + int(rng.integers(0, 5)), 1)
                else:
                    s = max(int(round(nn ** (1 / 3))), 6)
                    dims = (s, s + int(rng.integers(0, 3)), s)
                cnt = int(rng.integers(20, 81))
            Mx, ev = matrix(dims)
            lo = float(rng.uniform(0.2, 1.5))
            a0, b0, c = W.gap_interval(ev, lo, cnt)
            hi_b = 8.0 if dims[2] == 1 else 12.0
            reqs.append(("slice", t, dims, [a0, b0, 0.0, hi_b], c))
        else:
            dims = big[rng.integers(0, 2)]
            hi_b = 8.0 if dims[2] == 1 else 12.0
            reqs.append(("kpm", t, dims, [0.5, 1.5, 0.0, hi_b], (int(rng.integers(100, 501)),
                                                                  int(rng.integers(8, 65)))))
    eng = lib.engine(args.slots, hbm_budget=int(args.budget_gb * 1e9), precision=prec)
    pols = {}
    n_h2d = 0
    import time as _t

    t0 = _t.perf_counter()
    i, done, lat, lat_slice, found, ok = 0, 0, [], [], 0, True
    failures = []
    while i < len(reqs) or eng.pending() > 0:
        now = _t.perf_counter() - t0
        while i < len(reqs) and reqs[i][1] <= now:
            kind, _, dims, iv, extra = reqs[i]
            Mx, ev = matrix(dims)
            if kind == "slice":
                pol = lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
                pols[i] = pol
                v = np.random.default_rng(SEED + i).standard_normal(Mx.n)
                eng.submit_slice(Mx, iv, pol, MAXIT, TOL, v / np.linalg.norm(v), i)
                n_h2d += 8 * Mx.n
            else:
                eng.submit_kpm(Mx, extra[0], 1, extra[1], iv, SEED + i, i)
            i += 1
        if eng.pending() > 0:
            eng.step()
        elif i < len(reqs):
            _t.sleep(max(0.0, min(0.05, reqs[i][1] - (_t.perf_counter() - t0))))
        while True:
            r = eng.pop()
            if r is None:
                break
            k = int(r["tag"])
            kind, t_arr, dims, iv, extra = reqs[k]
            ms = 1e3 * (r["t_finish"] - r["t_submit"])
            lat.append(ms)
            done += 1
            if kind == "slice":
                lat_slice.append(ms)
                Mx, ev = matrix(dims)
                exact = ev[(ev >= iv[0]) & (ev <= iv[1])]
                good = r["rc"] == 0 and r["nev"] == len(exact) and bool(np.all(r["res"] < TOL))
                ok = ok and good
                if not good and len(failures) < 10:
                    failures.append({"kind": kind, "dims": dims, "interval": iv[:2], "rc": r["rc"], "nev": r["nev"],
                                     "exact": int(len(exact)), "lanczos_steps": r["lanczos_steps"],
                                     "max_res": float(np.max(r["res"])) if r["nev"] else None})
                found += r["nev"]
                lib.free_pol(pols.pop(k))
            else:
                ok = ok and r["rc"] == 0
                if r["rc"] != 0 and len(failures) < 10:
                    failures.append({"kind": kind, "dims": dims, "rc": r["rc"]})
    wall = _t.perf_counter() - t0
    eng.free()
    for Mx, _ in mats.values():
        Mx.free()
    print(json.dumps({
        "metric": METRIC, "value": found / wall, "unit": UNIT, "n_gpus": 1, "steps": len(reqs), "warmup": 0,
        "ms_per_step": 1e3 * wall / max(len(reqs), 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 filter + f64" if prec == E.PREC_MIXED else "f64",
        "data": "synthetic (seeded Poisson request stream over Dirichlet Laplacians)",
        "config": {"workload": "serve (%s mix): Poisson %.2f req/s for %.0f s, %d slots, HBM budget %.0f GB, %s" % (
            args.serve_mix, args.rate, args.duration, args.slots, args.budget_gb, args.precision),
                   "requests": len(reqs), "completed": done},
        "latency_ms": {"p50": float(np.percentile(lat, 50)) if lat else None,
                       "p99": float(np.percentile(lat, 99)) if lat else None,
                       "slice_p50": float(np.percentile(lat_slice, 50)) if lat_slice else None,
                       "slice_p99": float(np.percentile(lat_slice, 99)) if lat_slice else None},
        "e2e": {"value": found / wall, "unit": UNIT, "h2d_bytes_per_step": n_h2d / max(len(reqs), 1),
                "d2h_bytes_per_step": 16 * found / max(len(reqs), 1)},
        "all_ok": bool(ok), "failures": failures}))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "lap3d-filter":
        run_filter(args)
    elif args.workload == "lap3d-batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "lap3d-multifilter":
        run_multifilter(args)
    elif args.workload == "lap3d-reorth":
        run_reorth(args)
    elif args.workload == "lap3d-kpm":
        run_kpm(args)
    elif args.workload == "rspd-filter":
        run_rspd_filter(args)
    elif args.workload == "dgemm":
        run_dgemm(args)
    elif args.workload == "batch-uneven":
        run_batch_uneven(args)
    elif args.workload == "lap3d-pipeline":
        run_pipeline(args)
    elif args.workload == "block-cgs":
        run_block_cgs(args)
    elif args.workload == "rspd-kpm":
        run_rspd_kpm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
