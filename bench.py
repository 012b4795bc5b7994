"""Benchmark: factor+solve unknowns/s of the AIFMM-LS direct solver on B200.

Workload (one GPU): depth-7 uniform quadtree, 6x6 Chebyshev nodes per leaf
(589,824 unknowns), kappa = 40, contrast q = 1.5 exp(-32|x|^2), NCA/ACA and
recompression tolerance 1e-10, FP64 (complex128), 8 plane-wave right-hand
sides at angles drawn from the seed.  The leaf tables are precomputed once on
the GPU (reported separately).  One step = assemble (ACA skeletons, bases,
M2L, leaf P2P) + eliminate + back-substitute for the 8 right-hand sides.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value: unknowns x steps / device time (CUDA events on the solver's stream, the
right-hand sides and solutions resident in HBM).  e2e: the same through the C
ABI with host buffers (H2D of b and D2H of x inside every step).  With N > 1
each rank solves its own replica (the direct solver does not shard; replicas
only).  --impl reference times the CPU oracle (the reference algorithm restated
in C++/OpenMP) on the host cores on a bounded sample.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n_cheb=6, kappa=40.0, degree=6, L=1.0, depth=7, tol_pow=10, q_kind="gauss_aw", q_amp=1.5,
                q_width=32.0, q_radius=0.5)
NRHS = 8
SEED = 20261203 + 1
METRIC = "factor+solve unknowns/s (FP64, 8 RHS)"
# DRAM bytes per launch of the QR factorisation kernel, from one ncu capture of
# three launches in the depth-4 step (46,848 + 66,816 + 46,592 read, 0 written)
QR_FACTOR_DRAM_BYTES_PER_LAUNCH = 53419
FAR_ENTRY_FLOPS = 2450  # algorithmic flops of one far-field entry (121-term Graf series)
CPU_SAMPLE_DEPTH = 4


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, lrank


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

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
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def fp64_peak_tflops(device):
    """Measured FP64 peak: cuBLAS DGEMM 8192^3 through torch (best of 5)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    torch.cuda.synchronize(device)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


_TABLES = {}


def max_over_ranks(t, pg, device=None):
    """The slowest rank's time: every rank contributes its own device-timed seconds
    (NCCL needs the value on the GPU, gloo on the host)."""
    if pg is None:
        return t
    import torch
    on_gpu = pg.get_backend() == "nccl"
    tt = torch.tensor([t], dtype=torch.float64, device=f"cuda:{device}" if on_gpu else "cpu")
    pg.all_reduce(tt, op=pg.ReduceOp.MAX)
    return float(tt.item())


def replica_throughput(world_size, unknowns, steps, t_max):
    """Whole-job unknowns/s of `world_size` independent replicas, each solving
    `unknowns` per step for `steps` steps, timed as the slowest rank."""
    return world_size * unknowns * steps / t_max


def _oracle_solve_time(O, depth, physics, nrhs, theta_seed):
    """Seconds of one oracle assemble + eliminate + back-substitute (tables precomputed once per depth)."""
    p = O.params(**physics, depth=depth)
    key = (depth, tuple(sorted(physics.items())))
    if key not in _TABLES:
        _TABLES[key] = O.tables(p)
    M, near, _ = _TABLES[key]
    rng = np.random.default_rng(theta_seed)
    th = rng.uniform(0, 2 * np.pi, nrhs)
    P = O.Problem(p, M, near)
    b = P.rhs_plane_wave(th)
    t0 = time.perf_counter()
    P.solve(b)
    dt = time.perf_counter() - t0
    P.close()
    return dt, 4 ** depth * physics["n_cheb"] ** 2


def _physics():
    return {k: v for k, v in WORKLOAD.items() if k in ("n_cheb", "kappa", "degree", "L", "tol_pow", "q_kind",
                                                        "q_amp", "q_width", "q_radius")}


def _extrapolate(t4, n4, t5, n5, depth):
    """Seconds per unknown grows by g = c5 / c4 per level from depth 4 to 5;
    carried geometrically to the target depth."""
    c4, c5 = t4 / n4, t5 / n5
    g = max(c5 / c4, 1.0)
    c = c5 * g ** (depth - 5)
    return 1.0 / c, g


def run_reference(args):
    """CPU oracle (the reference algorithm restated) on the host cores.

    Each step solves the benchmark physics at depth 4 (9,216 unknowns, 8 RHS);
    one depth-5 solve (36,864 unknowns) fixes how the cost per unknown grows per
    level, and the reported value is the depth-7 throughput extrapolated from the
    two.  The reference driver's default run (depth 5, Qchoice 0, kappa 10,
    TOL 1e-8, one RHS) is timed once as a further reference point."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    phys = _physics()
    times = []
    n4 = None
    for it in range(args.warmup + args.steps):
        dt, n4 = _oracle_solve_time(O, CPU_SAMPLE_DEPTH, phys, NRHS, SEED)
        if it >= args.warmup:
            times.append(dt)
    t4 = sum(times) / len(times)
    t5, n5 = _oracle_solve_time(O, CPU_SAMPLE_DEPTH + 1, phys, NRHS, SEED)
    value, g = _extrapolate(t4, n4, t5, n5, WORKLOAD["depth"])
    c1 = dict(n_cheb=6, kappa=10.0, degree=6, L=1.0, tol_pow=8, q_kind="gaussian160", q_amp=1.5, q_width=32.0,
              q_radius=0.5)
    tc1, nc1 = _oracle_solve_time(O, 5, c1, 1, SEED)
    sample = ("oracle solves of the benchmark physics on %d host threads: depth 4 (%d unknowns, %d RHS) per step "
              "(mean %.2f s), one depth-5 solve (%d unknowns, %.2f s); the cost per unknown grows %.3fx per "
              "level from depth 4 to 5 and is carried geometrically to depth %d (value extrapolated)"
              % (cores, n4, NRHS, t4, n5, t5, g, WORKLOAD["depth"]))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "unknowns/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t4,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
            "data": "synthetic", "config": {"workload": "lippmann-schwinger AIFMM direct solve, depth %d, "
                                                        "extrapolated from CPU solves at depths 4 and 5"
                                                        % WORKLOAD["depth"], **WORKLOAD, "nrhs": NRHS},
            "cpu_baseline": {"value": value, "unit": "unknowns/s", "cores": cores, "kind": "port",
                             "extrapolated": True, "sample": sample,
                             "measured": {"depth4_unknowns_per_s": n4 / t4, "depth5_unknowns_per_s": n5 / t5,
                                          "growth_per_level": g},
                             "reference_default_run": {"argv": "6 10 6 1 0 8 5", "unknowns": nc1, "nrhs": 1,
                                                       "seconds": tc1, "unknowns_per_s": nc1 / tc1}},
            "e2e": {"value": value, "unit": "unknowns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample():
    """The oracle on a bounded sample (rank 0, N = 1): one depth-4 and one
    depth-5 solve of the benchmark physics (about 30 s on 16 cores), the depth-7
    value extrapolated from the two."""
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count()
    phys = _physics()
    t4, n4 = _oracle_solve_time(O, CPU_SAMPLE_DEPTH, phys, NRHS, SEED)
    t5, n5 = _oracle_solve_time(O, CPU_SAMPLE_DEPTH + 1, phys, NRHS, SEED)
    value, g = _extrapolate(t4, n4, t5, n5, WORKLOAD["depth"])
    return {"value": value, "unit": "unknowns/s", "cores": cores, "kind": "port", "extrapolated": True,
            "sample": "one oracle solve of the benchmark physics at depth 4 (%d unknowns, %.2f s) and at depth 5 "
                      "(%d unknowns, %.2f s), %d RHS, OpenMP on all host threads; the cost per unknown grows "
                      "%.3fx per level and is carried geometrically to depth %d"
                      % (n4, t4, n5, t5, NRHS, g, WORKLOAD["depth"]),
            "measured": {"depth4_unknowns_per_s": n4 / t4, "depth5_unknowns_per_s": n5 / t5}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--depth", type=int, default=WORKLOAD["depth"], help="override the tree depth (diagnostics)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer loop (profiling runs)")
    ap.add_argument("--no-serving", action="store_true", help="skip the solve-latency measurement with kept factors")
    ap.add_argument("--no-peak", action="store_true", help="skip the cuBLAS FP64 peak measurement (profiling runs)")
    ap.add_argument("--batched", type=int, default=1, help="1: also run the 64-problem batched configuration")
    ap.add_argument("--refined", type=int, default=1, help="1: also time the refined form (GMRES) on the same problem")
    ap.add_argument("--trace", type=float, default=30.0, help="seconds of the serving trace (0: skip)")
    ap.add_argument("--mixed-serving", type=int, default=0,
                    help="1: also run the batched configuration and the trace in the mixed form (complex64 "
                         "factors, refined solves, FP64 refactoring where the refinement stagnates)")
    ap.add_argument("--no-kernel-profile", action="store_true",
                    help="skip the extra event-instrumented step that feeds the roofline (profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import aifmm_ls_b200 as A

    ws, rank, lrank = _dist()
    device = lrank if ws > 1 else 0
    torch.cuda.set_device(device)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist

    wl = dict(WORKLOAD)
    wl["depth"] = args.depth
    K = A.LSKernel(device=device, **wl)
    t_tab0 = time.perf_counter()
    K.tables_compute(round6=True)
    t_tables = time.perf_counter() - t_tab0
    T = A.FMM2DTree(K)
    rng = np.random.default_rng(SEED)
    th = rng.uniform(0, 2 * np.pi, NRHS)
    b_host = K.rhs_plane_wave(th)            # (nrhs, N) complex128, pinned below
    N = K.N
    b_pin = torch.from_numpy(b_host.view(np.float64).copy()).pin_memory()
    x_pin = torch.empty_like(b_pin).pin_memory()
    b_dev = b_pin.to(f"cuda:{device}")
    x_dev = torch.empty_like(b_dev)
    lib = A.load()
    sp = ctypes_void = None
    import ctypes
    sptr = ctypes.c_void_p()
    lib.aifmm_get_stream(K.h, ctypes.byref(sptr))
    stream = torch.cuda.ExternalStream(sptr.value, device=device)

    def step(host_io):
        T.createTree()
        T.assemble()
        if host_io:
            st = lib.aifmm_factorize_solve(K.h, NRHS, ctypes.cast(b_pin.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                           ctypes.cast(x_pin.data_ptr(), ctypes.POINTER(ctypes.c_double)), 0)
        else:
            st = lib.aifmm_factorize_solve(K.h, NRHS, ctypes.cast(b_dev.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                           ctypes.cast(x_dev.data_ptr(), ctypes.POINTER(ctypes.c_double)), 1)
        if st != 0:
            raise A.AifmmError(st, lib.aifmm_last_error(K.h).decode())
        return T.launch_counts()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize(device)

    tune_ms, tune_cols = K.autotune()
    for _ in range(args.warmup):
        step(False)
    fp64_peak = fp64_peak_tflops(device) if rank == 0 and not args.no_peak else None
    clocks = ClockSampler(device)
    clocks.start()
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    launches = 0
    asm_ms = fs_ms = 0.0
    solver_stats = None
    for _ in range(args.steps):
        lc = step(False)
        launches += lc[0] + lc[1]
        ms = T.phase_times()
        asm_ms += ms[2]
        fs_ms += ms[3]
        solver_stats = T.stats()
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    t_dev = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, pg, device)
    value = replica_throughput(ws, N, args.steps, t_dev)
    # end to end through the C ABI with host buffers (at most 5 steps: each is a
    # full factor + solve with the same cost as a timed step)
    t_e2e = None
    e2e_steps = min(args.steps, 5)
    if not args.no_e2e:
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            step(True)
        e1.record(stream)
        barrier()
        t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3, pg, device)
    x = (x_pin if t_e2e is not None else x_dev.cpu()).numpy().view(np.complex128).reshape(NRHS, N)
    finite = bool(np.isfinite(x).all())
    # one more step, untimed, with CUDA events around every launch of the dense
    # kernels: per-kernel durations and algorithmic flops for the roofline
    kinds = {0: "qr_factor", 1: "qr_solve", 2: "gemm"}
    prof = None
    if not args.no_kernel_profile:
        for kd in kinds:
            T.kernel_profile(kd, True)
        step(False)
        torch.cuda.synchronize(device)
        prof = {kinds[kd]: T.kernel_profile_read(kd) for kd in kinds}
        for kd in kinds:
            T.kernel_profile(kd, False)
    extra = {}
    try:
        serving = None if args.no_serving else solve_latency(T, K, lib, stream, device, args)
    except Exception as e:  # reported, never fatal for the headline measurement
        serving = {"error": repr(e)}
    if args.refined and rank == 0:
        try:
            extra["refined_vs_plain"] = refined_vs_plain(T, K, th, value, x)
        except Exception as e:
            extra["refined_vs_plain"] = {"error": repr(e)}
    # the headline problem's assembly workspaces are not needed by what follows
    lib.aifmm_trim(K.h)
    torch.cuda.empty_cache()
    if args.refined and rank == 0:
        try:
            extra["refined_c3_physics"] = refined_c3(device)
        except Exception as e:
            extra["refined_c3_physics"] = {"error": repr(e)}
    if args.batched and rank == 0:
        forms = [("batched_uneven", 0)] + ([("batched_uneven_mixed", 1)] if args.mixed_serving else [])
        for key, prec in forms:
            try:
                extra[key] = batched_uneven(device, precision=prec)
            except Exception as e:
                extra[key] = {"error": repr(e)}
        if "unknowns_per_s" in extra.get("batched_uneven_mixed", {}):
            extra["mixed_batched_over_plain_fp64"] = extra["batched_uneven_mixed"]["unknowns_per_s"] / value
    if args.trace > 0 and rank == 0:
        forms = [("serving_trace", 0)] + ([("serving_trace_mixed", 1)] if args.mixed_serving else [])
        for key, prec in forms:
            try:
                extra[key] = serving_trace(device, seconds=args.trace, precision=prec)
            except Exception as e:
                extra[key] = {"error": repr(e)}
    if rank == 0:
        peaks = measured_peaks()
        line = {
            "metric": METRIC, "value": value, "unit": "unknowns/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic",
            "config": {"workload": "lippmann-schwinger AIFMM direct solve, depth %d, %d unknowns, %d RHS"
                                   % (args.depth, N, NRHS), **wl, "nrhs": NRHS, "seed": SEED,
                       "parallelism": "replicas" if ws > 1 else "single",
                       "l2": "working set (~17 GiB) far larger than L2; no flush needed"},
            "e2e": None if t_e2e is None else {
                "value": replica_throughput(ws, N, e2e_steps, t_e2e), "unit": "unknowns/s", "steps": e2e_steps,
                "h2d_bytes_per_step": int(b_pin.numel() * 8), "d2h_bytes_per_step": int(x_pin.numel() * 8)},
            "gpu_launches": int(launches),
            "phases_ms_per_step": {"assemble": asm_ms / args.steps, "factorize_solve": fs_ms / args.steps,
                                   "tables_once": 1e3 * t_tables},
            "solver_stats_last_step": solver_stats,
            "clocks": clk,
            "solution_finite": finite,
            "gemm_autotune": {"ms_thin16_thin32_wide16_wide32": tune_ms.tolist(), "tile_cols_thin_wide": tune_cols.tolist()},
            "solves_with_cached_factors": serving,
            **extra,
        }
        if not args.no_cpu_baseline and ws == 1:
            line["cpu_baseline"] = cpu_baseline_sample()
        line["roofline"] = roofline(prof, fp64_peak, t_dev / args.steps) if prof else None
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def solve_latency(T, K, lib, stream, device, args, nrhs_list=(1, 8, 64)):
    """Latency of aifmm_solve against factors kept on the device (one factorisation,
    then W untimed and K timed solves per right-hand-side count; right-hand sides
    and solutions resident in HBM), issued launch by launch ("eager") and replayed
    as one CUDA graph ("graph"; its first call records the graph).  Each solve is
    bracketed by CUDA events on the solver's stream."""
    import ctypes
    import torch
    T.createTree()
    T.assemble()
    t0 = time.perf_counter()
    T.factorize()
    t_factor = time.perf_counter() - t0
    N = K.N
    out = {"factorize_ms": 1e3 * t_factor, "unknowns": N}
    rng = np.random.default_rng(SEED + 7)
    dp = ctypes.POINTER(ctypes.c_double)
    for nr in nrhs_list:
        th = rng.uniform(0, 2 * np.pi, nr)
        b = torch.from_numpy(K.rhs_plane_wave(th).view(np.float64).copy()).to(f"cuda:{device}")
        x = torch.empty_like(b)
        res = {}
        for mode, flags in (("eager", 1), ("graph", 1 | 4)):  # AIFMM_PTR_DEVICE, | AIFMM_SOLVE_GRAPH
            ms = []
            launches = 0
            t_first = None
            for it in range(args.warmup + args.steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                h0 = time.perf_counter()
                e0.record(stream)
                st = lib.aifmm_solve(K.h, nr, ctypes.cast(b.data_ptr(), dp), N, ctypes.cast(x.data_ptr(), dp), N,
                                     None, flags)
                e1.record(stream)
                if st != 0:
                    raise RuntimeError(lib.aifmm_last_error(K.h).decode())
                e1.synchronize()
                if it == 0:
                    t_first = 1e3 * (time.perf_counter() - h0)
                if it >= args.warmup:
                    ms.append(e0.elapsed_time(e1))
                    launches = T.launch_counts_split()[1]
            ms = np.array(ms)
            res[mode] = {"p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
                         "mean_ms": float(ms.mean()), "solves": int(ms.size), "first_call_ms": t_first,
                         "rhs_unknowns_per_s": float(N * nr / (ms.mean() * 1e-3)),
                         "gpu_launches_per_solve": int(launches)}
        out["nrhs_%d" % nr] = res
        del b, x
    return out


def _refined_run(T, K, b, factor_tol_pow, rtol, precision=0):
    """createTree + assemble + factorise (recompression tolerance 10^-factor_tol_pow,
    assembly kept; precision 1: complex64 factors) + GMRES to rtol; host wall clock
    per phase."""
    T.set_factor_tolerance(factor_tol_pow)
    try:
        t0 = time.perf_counter()
        T.createTree()
        T.assemble()
        t1 = time.perf_counter()
        T.factorize(keep_assembly=True, precision=precision)
        t2 = time.perf_counter()
        try:
            x, iters, relres = T.solve_refined(b, rtol=rtol, maxit=90)
            err = None
        except Exception as e:  # stagnation is reported by the library, not hidden
            x, iters, relres, err = None, None, None, str(e)
        t3 = time.perf_counter()
    finally:
        T.set_factor_tolerance(0)
    out = {"assemble_s": t1 - t0, "factorize_s": t2 - t1, "gmres_s": t3 - t2, "total_s": t3 - t0,
           "gmres_iterations": iters, "relative_residual": relres, "converged": err is None,
           "factors": "complex64" if precision == 1 else "complex128"}
    if err is not None:
        out["error"] = err
    return x, out


def refined_vs_plain(T, K, th, plain_value, x_plain):
    """The refined forms on the benchmark problem itself: the same assembly (ACA
    tolerance 1e-10), the factorisation at recompression tolerance 1e-6 in complex128
    and in complex64 (the mixed form), FP64 GMRES against the compressed operator to
    relative residual 1e-10, for the same 8 right-hand sides; against the plain FP64
    direct solve of the timed steps.  The mixed form's error is stated against the
    complex128-factored refined solution of the same compressed system."""
    b = K.rhs_plane_wave(th)
    N = K.N
    res = {}
    for name, prec in (("fp64_factors", 0), ("mixed_c64_factors", 1)):
        x, out = _refined_run(T, K, b, 6, 1e-10, precision=prec)
        if x is not None:
            out["unknowns_per_s"] = N / out["total_s"]
            out["over_plain_fp64"] = out["unknowns_per_s"] / plain_value
            out["rel_diff_to_plain_solution"] = float(np.linalg.norm(x - x_plain) / np.linalg.norm(x_plain))
        res[name] = (x, out)
    x64 = res["fp64_factors"][0]
    xm, om = res["mixed_c64_factors"]
    if xm is not None and x64 is not None:
        om["rel_err_vs_fp64_refined"] = float(np.linalg.norm(xm - x64) / np.linalg.norm(x64))
    return {"plain_fp64_unknowns_per_s": plain_value,
            "fp64_factors": res["fp64_factors"][1], "mixed_c64_factors": om,
            "mixed_over_plain": om.get("over_plain_fp64"),
            "timing": "host wall clock of one run each (tree, assembly, factorisation, GMRES with host buffers)"}


def refined_c3(device, depth=6, nrhs=32, seed=SEED + 2):
    """The mixed-precision configuration's physics (8x8 nodes, kappa 80, disk q = 2 for
    |x| < 0.5, NCA tolerance 1e-6, 32 plane waves, refinement to 1e-10): factorisation
    at the problem's tolerance in complex64 (the mixed form) and in complex128, each
    the preconditioner of FP64 GMRES against the compressed operator.  The mixed
    form's error is stated against the complex128-factored refined solution."""
    import aifmm_ls_b200 as A
    K = A.LSKernel(n_cheb=8, kappa=80.0, degree=6, depth=depth, tol_pow=6, q_kind="disk", q_amp=2.0, q_radius=0.5,
                   device=device)
    res = {}
    try:
        t0 = time.perf_counter()
        K.tables_compute(round6=True)
        t_tab = time.perf_counter() - t0
        T = A.FMM2DTree(K)
        rng = np.random.default_rng(seed)
        b = K.rhs_plane_wave(rng.uniform(0, 2 * np.pi, nrhs))
        for name, prec in (("mixed_c64_factors", 1), ("fp64_factors", 0)):
            x, out = _refined_run(T, K, b, 0, 1e-10, precision=prec)
            xd = T.solve_factored(b)  # the direct solve alone, same factors
            out["direct_solve_relative_residual"] = float(
                np.max(np.linalg.norm(b - T.compressed_matvec(xd), axis=1) / np.linalg.norm(b, axis=1)))
            if x is not None:
                out["unknowns_per_s"] = K.N / out["total_s"]
            res[name] = (x, out)
            lib = A.load()
            lib.aifmm_trim(K.h)
    finally:
        K.close()
    xm, om = res["mixed_c64_factors"]
    x64, o64 = res["fp64_factors"]
    if xm is not None and x64 is not None:
        om["rel_err_vs_fp64_refined"] = float(np.linalg.norm(xm - x64) / np.linalg.norm(x64))
    ratio = om["unknowns_per_s"] / o64["unknowns_per_s"] if "unknowns_per_s" in om and "unknowns_per_s" in o64 else None
    return {"depth": depth, "unknowns": K.N, "nrhs": nrhs, "tables_s": t_tab,
            "mixed_c64_factors": om, "fp64_factors": o64, "mixed_over_fp64_factors": ratio,
            "note": "depth 6 instead of 7 (8x8 nodes)"}


def _random_problem(rng, depth):
    """A problem of the batched / serving configurations: 6x6 nodes, kappa log-uniform in
    [5, 60], contrast a Gaussian of amplitude U[0.5, 2] (width 32) or a disk of radius
    U[0.2, 0.7] (amplitude 2), NCA tolerance 1e-8."""
    kappa = float(np.exp(rng.uniform(np.log(5.0), np.log(60.0))))
    if rng.uniform() < 0.5:
        q = dict(q_kind="gauss_aw", q_amp=float(rng.uniform(0.5, 2.0)), q_width=32.0)
    else:
        q = dict(q_kind="disk", q_amp=2.0, q_radius=float(rng.uniform(0.2, 0.7)))
    return dict(n_cheb=6, kappa=kappa, degree=6, depth=int(depth), tol_pow=8, **q)


def batched_uneven(device, nprob=64, workers=4, seed=SEED + 3, precision=0, rtol=1e-8):
    """64 independent problems of depth U{4..7}, each factored and solved for one random
    complex Gaussian right-hand side, run through the serving engine (workers drive their
    own handles and streams, so the problems overlap on the GPU; admission by device
    memory).  precision 1: the mixed form (complex64 factors, each solve refined by FP64
    GMRES to rtol); 0: FP64 factors and direct solves.  Whole-job unknowns/s = total
    unknowns / wall time of the batch."""
    import aifmm_ls_b200 as A
    rng = np.random.default_rng(seed)
    probs = [_random_problem(rng, rng.integers(4, 8)) for _ in range(nprob)]
    S = A.Server(device=device, workers=workers, max_batch_rhs=64, factor_workers=workers, precision=precision,
                 rtol=rtol)
    try:
        t0 = time.perf_counter()
        fids = [S.factorize(i, **kw) for i, kw in enumerate(probs)]
        sids = []
        for i, kw in enumerate(probs):
            N = 4 ** kw["depth"] * 36
            b = rng.standard_normal((1, N)) + 1j * rng.standard_normal((1, N))
            sids.append(S.solve(i, b))
        bad = 0
        codes = {}
        for r in fids + sids:
            st = S.wait(r, timeout=3600)[0]
            bad += st != 0
            if st != 0:
                codes[str(st)] = codes.get(str(st), 0) + 1
        wall = time.perf_counter() - t0
        stats = S.stats()
    finally:
        S.close()
    unknowns = sum(4 ** kw["depth"] * 36 for kw in probs)
    depths = [kw["depth"] for kw in probs]
    return {"problems": nprob, "depth_counts": {str(d): depths.count(d) for d in range(4, 8)},
            "form": "mixed: complex64 factors, refined to %g" % rtol if precision == 1 else "plain FP64",
            "unknowns": unknowns, "wall_s": wall, "unknowns_per_s": unknowns / wall, "failed": bad,
            "failed_status_counts": codes,
            "workers": workers, "timing": "host wall clock around the whole batch (several streams)",
            "server": stats}


class _PlaneWaves:
    """Plane-wave right-hand sides b = -kappa^2 q(x) exp(i kappa (x cos t + y sin t))
    (LS/LS_functions.hpp:113-120) computed on the host from one grid per depth, so
    that the trace needs no solver handle per geometry.  The first geometry of each
    depth is checked against the library's own aifmm_rhs_plane_wave."""

    def __init__(self, A):
        self.A = A
        self.grids = {}

    @staticmethod
    def contrast(kw, xy):
        R2 = (xy ** 2).sum(1)
        if kw["q_kind"] == "gauss_aw":
            return kw["q_amp"] * np.exp(-kw["q_width"] * R2)
        return np.where(R2 < kw["q_radius"] ** 2, kw["q_amp"], 0.0)

    def __call__(self, kw, thetas):
        d = kw["depth"]
        th = np.atleast_1d(thetas)
        if d not in self.grids:
            K = self.A.LSKernel(**kw)
            self.grids[d] = K.gridPoints
            want = K.rhs_plane_wave(th)
            K.close()
            got = self._b(kw, self.grids[d], th)
            if not np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max()):
                raise RuntimeError("host plane waves disagree with aifmm_rhs_plane_wave")
        return self._b(kw, self.grids[d], th)

    def _b(self, kw, xy, th):
        q = self.contrast(kw, xy)
        ph = kw["kappa"] * (np.outer(np.cos(th), xy[:, 0]) + np.outer(np.sin(th), xy[:, 1]))
        return -kw["kappa"] ** 2 * q[None, :] * np.exp(1j * ph)


def serving_trace(device, seconds=30.0, rate=200.0, workers=8, seed=SEED + 4, precision=0, rtol=1e-8):
    """Poisson arrivals at `rate` req/s for `seconds`: 5% factorize requests for new
    geometries (depth 5, problem as the batched configuration), 95% solve requests
    of U{1..64} plane waves against a random geometry already submitted.  Latency =
    submission to completion (host clock); the engine batches the solves queued for
    a geometry.  precision 1: the mixed form (complex64 factors, each solve refined to
    rtol); 0: FP64 factors and direct solves."""
    import aifmm_ls_b200 as A
    rng = np.random.default_rng(seed)
    waves = _PlaneWaves(A)
    S = A.Server(device=device, workers=workers, max_batch_rhs=64, factor_workers=workers // 2, precision=precision,
                 rtol=rtol)
    lat = {"solve": [], "factorize": []}
    try:
        keys = []
        # a few geometries resident before the clock starts
        for key in range(4):
            kw = _random_problem(rng, 5)
            S.wait(S.factorize(key, **kw), timeout=3600)
            keys.append((key, kw))
        pending = []
        t0 = time.perf_counter()
        t_next = t0
        nreq = 0
        solved_unknowns = 0
        while True:
            now = time.perf_counter()
            if now - t0 >= seconds:
                break
            if now < t_next:
                time.sleep(min(t_next - now, 0.002))
                continue
            t_next += rng.exponential(1.0 / rate)
            nreq += 1
            if rng.uniform() < 0.05:
                key = len(keys)
                kw = _random_problem(rng, 5)
                keys.append((key, kw))
                pending.append(("factorize", S.factorize(key, **kw), 0))
            else:
                key, kw = keys[int(rng.integers(0, len(keys)))]
                nr = int(rng.integers(1, 65))
                b = waves(kw, rng.uniform(0, 2 * np.pi, nr))
                pending.append(("solve", S.solve(key, b), b.size))
        failed = 0
        codes = {}
        for kind, rid, nunk in pending:
            st, ms, br, _ = S.wait(rid, timeout=3600)
            if st == 0:
                lat[kind].append(ms)
                solved_unknowns += nunk
            else:
                failed += 1
                codes[str(st)] = codes.get(str(st), 0) + 1
        wall = time.perf_counter() - t0
        stats = S.stats()
    finally:
        S.close()
    out = {"seconds": seconds, "rate_req_per_s": rate, "requests": nreq, "failed": failed, "wall_s": wall,
           "failed_status_counts": codes,
           "form": "mixed: complex64 factors, refined to %g" % rtol if precision == 1 else "plain FP64",
           "rhs_unknowns_per_s": solved_unknowns / wall, "server": stats,
           "note": "trace shortened from 10 minutes to keep the benchmark within minutes; new geometries at "
                   "depth 5 (a depth-7 factorisation takes seconds, longer than the mean gap between factorize "
                   "requests at 5% of 200 req/s); wall_s includes draining the queue after the last arrival"}
    for kind, v in lat.items():
        if v:
            out[kind] = {"count": len(v), "p50_ms": float(np.percentile(v, 50)), "p99_ms": float(np.percentile(v, 99))}
    return out


def roofline(prof, fp64_peak, t_dev):
    """Dominant kernel of one event-instrumented step (by CUDA-event device time on the solver's
    stream): algorithmic flops per launch / average launch duration, against the
    FP64 peak measured above (cuBLAS DGEMM; MEASURED_PEAKS.json has no FP64 figure)."""
    name, (n, ms, fl) = max(prof.items(), key=lambda kv: kv[1][1])
    if n == 0 or ms <= 0:
        return None
    achieved = fl / (ms * 1e-3) / 1e12
    traffic = QR_FACTOR_DRAM_BYTES_PER_LAUNCH if name == "qr_factor" else None
    return {"bound": "tensor", "kernel": name, "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": achieved / fp64_peak if fp64_peak else None, "traffic": traffic,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum, mean of 3 launches of "
                               "qr_factor_smem_kernel in the depth-4 step") if traffic else None,
            "peak_source": "FP64, measured by bench.py (cuBLAS DGEMM 8192^3, best of 5)",
            "launches": n, "avg_launch_us": 1e3 * ms / n, "algorithmic_flops_per_launch": fl / n,
            "device_time_share": 1e-3 * ms / t_dev,
            "all_kernels": {k: {"launches": v[0], "ms": v[1], "flops": v[2]} for k, v in prof.items()}}


if __name__ == "__main__":
    main()
