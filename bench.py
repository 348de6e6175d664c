"""Benchmark: SIMPLEC outer iterations of an Euler nozzle on B200.

Workload (one step = one outer iteration `it` of src/mach2d_main.f90:94-445):
the C01 cosine nozzle (Lc = 2, Ld = 4, throat r = 1 m) at 512 x 256 real
volumes (514 x 258 with the ghost ring), Euler, constant properties
(gamma = 1.4, R = 287), p0 = 1e6 Pa, T0 = 1000 K, MSI for u, v and p'
(nitm_u = 5, nitm_p = 20, tol 1e-2), itpmax = 20, SCARBOROUGH time stepper,
FP64.  Metric: cell-updates/s = real cells x outer iterations / time.

Each outer iteration runs as one captured CUDA graph (m2d_ctx_set_graph: the
p' loop is a conditional node, its exit and the next time step are decided
on the device), which gives bitwise the results of the host-driven mode.

Each rank runs its own nozzle instance (replicas: a single grid does not
shard, see the MSI factorisation); value = total cell-updates of all ranks /
max-over-ranks time.  The per-iteration working set (~140 MB of fields,
coefficients and solver factors) exceeds the 126 MB L2, so no explicit L2
flush is inserted between iterations.

Besides the headline line, one-GPU runs add: `fp32_sweeps` (the same
workload with MSI factors and sweeps in FP32 inside the FP64 iteration),
`time_to_residual` (the 80x40 Euler nozzle to its stopping iteration, FP64
and FP32 sweeps on the GPU, and the serial oracle extrapolated from a
sample), and `learned` (the learned p' correction trained on this workload's
harvested p' systems, against plain MSI on held-out ones).

--impl reference times the CPU restatement of the reference (the reference
itself is Fortran and no Fortran compiler exists on this image) on the
host, serially like the reference build, on a bounded sample of the same
workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# Many instances' captured iterations are in flight at once in the batch and
# sweep figures; with the default 8 hardware work queues, streams share queues
# and serialise.  Read when the process creates its CUDA context, so set here,
# before torch or the library touches the device.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

NXR, NYR = 512, 256
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nxr", type=int, default=NXR)
    ap.add_argument("--nyr", type=int, default=NYR)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=16,
                    help="instances of the same workload for the batch throughput figure (0: skip)")
    ap.add_argument("--no-graph", action="store_true",
                    help="drive each iteration from the host instead of one captured graph (same results; for "
                         "profilers that do not look inside conditional graph nodes)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the time-to-residual, FP32-sweep and learned-correction figures")
    ap.add_argument("--ttr-cap", type=float, default=0.0,
                    help="wall-time cap (s) of each 512x256 time-to-residual run (0, the default: skip them; "
                         "the four runs take about ten minutes with 300)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def make_case(nxr, nyr):
    from mach2d_b200.simplec import euler_cosine_case
    return euler_cosine_case(nxr, nyr)


def workload_config(args, extra=None):
    cfg = {"workload": f"simplec-outer-iteration euler c01-cosine-nozzle {args.nxr}x{args.nyr}",
           "real_cells": args.nxr * args.nyr, "grid_with_ghosts": [args.nxr + 2, args.nyr + 2],
           "solver": "MSI (nitm_u=5, nitm_p=20, tol 1e-2), itpmax=20, SCARBOROUGH dt",
           "precision": "fp64", "parallelism": "replicas (one instance per rank)",
           "l2": "working set per iteration ~140 MB > 126 MB L2; no flush"}
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            self.rows.append([s.strip() for s in line.split(",")])

    def __exit__(self, *exc):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        sm = []
        mx = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for k, nm in enumerate(names):
                    if r[4 + k].lower().startswith("active"):
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- reference arm
def cpu_sample(args, seconds, skip=0):
    """Times the CPU restatement of the reference (serial, like the shipped
    reference build) on outer iterations of the same workload: `skip`
    untimed iterations from the initial guess, then iterations for about
    `seconds`."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _oracle import OracleCase
    o = OracleCase(make_case(args.nxr, args.nyr))
    for _ in range(skip):
        o.iterate()
    t0 = time.perf_counter()
    n = 0
    while True:
        rc, _ = o.iterate()
        n += 1
        if rc or time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return args.nxr * args.nyr * n / dt, n, dt


def _cpu_worker(nxr, nyr, skip, seconds, q):
    """One process of the all-cores CPU baseline: its own instance of the
    workload, `skip` untimed iterations, then iterations for about `seconds`."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _oracle import OracleCase
    from mach2d_b200.simplec import euler_cosine_case
    o = OracleCase(euler_cosine_case(nxr, nyr))
    for _ in range(skip):
        o.iterate()
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds:
        o.iterate()
        n += 1
    q.put((n, time.perf_counter() - t0))


def cpu_sample_all_cores(args, seconds, skip=0):
    """The serial CPU restatement on every host core at once: one process per
    core, each advancing its own instance of the workload (the reference's
    build is serial, so independent runs are how it uses more cores).
    Processes are started with `spawn`.  Returns (aggregate cell-updates/s,
    processes, iterations)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    nproc = os.cpu_count() or 1
    q = ctx.Queue()
    procs = [ctx.Process(target=_cpu_worker, args=(args.nxr, args.nyr, skip, seconds, q)) for _ in range(nproc)]
    for pr in procs:
        pr.start()
    res = [q.get() for _ in procs]
    for pr in procs:
        pr.join()
    rate = sum(args.nxr * args.nyr * n / t for n, t in res)
    return rate, nproc, sum(n for n, _ in res)


def run_reference(args):
    """The reference arm: the serial CPU restatement on the same iterations
    the GPU arm times -- W untimed warm-up iterations from the initial guess,
    then K timed iterations (each step one outer iteration)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _oracle import OracleCase
    o = OracleCase(make_case(args.nxr, args.nyr))
    for _ in range(args.warmup):
        o.iterate()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc, _ = o.iterate()
        if rc:
            raise RuntimeError(f"oracle iteration failed with {rc}")
    total_s = time.perf_counter() - t0
    value = args.nxr * args.nyr * args.steps / total_s
    line = {
        "impl": "reference", "metric": "cell-updates/s (SIMPLEC outer iterations)", "value": value,
        "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded nozzle geometry, isentropic initial guess)",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": 1, "kind": "port",
                         "sample": f"outer iterations {args.warmup + 1}..{args.warmup + args.steps} (the ones the "
                                   "GPU arm times), serial C restatement; the reference is Fortran, its shipped "
                                   "build is serial and no Fortran compiler exists on the image or the GPU box"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def msi_algorithmic_bytes(nd, N, nit):
    """FP64 compulsory traffic of one MSI solve launch: factorisation (A in,
    dl + du out), initial residual (A, x, b in; r out), and per iteration the
    forward sweep (r, dl in; w out), the backward sweep (w, du, x in; x out)
    and the residual (A, x, b in; r out)."""
    nl, nu = (5, 4) if nd == 9 else (4, 3)
    lu = nd + nl + nu
    res = nd + 3
    it = (1 + nl + 1) + (1 + nu + 2) + res
    return 8 * N * (lu + res + nit * it)


# FP64 bytes per cell of the non-MSI work of one Euler outer iteration (each
# distinct plane read once and written once per kernel, 8 B): u and v
# assembly 2 x 200, SIMPLEC d-coefficients 240, face velocities 320, nodal
# velocity correction 224, mass check 80, T from H and the densities 88,
# Scarborough coefficient means 256, boundary strips and backups 24; per p'
# cycle: p' coefficients 128 and source 120, face correction 184, p / rho /
# face-rho correction 96, max|p'| 8
STEP_FIXED_B = 1632
P_CYCLE_B = 536


def step_algorithmic_bytes(N, nit_u, nit_v, nit_p, itp):
    """Algorithmic HBM bytes of one outer iteration with the MSI iteration
    counts the device reported (the two MSI9 solves, itp p' cycles of one
    MSI5 solve each)."""
    return (N * STEP_FIXED_B + msi_algorithmic_bytes(9, N, nit_u) + msi_algorithmic_bytes(9, N, nit_v)
            + itp * (N * P_CYCLE_B + msi_algorithmic_bytes(5, N, nit_p)))


def run_ours(args):
    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    from mach2d_b200._lib import check, lib
    from mach2d_b200.simplec import Simplec

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    sim = Simplec(make_case(args.nxr, args.nyr), device=local)
    sim.set_graph(not args.no_graph)   # one captured CUDA graph per outer iteration (bitwise the same results)
    L = lib()
    stream_ptr = ctypes.c_void_p()
    L.m2d_ctx_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    check(L.m2d_ctx_stream(sim._ctx, ctypes.byref(stream_ptr)))
    st = torch.cuda.ExternalStream(stream_ptr.value, device=local)

    for _ in range(args.warmup):
        sim.iterate()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = sim.scalar("launches")
    itp = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    counts = []
    with ClockSampler(local) as clk:
        e0.record(st)
        for _ in range(args.steps):
            r = sim.iterate()
            itp.append(r.itp_used)
            counts.append((sim.scalar("nit_u"), sim.scalar("nit_v"), sim.scalar("nit_p"), r.itp_used))
        e1.record(st)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = int(sim.scalar("launches") - l0)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    cells = args.nxr * args.nyr
    value = cells * args.steps * world / (ms / 1e3)

    # ---- end to end through the public API with host buffers: every step
    # uploads the state a host driver owns from pinned memory, iterates, and
    # reads the state back
    state = ("u", "v", "p", "T", "ro", "ue", "ve", "un", "vn", "Uce", "Vcn", "roe", "ron")
    pinned = {}
    for f in state:
        t = torch.empty(sim.nx * sim.ny, dtype=torch.float64, pin_memory=True)
        a = t.numpy()
        a[:] = sim.field(f)
        pinned[f] = (t, a)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    host = {f: pinned[f][1] for f in state}
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.set_fields(host)         # one copy per field from pinned memory, one synchronisation
        sim.iterate()
        sim.get_fields(host)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = cells * args.steps * world / e2e_s
    nbytes = len(state) * sim.nx * sim.ny * 8

    # ---- roofline of the dominant kernel: the MSI5 p' solve, re-run on the
    # instance's last p' system with CUDA events on the launching stream
    N = sim.nx * sim.ny
    dptr = ctypes.POINTER(ctypes.c_double)()
    n = ctypes.c_long()
    L.m2d_ctx_field_device.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                       ctypes.POINTER(ctypes.POINTER(ctypes.c_double)), ctypes.POINTER(ctypes.c_long)]
    check(L.m2d_ctx_field_device(sim._ctx, b"ap", ctypes.byref(dptr), ctypes.byref(n)))
    d_ap = ctypes.cast(dptr, ctypes.c_void_p).value
    check(L.m2d_ctx_field_device(sim._ctx, b"bp", ctypes.byref(dptr), ctypes.byref(n)))
    d_bp = ctypes.cast(dptr, ctypes.c_void_p).value
    L.m2d_msi_workspace_doubles.restype = ctypes.c_long
    wsz = L.m2d_msi_workspace_doubles(5, sim.nx, sim.ny)
    work = torch.empty(wsz, dtype=torch.float64, device=f"cuda:{local}")
    xk = torch.zeros(N, dtype=torch.float64, device=f"cuda:{local}")
    nit_d = torch.zeros(1, dtype=torch.int32, device=f"cuda:{local}")
    L.m2d_msi_solve_device.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 6
    ks = torch.cuda.Stream(device=f"cuda:{local}")
    reps = 20
    durs = []
    with torch.cuda.stream(ks):
        for k in range(reps + 3):
            xk.zero_()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(ks)
            check(L.m2d_msi_solve_device(5, sim.nx, sim.ny, 20, 1e-2, d_ap, d_bp, xk.data_ptr(),
                                         work.data_ptr(), ks.cuda_stream, nit_d.data_ptr()))
            a1.record(ks)
            if k >= 3:
                durs.append((a0, a1))
    torch.cuda.synchronize()
    avg_ms = sum(a.elapsed_time(b) for a, b in durs) / len(durs)
    nit = int(nit_d.item())
    # the same solve with the kernel's %globaltimer stamps: median duration
    # of each phase (CTA 0's view), after the timed region
    L.m2d_msi_solve_device_timed.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 7
    stamps = torch.zeros(7, dtype=torch.int64, device=f"cuda:{local}")
    ph = []
    with torch.cuda.stream(ks):
        for k in range(8):
            xk.zero_()
            check(L.m2d_msi_solve_device_timed(5, sim.nx, sim.ny, 20, 1e-2, d_ap, d_bp, xk.data_ptr(),
                                               work.data_ptr(), ks.cuda_stream, nit_d.data_ptr(),
                                               stamps.data_ptr()))
            ks.synchronize()
            t = stamps.cpu().tolist()
            if k >= 3:
                ph.append([(t[q + 1] - t[q]) / 1e3 for q in range(6)])
    names = ("factorisation", "initial_residual", "first_forward", "first_backward", "first_residual",
             "remaining_iterations")
    phases_us = {nm: sorted(col)[len(col) // 2] for nm, col in zip(names, zip(*ph))}
    alg = msi_algorithmic_bytes(5, N, nit)
    achieved = alg / (avg_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    # the whole outer iteration: the byte model with the device's own
    # iteration counts, over the device time of the timed steps
    step_bytes = sum(step_algorithmic_bytes(N, *c) for c in counts) / len(counts)
    step_gbs = step_bytes * world / (ms / args.steps / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "msi5_traffic.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("bytes_per_launch")
        except Exception:
            traffic = None

    batch = None
    if world == 1 and args.batch > 0:
        from mach2d_b200.simplec import Batch
        b = Batch([make_case(args.nxr, args.nyr) for _ in range(args.batch)], device=local)
        for inst in b.instances:
            inst.set_graph(True)       # every instance's captured iteration in flight at once
        b.iterate(max(1, args.warmup))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bsteps = max(3, args.steps // 2)
        b.iterate(bsteps)
        torch.cuda.synchronize()
        bdt = time.perf_counter() - t0
        bgbs = args.batch * bsteps * step_bytes / bdt / 1e9
        batch = {"instances": args.batch, "steps": bsteps,
                 "value": args.batch * bsteps * args.nxr * args.nyr / bdt, "unit": "cell-updates/s",
                 "roofline_step": {"achieved": bgbs, "peak": peak, "unit": "GB/s", "frac": bgbs / peak,
                                   "note": "the single instance's bytes per outer iteration x instances x steps "
                                           "/ wall time"},
                 "timing": "host wall clock around m2d_batch_iterate with device synchronisation",
                 "note": "independent instances of the same workload, one context and stream each, every "
                         "instance's captured iteration in flight at once"}
        b.close()

    extras = {}
    if not args.no_extras:
        extras["sweep256"] = run_sweep(local, n=256, iters=20, world=world, rank=rank)
    if world == 1 and not args.no_extras:
        extras.update(run_extras(args, local))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, nsamp, secs = cpu_sample(args, args.cpu_seconds, skip=args.warmup)
        cpu = {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "port",
               "sample": f"outer iterations {args.warmup + 1}..{args.warmup + nsamp} ({secs:.1f} s) of the same "
                         f"{args.nxr}x{args.nyr} case, serial C restatement of the reference"}
        va, nprocs, na = cpu_sample_all_cores(args, 10.0, skip=args.warmup)
        cpu["all_cores"] = {"value": va, "unit": "cell-updates/s", "cores": nprocs, "kind": "port",
                            "sample": f"{nprocs} processes, one per host core, each its own instance of the same "
                                      f"case ({na} iterations in about 10 s); reported baseline only"}

    if rank == 0:
        line = {
            "metric": "cell-updates/s (SIMPLEC outer iterations)", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded nozzle geometry, isentropic initial guess)",
            "config": workload_config(args, {"p_cycles_per_iteration": sum(itp) / len(itp),
                                             "iteration_launch": "host loop" if args.no_graph else "captured CUDA graph"}),
            "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes},
            "gpu_launches": launches,
            "roofline": {"kernel": "k_msi_c<5,1,4> (MSI5 factorisation + fb2d5 iterations, one cluster)",
                         "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_launch": alg,
                         "launch_ms": avg_ms, "iterations_per_launch": nit, "phases_us": phases_us,
                         "step": {"achieved": step_gbs, "peak": peak, "unit": "GB/s", "frac": step_gbs / peak,
                                  "bytes_per_step": step_bytes, "ms_per_step": ms / args.steps,
                                  "mean_counts": {k: sum(c[q] for c in counts) / len(counts) for q, k in
                                                  enumerate(("nit_u", "nit_v", "nit_p", "p_cycles"))},
                                  "model": f"{STEP_FIXED_B} B/cell + 2 MSI9 solves + p' cycles x "
                                           f"({P_CYCLE_B} B/cell + MSI5 solve), MSI solves as "
                                           "msi_algorithmic_bytes, N = nx*ny with the ghost ring"}},
            "cpu_baseline": cpu,
            "batch": batch,
            "clocks": clk.summary(),
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_extras(args, local):
    """Secondary figures, each on one GPU: the same workload with FP32 sweeps;
    the time to the stopping residual of the 80x40 Euler nozzle (FP64, FP32
    sweeps, and the serial oracle extrapolated from a sample); and what the
    learned p' correction gains on this workload's p' systems."""
    import numpy as np
    import torch

    from mach2d_b200 import unet
    from mach2d_b200.simplec import Simplec, euler_cosine_case
    out = {}
    dev = torch.device("cuda", local)

    # FP32 factors and sweeps inside the FP64 iteration (solver 2)
    g = Simplec(euler_cosine_case(args.nxr, args.nyr, solver=2), device=local)
    g.set_graph(True)
    for _ in range(args.warmup):
        g.iterate()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.iterate()
    torch.cuda.synchronize()
    s32 = time.perf_counter() - t0
    out["fp32_sweeps"] = {"value": args.nxr * args.nyr * args.steps / s32, "unit": "cell-updates/s",
                          "ms_per_step": 1e3 * s32 / args.steps,
                          "timing": "host clock around the iterations (each ends in a read-back)",
                          "note": "solver 2: MSI factors and sweeps in FP32 inside the FP64 iteration"}
    g.close()

    # time to the stopping residual (normpl < 1e-10 first at it, stop at 2 it) of the 80x40 nozzle
    ttr = {"case": "C01 Euler 80x40, tolt 1e-10, SCARBOROUGH", "metric": "seconds to the stopping iteration"}
    fin = json.load(open(os.path.join(ROOT, "tests", "golden", "bench_workloads.json")))["c01_euler_80x40_converged"][
        "final"]
    for solver, key, lag in ((0, "gpu_fp64", 0), (2, "gpu_fp32_sweeps", 0), (2, "gpu_fp32_lagged_factors", 32)):
        g = Simplec(euler_cosine_case(80, 40, solver=solver, msi_lag=lag), device=local)
        g.set_graph(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rep = g.run(200000)
        torch.cuda.synchronize()
        fmi, fme, Fd, Cd, pw = g.integrals()
        pr = np.asarray(fin["pwall"])
        ttr[key] = {"seconds": time.perf_counter() - t0, "iterations": rep.it, "normpl": rep.normpl, "Cd": Cd,
                    "msi_lag": lag,
                    "rel_err_vs_oracle": {"Cd": abs(Cd - fin["Cd"]) / abs(fin["Cd"]),
                                          "fmi": abs(fmi - fin["fmi"]) / abs(fin["fmi"]),
                                          "fme": abs(fme - fin["fme"]) / abs(fin["fme"]),
                                          "Fd": abs(Fd - fin["Fd"]) / abs(fin["Fd"]),
                                          "pwall_max": float(np.max(np.abs(pw - pr)) / np.max(np.abs(pr)))}}
        g.close()
    ttr["oracle_converged"] = {"iterations": fin["it"], "Cd": fin["Cd"],
                               "fixture": "tests/golden/bench_workloads.json (make_bench_golden.py)"}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _oracle import OracleCase
    o = OracleCase(euler_cosine_case(80, 40))
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < 3.0:
        o.iterate()
        n += 1
    per = (time.perf_counter() - t0) / n
    it_gpu = ttr["gpu_fp64"]["iterations"]
    ttr["cpu_oracle_serial"] = {"seconds": per * it_gpu, "iterations": it_gpu, "cores": 1,
                                "sample": f"extrapolated from {n} iterations of the serial C restatement"}
    out["time_to_residual"] = ttr

    # learned p' correction on this workload's p' systems
    g = Simplec(make_case(args.nxr, args.nyr), device=local)
    nx, ny = g.nx, g.ny
    H, W = unet.image_shape(nx, ny)
    pairs = unet.PairSet(48, H, W, device=local)
    held = []
    for _ in range(3):
        g.iterate()
    unet.harvest(g, pairs, iters_between=2, count=40)
    hp = unet.PairSet(8, H, W, device=local)
    unet.harvest(g, hp, iters_between=3, count=8, held_out=held)
    Jp = torch.from_numpy(g.field("Jp")).to(dev)
    g.close()
    net = unet.UNet(8, H, W, device=local, seed=1)
    t0 = time.perf_counter()
    hist = unet.train(net, pairs, 300, batch=8, lr=2e-3, lr_final=1e-4)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    one = unet.UNet(1, H, W, device=local, params=net.params())
    net.close()
    Lb = unet._bind()
    work = torch.empty(Lb.m2d_msi_workspace_doubles(5, nx, ny), dtype=torch.float64, device=dev)
    nit = torch.zeros(2, dtype=torch.int32, device=dev)
    res = {"msi_fp64": [], "msi_fp32": [], "learned_fp32": []}
    nits = {"msi_fp64": [], "msi_fp32": [], "learned_fp32": []}
    ratio = []
    for a, b in held:
        for key, prec in (("msi_fp64", 0), ("msi_fp32", 1)):
            x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            unet.msi5(nx, ny, 20, 1e-2, a, b, x, work, nit, prec=prec)
            torch.cuda.synchronize()
            res[key].append(time.perf_counter() - t0)
            nits[key].append(int(nit[0].item()))
        x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = one.solve(nx, ny, 20, 1e-2, a, b, x, Jp, work, prec=1)
        torch.cuda.synchronize()
        res["learned_fp32"].append(time.perf_counter() - t0)
        nits["learned_fp32"].append(r.nit)
        ratio.append(r.r1 / r.r0)
    if args.ttr_cap > 0:
        out["time_to_residual_512x256"] = run_ttr512(local, one, args.ttr_cap)
    one.close()
    out["isolated_system"] = run_isolated(local)
    out["krylov"] = run_krylov(local)
    out["config3"] = run_config3(args, local)
    out["learned"] = {
        "train": {"pairs": pairs.n, "steps": 300, "batch": 8, "seconds": train_s, "loss_first": hist[0],
                  "loss_last50": float(np.mean(hist[-50:]))},
        "held_out_systems": len(held),
        "residual_after_correction_median": float(np.median(ratio)),
        "p_solve_ms_median": {k: 1e3 * float(np.median(v)) for k, v in res.items()},
        "msi_iterations_mean": {k: float(np.mean(v)) for k, v in nits.items()},
        "tolerance": "p' solve to |r| < 1e-2 |r0| (nitm_p = 20), host clock per solve"}
    return out


def config3_case(solver):
    """The turbulent 512x256 case: C01 nozzle, Navier-Stokes, MIXTURE air,
    Baldwin-Lomax eddy viscosity (Pr_t 0.9), geometric wall clustering with a
    1e-6 m first cell, p0 = 2 MPa, T0 = 1500 K, adiabatic wall."""
    from mach2d_b200.simplec import euler_cosine_case
    from mach2d_b200.thermo import mixture_init
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "air_species.json")))
    mix = mixture_init(d["base"], d["fractions"], d["Mi"], d["cpi"], d["mui"], d["kpi"])
    return euler_cosine_case(512, 256, modvis=1, kg=2, a1=1e-6, p0=2e6, T0=1500.0, Twall=-1.0, ktm=1, mix=mix,
                             solver=solver, modtur=1, prt=0.9)


def run_config3(args, local, warm=5, steps=20):
    """Throughput of the turbulent 512x256 case over outer iterations
    warm+1 .. warm+steps (FP64 MSI, and FP32 sweeps), device time of the
    captured iterations, and the serial oracle on the same iterations."""
    import torch

    from mach2d_b200.simplec import Simplec
    out = {"case": "C01 512x256 Navier-Stokes + MIXTURE air + Baldwin-Lomax (Pr_t 0.9), first cell 1e-6 m, "
                   "p0 2 MPa, T0 1500 K, adiabatic wall", "iterations_timed": [warm + 1, warm + steps]}
    cells = 512 * 256
    for solver, key in ((0, "gpu_fp64"), (2, "gpu_fp32_sweeps")):
        g = Simplec(config3_case(solver), device=local)
        g.set_graph(True)
        for _ in range(warm):
            g.iterate()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            r = g.iterate()
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        out[key] = {"value": cells * steps / secs, "unit": "cell-updates/s", "ms_per_step": 1e3 * secs / steps,
                    "normpl_last": r.normpl}
        g.close()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _oracle import OracleCase
    o = OracleCase(config3_case(0))
    for _ in range(warm):
        o.iterate()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.iterate()
    secs = time.perf_counter() - t0
    out["cpu_oracle_serial"] = {"value": cells * steps / secs, "unit": "cell-updates/s", "cores": 1,
                                "ms_per_step": 1e3 * secs / steps}
    out["note"] = ("host clock around iterations that each end in a read-back; the run stops with a NaN at "
                   "iteration 982 in both implementations (tests/test_gpu_ns512.py), so no time to a residual "
                   "of 1e-8 exists for this case")
    return out


def run_ttr512(local, net, cap_s, tol=1e-8):
    """Time to the outer residual normpl < 1e-8 (src/mach2d_main.f90:307) of
    the C01 Euler nozzle at 512x256 (the turbulent Navier-Stokes case of this
    size stops with a NaN in both implementations, so the same-size Euler
    nozzle stands in for it), from the initial guess: plain FP64 MSI, FP32
    factors and sweeps, and FP32 with lagged factors (msi_lag = 32: factors
    reused while one iteration meets the tolerance), each iteration one
    captured graph; and the learned p' correction with FP32 sweeps (solver
    3, the network trained on this workload's p' systems, msi_lag = 32 for
    the u and v solves; host-driven iterations).  Each run is capped at
    cap_s seconds.  Integrals at the first iteration below 1e-8 are compared
    with the FP64 oracle's at its own first such iteration
    (tests/golden/ttr512_c01_euler.json, make_ttr512_golden.py)."""
    import numpy as np
    import torch

    from mach2d_b200.simplec import Simplec, euler_cosine_case
    ref = None
    fx = os.path.join(ROOT, "tests", "golden", "ttr512_c01_euler.json")
    if os.path.exists(fx):
        ref = json.load(open(fx)).get("first_below")
    out = {"case": "C01 Euler 512x256, tolt 1e-8, SCARBOROUGH; stands in for the 512x256 Navier-Stokes case, "
                   "which stops with a NaN (both implementations)",
           "cap_s": cap_s, "oracle_first_below_it": ref["it"] if ref else None}
    for key, solver, lag in (("plain_fp64", 0, 0), ("fp32_sweeps", 2, 0), ("fp32_lagged_factors", 2, 32),
                             ("learned_fp32", 3, 32)):
        g = Simplec(euler_cosine_case(512, 256, solver=solver, tolt=tol, msi_lag=lag), device=local)
        if solver >= 3:
            g.set_unet(net)
        else:
            g.set_graph(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r, reached = None, False
        while time.perf_counter() - t0 < cap_s:
            r = g.iterate()
            if r.normpl < tol:
                reached = True
                break
        secs = time.perf_counter() - t0
        fmi, fme, Fd, Cd, pw = g.integrals()
        e = {"seconds": secs, "iterations": r.it, "reached": reached, "normpl": r.normpl, "Cd": Cd,
             "ms_per_iteration": 1e3 * secs / r.it, "msi_lag": lag}
        if solver >= 3:
            e["learned_calls"] = g.scalar("learned_calls")
            e["learned_accepted"] = g.scalar("learned_accepted")
            e["learned_alone"] = g.scalar("learned_alone")
        if ref and reached:
            pr = np.asarray(ref["pwall"])
            e["rel_err_vs_oracle"] = {"Cd": abs(Cd - ref["Cd"]) / abs(ref["Cd"]),
                                      "fmi": abs(fmi - ref["fmi"]) / abs(ref["fmi"]),
                                      "fme": abs(fme - ref["fme"]) / abs(ref["fme"]),
                                      "Fd": abs(Fd - ref["Fd"]) / abs(ref["Fd"]),
                                      "pwall_max": float(np.max(np.abs(pw - pr)) / np.max(np.abs(pr)))}
        out[key] = e
        g.close()
    p = out["plain_fp64"]
    for key in ("fp32_sweeps", "fp32_lagged_factors", "learned_fp32"):
        q = out[key]
        if p["reached"] and q["reached"]:
            out[f"speedup_{key}_vs_plain_fp64"] = p["seconds"] / q["seconds"]
    return out


def isolated_system9(nx, ny, seed=1, dominance=1.05):
    """The isolated 9-diagonal system: off-diagonals i.i.d. U[-1, 0], aP =
    1.05 sum|a_nb|, rhs N(0, 1), a zero-Dirichlet ghost ring (ghost rows aP =
    1, b = 0; couplings into the ring dropped).  Plane-major, reference order."""
    import numpy as np
    rng = np.random.default_rng(seed)
    off = [(-1, -1), (0, -1), (1, -1), (-1, 0), (0, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]
    inner = np.zeros((ny, nx), bool)
    inner[1:-1, 1:-1] = True
    a = np.zeros((9, ny, nx))
    for k, (di, dj) in enumerate(off):
        if k == 4:
            continue
        nb = np.zeros((ny, nx), bool)        # neighbour (i + di, j + dj) is a real cell
        nb[max(0, -dj):ny - max(0, dj), max(0, -di):nx - max(0, di)] = \
            inner[max(0, dj):ny - max(0, -dj), max(0, di):nx - max(0, -di)]
        a[k] = np.where(inner & nb, -rng.uniform(0.0, 1.0, (ny, nx)), 0.0)
    a[4] = np.where(inner, dominance * np.abs(a).sum(axis=0), 1.0)
    b = np.where(inner, rng.standard_normal((ny, nx)), 0.0)
    return a.reshape(-1).copy(), b.reshape(-1).copy()


def isolated_system5(nx, ny, seed=1, dominance=1.05):
    """The 5-diagonal analogue of the isolated system (the p' system's
    stencil): the S, W, E, N couplings of isolated_system9 with aP = 1.05
    sum|a_nb| of those four."""
    import numpy as np
    a9, b = isolated_system9(nx, ny, seed, dominance)
    N = nx * ny
    a = a9.reshape(9, N)[[1, 3, 4, 5, 7]].copy()
    inner = np.zeros((ny, nx), bool)
    inner[1:-1, 1:-1] = True
    a[2] = np.where(inner.ravel(), dominance * np.abs(a[[0, 1, 3, 4]]).sum(axis=0), 1.0)
    return a.reshape(-1).copy(), b


def _timed(fn, reps=2):
    """Host time of the last of `reps` calls of fn() (each synchronising)."""
    import torch
    out = None
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
    return 1e3 * secs, out


def run_krylov(local, nx=1026, ny=514, tol=1e-12, train_systems=48, train_steps=1000):
    """Flexible GMRES (m2d_fgmres_solve) against MSI iterated alone on the
    isolated systems at 1024x512 real cells: the 9-diagonal one with the MSI
    factorisation as preconditioner (FP64, FP32), and the 5-diagonal one also
    with the learned correction followed by one FP32 MSI step as the
    preconditioner; the network is trained here, by the library's kernels,
    on the MSI solutions of `train_systems` other seeds of the same system."""
    import ctypes

    import numpy as np
    import torch

    from mach2d_b200 import unet
    from mach2d_b200._lib import check, lib
    from mach2d_b200.solvers import fgmres
    dev = torch.device("cuda", local)
    L = lib()
    L.m2d_msi_workspace_doubles.restype = ctypes.c_long
    L.m2d_msi_workspace_doubles.argtypes = [ctypes.c_int] * 3
    for fn in ("m2d_msi_solve_device", "m2d_msi_solve_device_mixed"):
        getattr(L, fn).argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 6
    out = {"tolerance": tol, "metric": "host ms per solve to |b - A x| <= tol |b| from x = 0, restart 30"}
    Jp = torch.ones(nx * ny, dtype=torch.float64, device=dev)
    one = None
    for nd in (9, 5):
        a, b = isolated_system9(nx, ny) if nd == 9 else isolated_system5(nx, ny)
        da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        ws = torch.empty(L.m2d_msi_workspace_doubles(nd, nx, ny), dtype=torch.float64, device=dev)
        nit = torch.zeros(2, dtype=torch.int32, device=dev)
        e = {"system": f"{nd}-diagonal {nx - 2}x{ny - 2}, aP = 1.05 sum|a_nb|, seed 1"}
        for key, fn in (("msi_fp64", "m2d_msi_solve_device"), ("msi_fp32_refined", "m2d_msi_solve_device_mixed")):
            def run(fn=fn):
                x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
                check(getattr(L, fn)(nd, nx, ny, 5000, tol, da.data_ptr(), db.data_ptr(), x.data_ptr(),
                                     ws.data_ptr(), None, nit.data_ptr()))
            ms, _ = _timed(run)
            e[key] = {"ms": ms, "msi_iterations": int(nit[0].item())}
        if nd == 5:
            H, W = unet.image_shape(nx, ny)
            systems = []
            for sd in range(100, 100 + train_systems):
                a_t, b_t = isolated_system5(nx, ny, sd)
                systems.append((torch.from_numpy(a_t).to(dev), torch.from_numpy(b_t).to(dev)))
            pairs = unet.PairSet(len(systems), H, W, device=local)
            unet.harvest_systems(systems, nx, ny, Jp, pairs)
            del systems
            net = unet.UNet(8, H, W, device=local, seed=1)
            t0 = time.perf_counter()
            hist = unet.train(net, pairs, train_steps, batch=8, lr=2e-3, lr_final=1e-4)
            torch.cuda.synchronize()
            e["learned_training"] = {"systems": pairs.n, "steps": train_steps, "seconds": time.perf_counter() - t0,
                                     "loss_first": hist[0], "loss_last50": float(np.mean(hist[-50:]))}
            one = unet.UNet(1, H, W, device=local, params=net.params())
            net.close()
            del pairs
        for key, prec in (("fgmres_msi_fp64", 0), ("fgmres_msi_fp32", 1), ("fgmres_learned_fp32", 2)):
            if prec == 2 and nd != 5:
                continue

            def run(prec=prec):
                x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
                return fgmres(nd, nx, ny, da, db, x, tol, prec=prec, restart=30, net=one if prec == 2 else None,
                              Jp=Jp if prec == 2 else None)
            ms, r = _timed(run)
            e[key] = {"ms": ms, "krylov_steps": r.iterations, "msi_applications": r.msi_applications,
                      "learned_applications": r.learned_applications, "relative_residual": r.rel_residual}
        base = e["msi_fp64"]["ms"]
        e["speedup_vs_msi_fp64"] = {k: base / e[k]["ms"] for k in e if k.startswith("fgmres")}
        out[f"nd{nd}"] = e
    if one is not None:
        one.close()
    return out


def run_isolated(local, nx=1026, ny=514, tol=1e-12):
    """MSI on the isolated 1024x512 system to a relative residual of 1e-12:
    FP64 and FP32 factors and sweeps inside the FP64 iteration on the GPU
    (device time of the solve launch), and the serial oracle."""
    import ctypes

    import numpy as np
    import torch

    from mach2d_b200._lib import check, lib
    a, b = isolated_system9(nx, ny)
    dev = torch.device("cuda", local)
    L = lib()
    L.m2d_msi_workspace_doubles.restype = ctypes.c_long
    L.m2d_msi_workspace_doubles.argtypes = [ctypes.c_int] * 3
    wsz = L.m2d_msi_workspace_doubles(9, nx, ny)
    da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    work = torch.empty(wsz, dtype=torch.float64, device=dev)
    nit = torch.zeros(2, dtype=torch.int32, device=dev)
    out = {"system": f"9-diagonal {nx - 2}x{ny - 2} (+ghost ring), aP = 1.05 sum|a_nb|, seed 1",
           "tolerance": tol}
    for key, fn in (("gpu_fp64", "m2d_msi_solve_device"), ("gpu_fp32_refined", "m2d_msi_solve_device_mixed")):
        f = getattr(L, fn)
        f.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 6
        times = []
        for rep in range(3):
            x = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            check(f(9, nx, ny, 5000, tol, da.data_ptr(), db.data_ptr(), x.data_ptr(), work.data_ptr(), None,
                    nit.data_ptr()))
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        rr = work[wsz - 4:wsz - 2].cpu().numpy()
        out[key] = {"ms": min(times), "iterations": int(nit[0].item()),
                    "relative_residual": float(np.sqrt(rr[1] / rr[0]))}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _oracle import call
    x = np.zeros(nx * ny)
    t0 = time.perf_counter()
    its = call("msi9_solve", nx, ny, 5000, tol, a, b, x)
    out["cpu_oracle_serial"] = {"ms": 1e3 * (time.perf_counter() - t0), "iterations": int(its), "cores": 1}
    # 512 independent tridiagonal lines of 1024 unknowns, aP = 1.05 (|aW| + |aE|)
    from mach2d_b200.solvers import tdma_lines
    rng = np.random.default_rng(2)
    nl, n = 512, 1024
    aw, ae = -rng.uniform(0, 1, (nl, n)), -rng.uniform(0, 1, (nl, n))
    aw[:, 0] = 0.0
    ae[:, -1] = 0.0
    ap = 1.05 * (np.abs(aw) + np.abs(ae))
    d = rng.standard_normal((nl, n))
    tdma_lines(aw, ap, ae, d)
    t0 = time.perf_counter()
    xg = tdma_lines(aw, ap, ae, d)
    tg = time.perf_counter() - t0
    xo = np.zeros(n)
    t0 = time.perf_counter()
    err = 0.0
    for k in range(nl):
        call("tdma_line", n, np.ascontiguousarray(aw[k]), np.ascontiguousarray(ap[k]), np.ascontiguousarray(ae[k]),
             np.ascontiguousarray(d[k]), xo)
        err = max(err, float(np.max(np.abs(xo - xg[k]))))
    cpu_ms = 1e3 * (time.perf_counter() - t0)
    # device time of the kernels themselves (CUDA events, inputs resident):
    # method 0 the sequential recurrence (bitwise), method 1 cyclic reduction;
    # algorithmic bytes 40 per unknown (aw, ap, ae, d in, x out)
    L.m2d_tdma_lines_device.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 6 + [ctypes.c_int,
                                                                                                ctypes.c_void_p]
    tl = [torch.from_numpy(np.ascontiguousarray(v)).to(dev) for v in (aw, ap, ae, d)]
    xw = torch.empty(2 * n * nl, dtype=torch.float64, device=dev)
    xd = torch.zeros(nl, n, dtype=torch.float64, device=dev)
    peak, peak_kind = peaks()
    dev_ms, diff = {}, {}
    for method, key in ((0, "recurrence"), (1, "cyclic_reduction")):
        ts = []
        for rep in range(8):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            check(L.m2d_tdma_lines_device(n, nl, *[v.data_ptr() for v in tl], xd.data_ptr(), xw.data_ptr(), method,
                                          None))
            e1.record()
            torch.cuda.synchronize()
            if rep >= 3:
                ts.append(e0.elapsed_time(e1))
        dev_ms[key] = min(ts)
        diff[key] = float(np.max(np.abs(xd.cpu().numpy() - xg)) / np.max(np.abs(xg)))
    alg = 40.0 * n * nl
    out["tdma_lines"] = {"lines": nl, "n": n, "gpu_host_api_ms": 1e3 * tg, "cpu_oracle_serial_ms": cpu_ms,
                         "max_abs_difference": err,
                         "gpu_device_ms": dev_ms,
                         "relative_difference_to_recurrence": diff,
                         "roofline": {k: {"achieved_gbs": alg / (v / 1e3) / 1e9, "frac": alg / (v / 1e3) / 1e9 / peak,
                                          "peak_gbs": peak, "peak_source": peak_kind} for k, v in dev_ms.items()},
                         "algorithmic_bytes": alg,
                         "note": "gpu_host_api_ms: the host call m2d_tdma_lines, copies in and out included; "
                                 "gpu_device_ms: the kernel alone on resident inputs (best of 5 after 3 warm-ups)"}
    return out


def sweep_cases(n, seed=2024):
    """The batched sweep: n Euler nozzles drawn from the seed, nx in 64..512,
    ny in 32..128, Rin in [1.5, 2.5], Rout in [1.3, 2.2], Lc in [1, 3],
    Ld in [2, 6], p0 in [5e5, 3e6] Pa, T0 in [600, 1500] K; FP32 sweeps."""
    import numpy as np

    from mach2d_b200.simplec import euler_cosine_case
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(n):
        cases.append(euler_cosine_case(int(rng.integers(64, 513)), int(rng.integers(32, 129)),
                                       Rin=rng.uniform(1.5, 2.5), Rout=rng.uniform(1.3, 2.2), Lc=rng.uniform(1, 3),
                                       Ld=rng.uniform(2, 6), p0=rng.uniform(5e5, 3e6), T0=rng.uniform(600, 1500),
                                       solver=2))
    return cases


def run_sweep(local, n, iters, world=1, rank=0):
    """The sweep sharded over the ranks (mach2d_b200.sweep): each rank runs its
    share (balanced by cells) as one batch; time = max over ranks; results
    gathered in the sweep's order."""
    import torch

    from mach2d_b200.sweep import gather_results, run_shard, shard_indices
    cases = sweep_cases(n)
    parts = shard_indices([c.nxr * c.nyr for c in cases], world)
    mine = parts[rank]
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    tm = {}
    res, secs = run_shard(cases, mine, local, iters, timings=tm, tune=2)
    setup = tm["setup_s"]
    if world > 1:
        t = torch.tensor([secs, setup], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        secs, setup = float(t[0].item()), float(t[1].item())
    allres = gather_results(res, n)
    cells = sum(c.nxr * c.nyr for c in cases)
    cds = [r[5] for r in allres]
    return {"instances": n, "iterations": iters, "value": cells * iters / secs, "unit": "cell-updates/s",
            "real_cells": cells, "ranks": world, "scaling": "strong", "seconds_max_over_ranks": secs,
            "setup_seconds_max_over_ranks": setup,
            "Cd_mean_after": sum(cds) / len(cds),
            "msi_schedule": tm.get("schedule"),
            "note": "independent Euler nozzles of the seeded sweep distribution sharded over the ranks by cells, "
                    "FP32 sweeps, one captured graph per instance iteration with every instance's graph in flight "
                    "at once; the MSI schedule autotuned on the batch's first iterations (rank 0's choice shown), "
                    "then the timed iterations; batch set-up (grids, metrics and initial fields on the device) "
                    "timed apart"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
