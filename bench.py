"""Benchmark: full FSD time steps per second at N=32768, phi=0.4.

Workload (one "step"): neighbour list, preconditioner build, pair forces,
far-field Brownian slip (wave-space noise + Lanczos on the real-space
mobility), near-field Brownian force (Lanczos on R_FU), random finite
difference drift (two saddle solves), main saddle solve to relative residual
1e-4 (warm-started), Euler update with simple shear 1.0.  kT = 1, dt = 1e-4,
Ewald accuracy 1e-3 (xi 0.5, 72^3 grid, P = 6).  Positions from seeded random
sequential addition followed by overlap relaxation.

The timed preconditioner is the learned one by default (two-hop sparse
approximate inverse of the lubrication block, inner GMRES steps, flexible outer
GMRES, and the trained network's correction when fsd_b200/data holds
weights); the same steps with the plain IChol preconditioner are timed after
it for the metric's comparison ("ichol" in the JSON line).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fsd|reference]
                  [--precond learned|ichol|none] [--inner k] [--no-ichol] [--no-net]

Under torchrun each rank steps its own independent suspension (the path does
not shard within one suspension; replicas only).  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FSD steps/sec at N=32768 φ=0.4, learned-precond vs IChol at 1e-4 residual"
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fsd", choices=["fsd", "reference"])
    ap.add_argument("--N", type=int, default=32768)
    ap.add_argument("--phi", type=float, default=0.4)
    ap.add_argument("--precond", default="learned", choices=["ichol", "none", "learned"])
    ap.add_argument("--inner", type=int, default=6, help="inner GMRES steps of the learned preconditioner")
    ap.add_argument("--no-ichol", action="store_true", help="skip the IChol comparison run")
    ap.add_argument("--no-net", action="store_true", help="learned preconditioner without the network correction")
    ap.add_argument("--no-autotune", action="store_true", help="fixed spreading tiles and FFT batches")
    ap.add_argument("--replicas", type=int, default=0,
                    help="batched-replica mode: this many independent suspensions, N log-uniform in [500, 8000], "
                         "phi uniform in [0.1, 0.5], shear rate uniform in [0, 2], stepped concurrently and then "
                         "one by one (prints its own JSON line)")
    ap.add_argument("--ichol-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-sample-seconds", type=float, default=20.0)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        rows = [l.split(",") for l in Path(self.out.name).read_text().splitlines() if l.strip()]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if len(r) > 2 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 2 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def peak_hbm():
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def region_bytes(name, N, G, pairs_real, pairs_lub):
    """Algorithmic DRAM bytes of one launch of a single-kernel region: each
    array the kernel must read or write once."""
    if name == "fft":
        return 2 * 6 * G * 8  # y+z plane pass over the 6 packed complex grids, read + write once
    if name == "spread":
        return N * (16 + 48) + 6 * G * 8
    if name == "contract":
        return 6 * G * 8 + N * (16 + 44)
    if name == "green":
        return 2 * 6 * G * 8 + G * 16
    if name == "real_space":
        return N * (16 + 16 + 32) + 4 * pairs_real + N * 44
    if name == "rfu":
        return N * (16 + 24 + 24) + 4 * pairs_lub
    return None


# Launches per region entry: on the 72^3 grid each FFT region (z+y forward or
# y+z inverse) is one plane-kernel launch, and the x pass with the Green step
# is one launch.
SINGLE_KERNEL_REGIONS = {"fft": 1, "spread": 1, "contract": 1, "green": 1, "real_space": 1, "rfu": 1}
WEIGHTS = ROOT / "fsd_b200" / "data" / "learned_precond.f32"


def make_solver(args, precond, N, L, dev, seed):
    from fsd_b200.core import FSD

    s = FSD(N, (L, L, L, 0.0), device=dev, T=1.0, dt=1e-4, seed=seed, error=1e-3, solver_tol=1e-4,
            lanczos_tol=1e-3, rfd_epsilon=1e-3, precond=precond, period=0, gmres_max_iter=3000,
            gmres_restart=200 if precond == "ichol" else 100, learned_inner=args.inner if precond == "learned" else 0,
            autotune=0 if args.no_autotune else 1)
    net = False
    if precond == "learned" and WEIGHTS.exists() and not args.no_net:
        s.learned_set_weights(np.fromfile(WEIGHTS, "<f4"))
        net = True
    return s, net


def timed_steps(args, s, state, steps, warmup, dev, ws, clocks=False, profile=False):
    """Warm-up, then `steps` steps each bracketed by CUDA events on the launching
    stream with a 256 MiB L2 flush before it (outside the events)."""
    import torch

    from fsd_b200 import _lib

    p, ori, img, F, V, step_no = state
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def one_step():
        st = s.step(step_no[0], 1.0, p, ori, img, F, V, raise_on_error=False)
        step_no[0] += 1
        if st not in (0, 4):  # Lanczos not converged (4) is reported, not fatal, as in the reference
            raise RuntimeError(f"fsd_step status {st}")

    for _ in range(warmup):
        one_step()
    lib = _lib.lib()
    nreg = len(_lib.REGIONS)
    ms_regions = np.zeros(nreg)
    cnt_regions = np.zeros(nreg, np.int64)
    if profile:
        lib.fsd_profile_enable(s._h, 1)
        lib.fsd_profile_read(s._h, ms_regions.ctypes.data_as(C.c_void_p), cnt_regions.ctypes.data_as(C.c_void_p),
                             nreg, 1)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    iters = []
    torch.cuda.synchronize(dev)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    launch0 = lib.fsd_launch_count()
    clk = ClockSampler(dev.index) if clocks else None
    if clk:
        clk.__enter__()
    for k in range(steps):
        flush.fill_(float(k))
        evs[k][0].record(stream)
        one_step()
        evs[k][1].record(stream)
        si = s.solve_info()
        iters.append(si["gmres_iters"] + [si["lanczos_ff_iters"], si["lanczos_nf_iters"]])
    torch.cuda.synchronize(dev)
    if clk:
        clk.__exit__()
    launches = lib.fsd_launch_count() - launch0
    if ws > 1:
        torch.distributed.barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = float(sum(step_ms))
    if ws > 1:
        t = torch.tensor([total_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    regions = None
    if profile:
        lib.fsd_profile_read(s._h, ms_regions.ctypes.data_as(C.c_void_p), cnt_regions.ctypes.data_as(C.c_void_p),
                             nreg, 1)
        lib.fsd_profile_enable(s._h, 0)
        regions = {n: {"ms": float(ms_regions[i]), "calls": int(cnt_regions[i])} for i, n in enumerate(_lib.REGIONS)}
    it = np.array(iters, np.float64)
    iters_out = {"gmres_rfd_plus": float(it[:, 0].mean()), "gmres_rfd_minus": float(it[:, 1].mean()),
                 "gmres_main": float(it[:, 2].mean()), "lanczos_ff": float(it[:, 3].mean()),
                 "lanczos_nf": float(it[:, 4].mean())}
    return {"total_ms": total_ms, "step_ms": step_ms, "iters": iters_out, "launches": int(launches),
            "regions": regions, "clocks": clk.summary() if clk else None}


def run_fsd(args, ws, rank, local):
    import torch

    from fsd_b200.configs import suspension

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    N, phi = args.N, args.phi
    pos, L = suspension(N, phi, seed=1 + rank)

    def fresh_state():
        p = torch.as_tensor(pos, device=dev).view(-1).contiguous()
        ori = torch.as_tensor(np.tile([0.0, 0.0, 1.0], N).astype(np.float32), device=dev).contiguous()
        img = torch.zeros(3 * N, dtype=torch.int32, device=dev)
        F = torch.zeros(6 * N, device=dev)
        V = torch.zeros(11 * N, device=dev)
        return [p, ori, img, F, V, [0]]

    s, net = make_solver(args, args.precond, N, L, dev, 1 + rank)
    info = s.pse_info()
    state = fresh_state()
    main = timed_steps(args, s, state, args.steps, args.warmup, dev, ws, clocks=True, profile=True)
    value = ws * args.steps / (main["total_ms"] / 1e3)
    # --- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        p, ori, img, F, V, step_no = state
        stream = torch.cuda.current_stream(dev)
        pin = lambda t: t.detach().cpu().pin_memory()
        h_pos, h_ori, h_img = pin(p), pin(ori), pin(img)
        h_V, h_P = torch.empty(11 * N).pin_memory(), torch.empty(4 * N).pin_memory()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for k in range(args.steps):
            p.copy_(h_pos, non_blocking=True)
            ori.copy_(h_ori, non_blocking=True)
            img.copy_(h_img, non_blocking=True)
            st = s.step(step_no[0], 1.0, p, ori, img, F, V, raise_on_error=False)
            step_no[0] += 1
            if st not in (0, 4):
                raise RuntimeError(f"fsd_step status {st}")
            h_V.copy_(V, non_blocking=True)
            h_P.copy_(p, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = e0.elapsed_time(e1)
        if ws > 1:
            t = torch.tensor([e2e_ms], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": ws * args.steps / (e2e_ms / 1e3), "unit": "steps/s",
               "h2d_bytes_per_step": int(h_pos.numel() * 4 + h_ori.numel() * 4 + h_img.numel() * 4),
               "d2h_bytes_per_step": int(h_V.numel() * 4 + h_P.numel() * 4)}
    s.close()
    # --- the same step with the plain IChol preconditioner (the metric's comparison)
    ichol = None
    if not args.no_ichol and args.precond != "ichol":
        si, _ = make_solver(args, "ichol", N, L, dev, 1 + rank)
        r = timed_steps(args, si, fresh_state(), args.ichol_steps, 1, dev, ws)
        si.close()
        ichol = {"value": ws * args.ichol_steps / (r["total_ms"] / 1e3), "unit": "steps/s",
                 "ms_per_step": r["total_ms"] / args.ichol_steps, "steps": args.ichol_steps, "warmup": 1,
                 "iterations_per_step": r["iters"]}
    # --- roofline of the dominant single-kernel region
    regions = main["regions"]
    G = info.Nx * info.Ny * info.Nz
    cands = {n: r for n, r in regions.items() if n in SINGLE_KERNEL_REGIONS and r["calls"] > 0}
    dom = max(cands, key=lambda n: cands[n]["ms"])
    avg_launch_ms = cands[dom]["ms"] / cands[dom]["calls"] / SINGLE_KERNEL_REGIONS[dom]
    nb = region_bytes(dom, N, G, pairs_real=int(N * 60), pairs_lub=int(N * 75))
    peak, peak_kind = peak_hbm()
    achieved = nb / (avg_launch_ms * 1e-3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "dram_traffic.json"
    if tf.exists():
        traffic = json.loads(tf.read_text()).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "avg_launch_us": avg_launch_ms * 1e3,
                "algorithmic_bytes_per_launch": nb}
    out = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 Krylov/Lanczos scalars, IC pivots, SPAI solves)",
        "data": "synthetic: seeded random sequential addition + overlap relaxation, min gap 1e-3",
        "config": {"workload": f"full FSD step, N={N}, phi={phi}, shear 1.0, kT 1, dt 1e-4, Ewald 1e-3, "
                               f"GMRES 1e-4, {args.precond} preconditioner", "N": N, "phi": phi,
                   "grid": [info.Nx, info.Ny, info.Nz], "P": info.P, "precond": args.precond,
                   "learned_inner": args.inner if args.precond == "learned" else None, "learned_network": net,
                   "autotune": not args.no_autotune,
                   "gmres_tol": 1e-4, "ewald_error": 1e-3, "l2": "flushed before every timed step (256 MiB write)",
                   "parallelism": f"replicas x{ws}"},
        "e2e": e2e, "gpu_launches": main["launches"], "roofline": roofline,
        "iterations_per_step": main["iters"],
        "regions_ms_per_step": {n: r["ms"] / args.steps for n, r in regions.items()},
        "ichol": ichol,
        "speedup_vs_ichol": (value / ichol["value"]) if ichol else None,
        "clocks": main["clocks"],
    }
    if rank == 0:
        out["cpu_baseline"] = cpu_baseline(args, pos, L, out)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return out if rank == 0 else None


def run_replicas(args, rank, local):
    """Independent suspensions of uneven size on their own streams, stepped
    concurrently by fsd_step_batch, then the same replicas one by one through
    the same kernels.  Device time: the span from the earliest start event to
    the latest end event over all replica streams."""
    import torch

    from fsd_b200.configs import suspension
    from fsd_b200.core import FSD, step_batch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rng = np.random.default_rng(1234 + rank)
    R = args.replicas
    spec = [(int(np.exp(rng.uniform(np.log(500), np.log(8000)))), float(rng.uniform(0.1, 0.5)),
             float(rng.uniform(0.0, 2.0))) for _ in range(R)]
    confs = [suspension(N, phi, 100 + k) for k, (N, phi, _) in enumerate(spec)]

    def make():
        reps = []
        for k, ((N, phi, rate), (pos, L)) in enumerate(zip(spec, confs)):
            stream = torch.cuda.Stream(dev)
            with torch.cuda.stream(stream):
                s, _ = make_solver(args, args.precond, N, L, dev, 100 + k)
                st = [torch.as_tensor(pos, device=dev).view(-1).contiguous(),
                      torch.as_tensor(np.tile([0.0, 0.0, 1.0], N).astype(np.float32), device=dev),
                      torch.zeros(3 * N, dtype=torch.int32, device=dev), torch.zeros(6 * N, device=dev),
                      torch.zeros(11 * N, device=dev)]
            reps.append((s, st, rate, stream))
        torch.cuda.synchronize(dev)
        return reps

    def run(reps, t0, steps, threads):
        starts = [torch.cuda.Event(enable_timing=True) for _ in reps]
        ends = [torch.cuda.Event(enable_timing=True) for _ in reps]
        origin = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        origin.record(torch.cuda.current_stream(dev))
        torch.cuda.synchronize(dev)
        for e, r in zip(starts, reps):
            e.record(r[3])
        for t in range(t0, t0 + steps):
            args_ = [s.step_args(t, rate, *st) for s, st, rate, _ in reps]
            status = step_batch([r[0] for r in reps], args_, nthreads=threads, raise_on_error=False)
            bad = [x for x in status if x not in (0, 4)]
            if bad:
                raise RuntimeError(f"fsd_step_batch status {bad[0]}")
        for e, r in zip(ends, reps):
            e.record(r[3])
        torch.cuda.synchronize(dev)
        return max(origin.elapsed_time(e) for e in ends) - min(origin.elapsed_time(e) for e in starts)

    reps = make()
    run(reps, 0, args.warmup, 0)
    batched_ms = run(reps, args.warmup, args.steps, 0)
    for s, *_ in reps:
        s.close()
    reps = make()
    run(reps, 0, args.warmup, 1)
    seq_ms = run(reps, args.warmup, args.steps, 1)
    for s, *_ in reps:
        s.close()
    value = R * args.steps / (batched_ms / 1e3)
    return {"metric": f"aggregate replica steps/s, {R} independent suspensions (N log-uniform in [500, 8000], "
                      f"phi uniform in [0.1, 0.5], shear rate uniform in [0, 2])",
            "value": value, "unit": "replica-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": batched_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic: seeded random sequential addition + overlap relaxation",
            "config": {"workload": "batched replicas", "replicas": R, "precond": args.precond,
                       "N": [n for n, _, _ in spec], "phi": [round(p, 3) for _, p, _ in spec]},
            "sequential": {"value": R * args.steps / (seq_ms / 1e3), "unit": "replica-steps/s",
                           "ms_per_step": seq_ms / args.steps},
            "speedup_vs_sequential": seq_ms / batched_ms}


# Saddle-operator applications per step of the IChol-preconditioned step (the
# reference's method), as the GPU arm measures them: RFD +/- and main GMRES
# iterations plus the far-field Lanczos steps.  N = 32768, phi = 0.4:
# 538.5 + 194 + 428 + 9.
ICHOL_OPS_PER_STEP = {(32768, 0.4): 1170.0}


def oracle_problem(pos, L):
    """The FP64 oracle's set-up of one configuration (neighbour rows, tables)."""
    from oracle import fsd_oracle as O

    golden = np.load(ROOT / "tests" / "golden" / "ewald_xi0.5_err1e-3.npz")
    table = (golden["table"], float(golden["self_x"]), float(golden["self_y"]), float(golden["cut"]), int(golden["n"]))
    return O.Problem(pos, (L, L, L), table=table)


def cpu_baseline(args, pos, L, gpu_out=None, pr=None, setup_s=None):
    """FP64 NumPy oracle of the same method on one host core: the saddle
    operator (mobility + lubrication, the work of every GMRES iteration) timed
    at the full N, scaled to steps/s by the operator applications one step
    needs.  A prebuilt oracle set-up may be passed in."""
    if pr is None:
        t0 = time.time()
        pr = oracle_problem(pos, L)
        setup_s = time.time() - t0
    x = np.random.default_rng(0).standard_normal(17 * len(pos))
    n, t = 0, time.time()
    while True:
        pr.saddle_multiply(x)
        n += 1
        if time.time() - t > args.cpu_sample_seconds:
            break
    t_op = (time.time() - t) / n
    if gpu_out is not None:
        it = (gpu_out.get("ichol") or gpu_out)["iterations_per_step"]
        ops = it["gmres_rfd_plus"] + it["gmres_rfd_minus"] + it["gmres_main"] + 9
    else:
        ops = ICHOL_OPS_PER_STEP.get((len(pos), round(float(getattr(args, "phi", 0.0)), 3)), 600.0)
    setup = f", setup {setup_s:.1f} s" if setup_s is not None else ""
    return {"value": 1.0 / (t_op * ops), "unit": "steps/s", "cores": 1, "kind": "port",
            "sample": f"{n} FP64 NumPy saddle-operator applications at N={len(pos)} ({t_op:.2f} s each{setup}) "
                      f"scaled by {ops:.0f} applications per step"}


def run_reference(args, ws, rank):
    if rank != 0:
        return None
    from fsd_b200.configs import suspension

    pos, L = suspension(args.N, args.phi, seed=1)
    t_all = time.time()
    t0 = time.time()
    pr = oracle_problem(pos, L)  # built once; each step samples the operator on it
    setup_s = time.time() - t0
    if args.warmup > 0:
        pr.saddle_multiply(np.random.default_rng(1).standard_normal(17 * len(pos)))
    vals = []
    sample_s = max(2.0, 10.0 / max(1, args.steps))
    for _ in range(max(1, args.steps)):
        cb = cpu_baseline(argparse.Namespace(cpu_sample_seconds=sample_s, phi=args.phi), pos, L, None, pr=pr,
                          setup_s=setup_s)
        vals.append(cb["value"])
    v = float(np.median(vals))
    return {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded random sequential addition + overlap relaxation",
            "config": {"workload": f"full FSD step, N={args.N}, phi={args.phi} (CPU FP64 oracle port)",
                       "N": args.N, "phi": args.phi},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": 1, "kind": "port", "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.time() - t_all}


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        out = run_reference(args, ws, rank)
    elif args.replicas > 0:
        out = run_replicas(args, rank, local)
    else:
        out = run_fsd(args, ws, rank, local)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
