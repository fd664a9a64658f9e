"""Benchmark: full FSD time steps per second at N=32768, phi=0.4.

Workload (one "step"): neighbour list, preconditioner build, pair forces,
far-field Brownian slip (wave-space noise + Lanczos on the real-space
mobility), near-field Brownian force (Lanczos on R_FU), random finite
difference drift (two saddle solves), main saddle solve to relative residual
1e-4 (warm-started), Euler update with simple shear 1.0.  kT = 1, dt = 1e-4,
Ewald accuracy 1e-3 (xi 0.5, 72^3 grid, P = 6).  Positions from seeded random
sequential addition followed by overlap relaxation.

The headline preconditioner is the learned family's fastest form at this
configuration: the two-hop sparse approximate inverse of the lubrication block
with six inner GMRES steps and flexible outer GMRES (no network,
"learned_network": false).  The same steps are then timed with the family's
other forms -- the inner Chebyshev polynomial whose interval the trained
network predicts ("learned_interval_polynomial"), a fixed interval, and
coefficients fitted at every build ("other_forms") -- and with the plain IChol
preconditioner for the metric's comparison ("ichol").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fsd|reference]
                  [--precond learned|ichol|none] [--inner k] [--poly k] [--no-ichol]
  python bench.py --config5          # held-out dense suspensions, one velocity computation per form
  python bench.py --case mobility|poly_apply|gmres_apply|precond_build   # one operator (profiling cases)
  python bench.py --replicas 64      # batched replicas

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
    ap.add_argument("--poly", type=int, default=0,
                    help="main arm: terms of the learned inner polynomial (0: inner GMRES steps)")
    ap.add_argument("--poly-terms", type=int, default=10,
                    help="terms of the inner polynomial in the comparison arms (and in --case / --config5)")
    ap.add_argument("--no-compare", action="store_true", help="skip the other forms of the preconditioner")
    ap.add_argument("--no-ichol", action="store_true", help="skip the IChol comparison run")
    ap.add_argument("--no-net", action="store_true", help="learned preconditioner without the network correction")
    ap.add_argument("--no-autotune", action="store_true", help="fixed spreading tiles and FFT batches")
    ap.add_argument("--replicas", type=int, default=0,
                    help="batched-replica mode: this many independent suspensions, N log-uniform in [500, 8000], "
                         "phi uniform in [0.1, 0.5], shear rate uniform in [0, 2], stepped concurrently and then "
                         "one by one (prints its own JSON line)")
    ap.add_argument("--ichol-steps", type=int, default=2)
    ap.add_argument("--config5", action="store_true",
                    help="learned vs IChol vs SPAI + inner GMRES on held-out dense suspensions (own JSON line)")
    ap.add_argument("--config5-phis", type=float, nargs="+", default=[0.45, 0.5, 0.55])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the host-core timing (profiling runs)")
    ap.add_argument("--case", choices=["mobility", "poly_apply", "gmres_apply", "precond_build"], default=None,
                    help="one operator on the benchmarked suspension, --steps times after one untimed call "
                         "(the small cases the kernel profiles are captured on; prints its own JSON line)")
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


def precond_form(args, net, form=None, interval=0.05):
    if args.precond == "ichol":
        return "RCM + block IC(0) of the pruned lubrication block (the reference's preconditioner)"
    if args.precond == "none":
        return "identity"
    form = form or ("poly" if args.poly >= 2 else "gmres")
    if form == "poly":
        if net:
            src = "Chebyshev interval [rho lambda, lambda] with rho predicted by the trained message-passing network"
        elif interval > 0:
            src = f"fixed Chebyshev interval [{interval} lambda, lambda] (no network)"
        else:
            src = "coefficients fitted to four probe vectors at every build (no network)"
        return (f"two-hop sparse approximate inverse G, inner polynomial y = G q(AG) t of degree {args.poly - 1}, "
                f"{src}; plain outer GMRES")
    return (f"two-hop sparse approximate inverse + {args.inner} inner GMRES steps, flexible outer GMRES"
            + (", trained network correction" if net else ", no network"))


def poly_weights(k):
    return ROOT / "fsd_b200" / "data" / f"learned_poly_k{k}.f32"


def make_solver(args, precond, N, L, dev, seed, form=None, interval=0.05):
    """form (learned only): "poly" = the inner Chebyshev polynomial, its
    interval predicted by the network when weights ship (else the fixed
    interval ratio `interval`, or a least-squares fit to probes for 0);
    "gmres" = inner GMRES steps on the approximate inverse; default from --poly."""
    from fsd_b200.core import FSD

    form = form or ("poly" if args.poly >= 2 else "gmres")
    poly = precond == "learned" and form == "poly"
    s = FSD(N, (L, L, L, 0.0), device=dev, T=1.0, dt=1e-4, seed=seed, error=1e-3, solver_tol=1e-4,
            lanczos_tol=1e-3, rfd_epsilon=1e-3, precond=precond, period=0, gmres_max_iter=3000,
            gmres_restart=200 if precond == "ichol" else 100,
            learned_inner=args.inner if (precond == "learned" and not poly) else 0,
            learned_poly=args.poly if poly else 0, poly_interval=interval, autotune=0 if args.no_autotune else 1)
    net = False
    wf = poly_weights(args.poly) if poly else WEIGHTS
    if precond == "learned" and wf.exists() and not args.no_net:
        s.learned_set_weights(np.fromfile(wf, "<f4"))
        net = True
    return s, net


def max_over_ranks(value: float, dev, ws: int) -> float:
    """The largest of the ranks' values (every rank takes part; a no-op on one
    rank): the device time of a multi-GPU run is its slowest rank's."""
    if ws <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(ws: int, steps: int, ms: float) -> float:
    """Steps per second of the whole job: every rank steps its own replica."""
    return ws * steps / (ms / 1e3)


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
    total_ms = max_over_ranks(float(sum(step_ms)), dev, ws)
    regions = None
    if profile:
        lib.fsd_profile_read(s._h, ms_regions.ctypes.data_as(C.c_void_p), cnt_regions.ctypes.data_as(C.c_void_p),
                             nreg, 1)
        lib.fsd_profile_enable(s._h, 0)
        regions = {n: {"ms": float(ms_regions[i]), "calls": int(cnt_regions[i])} for i, n in enumerate(_lib.REGIONS)}
    return {"total_ms": total_ms, "step_ms": step_ms, "iters": iters_summary(iters), "launches": int(launches),
            "regions": regions, "clocks": clk.summary() if clk else None, "steps": steps}


def iters_summary(iters):
    it = np.array(iters, np.float64)
    return {"gmres_rfd_plus": float(it[:, 0].mean()), "gmres_rfd_minus": float(it[:, 1].mean()),
            "gmres_main": float(it[:, 2].mean()), "lanczos_ff": float(it[:, 3].mean()),
            "lanczos_nf": float(it[:, 4].mean())}


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
    # Headline: device time of the steps with the library's region profiler off.
    main = timed_steps(args, s, state, args.steps, args.warmup, dev, ws, clocks=True, profile=False)
    value = whole_job_rate(ws, args.steps, main["total_ms"])
    # Per-region breakdown and the roofline's launch times: a separate pass over
    # the next steps of the same trajectory with the CUDA-event profiler on.
    prof = timed_steps(args, s, state, max(1, min(3, args.steps)), 0, dev, ws, profile=True)
    # --- end to end through the C ABI with host buffers: the same warm-up and
    # timed steps of the same trajectory on a second handle (the step is
    # deterministic, so the iteration counts repeat the headline's), every
    # step uploading the state the previous step left in host memory and
    # reading back the velocity and the new state, with the same L2 flush
    # (outside the events) as above.
    e2e = None
    if not args.no_e2e:
        s.close()
        s, _ = make_solver(args, args.precond, N, L, dev, 1 + rank)
        p, ori, img, F, V, step_no = fresh_state()
        for _ in range(args.warmup):
            st = s.step(step_no[0], 1.0, p, ori, img, F, V, raise_on_error=False)
            step_no[0] += 1
            if st not in (0, 4):
                raise RuntimeError(f"fsd_step status {st}")
        stream = torch.cuda.current_stream(dev)
        pin = lambda t: t.detach().cpu().pin_memory()
        h_pos, h_ori, h_img = pin(p), pin(ori), pin(img)
        h_V = torch.empty(11 * N).pin_memory()
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        e2e_iters = []
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            p.copy_(h_pos, non_blocking=True)
            ori.copy_(h_ori, non_blocking=True)
            img.copy_(h_img, non_blocking=True)
            st = s.step(step_no[0], 1.0, p, ori, img, F, V, raise_on_error=False)
            step_no[0] += 1
            if st not in (0, 4):
                raise RuntimeError(f"fsd_step status {st}")
            h_V.copy_(V, non_blocking=True)
            h_pos.copy_(p, non_blocking=True)
            h_ori.copy_(ori, non_blocking=True)
            h_img.copy_(img, non_blocking=True)
            evs[k][1].record(stream)
            si = s.solve_info()
            e2e_iters.append(si["gmres_iters"] + [si["lanczos_ff_iters"], si["lanczos_nf_iters"]])
        torch.cuda.synchronize(dev)
        e2e_ms = max_over_ranks(float(sum(a.elapsed_time(b) for a, b in evs)), dev, ws)
        e2e = {"value": whole_job_rate(ws, args.steps, e2e_ms), "unit": "steps/s",
               "h2d_bytes_per_step": int(4 * (h_pos.numel() + h_ori.numel() + h_img.numel())),
               "d2h_bytes_per_step": int(4 * (h_V.numel() + h_pos.numel() + h_ori.numel() + h_img.numel())),
               "ms_per_step": e2e_ms / args.steps,
               "iterations_per_step": iters_summary(e2e_iters),
               "note": "state carried between steps through pinned host memory; L2 flushed before each step"}
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
    # --- the preconditioner's other forms on the same steps of the same
    # trajectory: inner GMRES steps on the approximate inverse, and the inner
    # polynomial with the network's interval, a fixed interval, or
    # coefficients fitted to probe vectors at every build
    forms = {}
    if args.precond == "learned" and not args.no_compare:
        main_poly = args.poly >= 2
        cand = {"spai_inner_gmres": ("gmres", 0.05, False)} if main_poly else {}
        if not main_poly:
            cand["learned_interval_polynomial"] = ("poly", 0.05, True)
        cand["fixed_interval_polynomial"] = ("poly", 0.05, False)
        cand["fitted_polynomial"] = ("poly", 0.0, False)
        for name, (form, interval, with_net) in cand.items():
            a2 = argparse.Namespace(**vars(args))
            a2.no_net = not with_net
            if form == "poly":
                a2.poly = args.poly if main_poly else args.poly_terms
            sc, net2 = make_solver(a2, "learned", N, L, dev, 1 + rank, form=form, interval=interval)
            r = timed_steps(a2, sc, fresh_state(), args.steps, args.warmup, dev, ws)
            sc.close()
            forms[name] = {"value": ws * args.steps / (r["total_ms"] / 1e3), "unit": "steps/s",
                           "ms_per_step": r["total_ms"] / args.steps, "iterations_per_step": r["iters"],
                           "learned_network": net2, "precond_form": precond_form(a2, net2, form, interval)}
    # --- roofline of the dominant single-kernel region (profiled pass)
    regions = prof["regions"]
    prof_steps = prof["steps"]
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
        "config": {"workload": workload_name(N, phi), "N": N, "phi": phi,
                   "grid": [info.Nx, info.Ny, info.Nz], "P": info.P, "precond": args.precond,
                   "learned_inner": args.inner if (args.precond == "learned" and args.poly < 2) else None,
                   "learned_poly": args.poly if (args.precond == "learned" and args.poly >= 2) else None,
                   "learned_network": net,
                   "precond_form": precond_form(args, net),
                   "autotune": not args.no_autotune,
                   "gmres_tol": 1e-4, "ewald_error": 1e-3, "l2": "flushed before every timed step (256 MiB write)",
                   "parallelism": f"replicas x{ws}"},
        "e2e": e2e, "gpu_launches": main["launches"], "roofline": roofline,
        "iterations_per_step": main["iters"],
        "regions_ms_per_step": {n: r["ms"] / prof_steps for n, r in regions.items()},
        "profiled_pass": {"steps": prof_steps, "ms_per_step": prof["total_ms"] / prof_steps,
                          "note": "separate pass with the CUDA-event region profiler on; the headline is timed "
                                  "with it off"},
        "ichol": ichol,
        "speedup_vs_ichol": (value / ichol["value"]) if ichol else None,
        "other_forms": forms,
        "speedup_vs_ichol_other_forms": {k: v["value"] / ichol["value"] for k, v in forms.items()} if ichol
        else None,
        "headline_over_other_forms": {k: value / v["value"] for k, v in forms.items()},
        "clocks": main["clocks"],
    }
    if rank == 0 and not args.no_cpu_baseline:
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


# Iteration counts of the IChol-preconditioned step (the reference's method)
# measured by the GPU arm at N = 32768, phi = 0.4; used when the CPU legs run
# without a GPU measurement beside them.
ICHOL_ITERS = {(32768, 0.4): {"gmres_rfd_plus": 538.5, "gmres_rfd_minus": 194.0, "gmres_main": 428.0,
                              "lanczos_ff": 9.0, "lanczos_nf": 25.0}}


def workload_name(N, phi):
    return f"full FSD step, N={N}, phi={phi}, shear 1.0, kT 1, dt 1e-4, Ewald 1e-3, GMRES 1e-4"


def ewald_table_golden():
    golden = np.load(ROOT / "tests" / "golden" / "ewald_xi0.5_err1e-3.npz")
    return (golden["table"], float(golden["self_x"]), float(golden["self_y"]), float(golden["cut"]), int(golden["n"]))


def cpu_baseline(args, pos, L, gpu_out=None, sampler=None):
    """The same step in FP64 on the host cores (oracle.cpu_step): every stage
    of the step timed once on the full configuration, assembled with the
    iteration counts of the IChol method (the reference's preconditioner)."""
    from oracle.cpu_step import StepSampler, cpu_model

    t0 = time.time()
    if sampler is None:
        sampler = StepSampler(pos, L, ewald_table_golden()).sample_setup().sample_iteration()
    if gpu_out is not None and gpu_out.get("ichol"):
        iters, src = gpu_out["ichol"]["iterations_per_step"], "this run's IChol arm"
    else:
        iters = ICHOL_ITERS.get((len(pos), round(float(args.phi), 3)))
        src = "the IChol arm at this configuration"
        if iters is None:
            iters, src = {"gmres_rfd_plus": 300.0, "gmres_rfd_minus": 300.0, "gmres_main": 300.0,
                          "lanczos_ff": 9.0, "lanczos_nf": 25.0}, "an assumed 300 per solve"
    sec, parts = sampler.step_seconds(iters)
    # a complete step run end to end at a size the FP64 oracle finishes in seconds
    from fsd_b200.configs import suspension
    from oracle.cpu_step import full_step_seconds
    pos_s, L_s = suspension(1000, float(args.phi), seed=1)
    fs, fparts, fits = full_step_seconds(pos_s, L_s, ewald_table_golden())
    full = {"N": 1000, "phi": float(args.phi), "seconds": fs, "steps_per_s": 1.0 / fs,
            "iterations": fits, "stage_seconds": {k: round(v, 3) for k, v in fparts.items()},
            "note": "one complete FP64 step measured end to end (oracle.cpu_step.full_step_seconds): "
                    "Lanczos samplers, two RFD solves and the main solve with GMRES(200) to 1e-4 and SciPy's "
                    "incomplete LU in the IC(0) slot"}
    return {"value": 1.0 / sec, "unit": "steps/s", "cores": sampler.threads, "kind": "port",
            "cpu_model": cpu_model(), "full_step_measured": full,
            "sample": f"FP64 oracle at N={len(pos)}: every stage of one step timed once on the configuration "
                      f"({time.time() - t0:.0f} s of host time), GMRES/Lanczos stage costs per iteration scaled by "
                      f"the iteration counts of {src}; FFTs on {sampler.threads} threads, pair sums single-threaded",
            "stage_seconds": {k: round(v, 3) for k, v in parts.items()}}


def run_reference(args, ws, rank):
    """Reference arm: the reference's CUDA code does not build with CUDA >= 12
    and it has no CPU implementation of this path, so the arm is the FP64
    oracle port of the same method on the host cores (oracle.cpu_step).  Its
    set-up samples every stage of the step once; each step then re-times one
    GMRES iteration (operator, preconditioner, Gram-Schmidt) and reports the
    full step assembled from it."""
    if rank != 0:
        return None
    from fsd_b200.configs import suspension
    from oracle.cpu_step import StepSampler, cpu_model

    pos, L = suspension(args.N, args.phi, seed=1)
    t_all = time.time()
    sampler = StepSampler(pos, L, ewald_table_golden()).sample_setup()
    for _ in range(max(0, min(args.warmup, 1))):
        sampler.sample_iteration()
    iters = ICHOL_ITERS.get((args.N, round(float(args.phi), 3)),
                            {"gmres_rfd_plus": 300.0, "gmres_rfd_minus": 300.0, "gmres_main": 300.0,
                             "lanczos_ff": 9.0, "lanczos_nf": 25.0})
    secs, walls = [], []
    for _ in range(max(1, args.steps)):
        t = time.time()
        sampler.sample_iteration()
        secs.append(sampler.step_seconds(iters)[0])
        walls.append(time.time() - t)
    sec = float(np.median(secs))
    v = 1.0 / sec
    cb = cpu_baseline(args, pos, L, None, sampler=sampler)
    return {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded random sequential addition + overlap relaxation, min gap 1e-3",
            "config": {"workload": workload_name(args.N, args.phi), "N": args.N, "phi": args.phi, "precond": "ichol",
                       "gmres_tol": 1e-4, "ewald_error": 1e-3, "implementation": "FP64 CPU oracle port"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cb["cores"], "kind": "port",
                             "cpu_model": cb["cpu_model"], "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "timing": "each step's figure is assembled from stage times sampled on the host (about "
                      f"{np.mean(walls):.1f} s of sampling per step), not a step run to completion",
            "wall_s": time.time() - t_all}


def run_config5(args, local):
    """Learned preconditioner on dense suspensions (N = 32768 at phi 0.45,
    0.5, 0.55, shear rate 1, kT = 1) on held-out seeds: one velocity
    computation (RFD +/- and main saddle solves to 1e-4) per preconditioner,
    with the outer GMRES iterations of each solve and the device time."""
    import torch

    from fsd_b200 import _lib
    from fsd_b200.configs import suspension
    from fsd_b200.core import FSD

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N = args.N
    forms = {
        "ichol": dict(precond="ichol", gmres_restart=200, learned_inner=0),
        "spai_gmres6": dict(precond="learned", gmres_restart=100, learned_inner=6),
        "fitted_poly10": dict(precond="learned", gmres_restart=100, learned_inner=0, learned_poly=10,
                              poly_interval=0.0),
        "fixed_interval_poly10": dict(precond="learned", gmres_restart=100, learned_inner=0, learned_poly=10,
                                      poly_interval=0.05),
        "learned_poly10": dict(precond="learned", gmres_restart=100, learned_inner=0, learned_poly=10),
    }
    w = np.fromfile(poly_weights(10), "<f4") if poly_weights(10).exists() else None  # the shipped k = 10 network
    results = {}
    for phi in args.config5_phis:
        pos, L = suspension(N, phi, seed=1000 + int(round(phi * 100)))  # seeds the training never used
        res = {}
        for name, kw in forms.items():
            if name == "learned_poly10" and w is None:
                continue
            s = FSD(N, (L, L, L, 0.0), device=dev, T=1.0, dt=1e-4, seed=7, solver_tol=1e-4, lanczos_tol=1e-3,
                    rfd_epsilon=1e-3, period=0, gmres_max_iter=6000, **kw)
            if name == "learned_poly10":
                s.learned_set_weights(w)
            times, iters, resid = [], [], []
            # the first call also captures graphs and tunes; the second is timed
            # at the next timestep (new Brownian draws; the main solve starts
            # from the first call's solution, as in a trajectory)
            for rep in range(2):
                p = torch.as_tensor(pos, device=dev).view(-1).contiguous()
                ori = torch.as_tensor(np.tile([0.0, 0.0, 1.0], N).astype(np.float32), device=dev)
                img = torch.zeros(3 * N, dtype=torch.int32, device=dev)
                F = torch.zeros(6 * N, device=dev)
                V = torch.zeros(11 * N, device=dev)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize(dev)
                e0.record()
                a = s.step_args(rep, 1.0, p, ori, img, F, V)
                st = _lib.lib().fsd_compute_velocity(s._h, C.byref(a))
                e1.record()
                torch.cuda.synchronize(dev)
                if st not in (0, 3, 4):
                    raise RuntimeError(f"{name} phi={phi}: status {st}")
                si = s.solve_info()
                si["status"] = st
                times.append(e0.elapsed_time(e1))
                iters.append(si["gmres_iters"])
                resid.append(si["gmres_resid"])
            s.close()
            res[name] = {"outer_iterations": iters[-1], "residuals": resid[-1], "ms": times[-1],
                         "converged": si["status"] != 3}
            if "poly" in name:
                res[name].update(poly_source=si["poly_source"], poly_ratio=si["poly_ratio"])
        results[str(phi)] = res
    return {"metric": "config 5: learned preconditioner on held-out dense suspensions, one velocity computation "
                      "(three saddle solves to 1e-4)", "unit": "ms", "N": N, "higher_is_better": False,
            "data": "synthetic: seeded random sequential addition + overlap relaxation, seeds not used in training",
            "results": results}


def run_case(args, local):
    """One operator of the path on the benchmarked suspension (N, phi, seed 1):
    the mobility (wave + real space), one application of the learned inner
    polynomial (k = --poly-terms, fixed interval 0.05) or of the inner-GMRES form
    (--inner steps), or one build of the learned preconditioner with the
    shipped network; CUDA-event time per call."""
    import torch

    from fsd_b200.configs import suspension
    from fsd_b200.core import FSD

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N = args.N
    pos, L = suspension(N, args.phi, seed=1)
    p = torch.as_tensor(pos, device=dev).view(-1).contiguous()
    kw = {}
    if args.case == "poly_apply":
        kw = dict(precond="learned", learned_inner=0, learned_poly=args.poly_terms, poly_interval=0.05)
    elif args.case == "gmres_apply":
        kw = dict(precond="learned", learned_inner=args.inner)
    elif args.case == "precond_build":
        kw = dict(precond="learned", learned_inner=0, learned_poly=args.poly_terms)
    s = FSD(N, (L, L, L, 0.0), device=dev, **kw)
    if args.case == "precond_build" and poly_weights(args.poly_terms).exists():
        s.learned_set_weights(np.fromfile(poly_weights(args.poly_terms), "<f4"))
    s.build_neighbor_list(p)
    rng = np.random.default_rng(0)
    if args.case == "mobility":
        x = torch.as_tensor(rng.standard_normal(11 * N), dtype=torch.float32, device=dev)
        op = lambda: s.mobility(p, x)  # noqa: E731
    elif args.case in ("poly_apply", "gmres_apply"):
        s.precond_build(p)
        x = torch.as_tensor(rng.standard_normal(17 * N), dtype=torch.float32, device=dev)
        op = lambda: s.precond_apply(x)  # noqa: E731
    else:
        op = lambda: s.precond_build(p)  # noqa: E731
    op()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        op()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / max(1, args.steps)
    s.close()
    return {"case": args.case, "N": N, "phi": args.phi, "calls": args.steps, "us_per_call": 1e3 * ms}


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.case:
        out = run_case(args, local) if rank == 0 else None
    elif args.impl == "reference":
        out = run_reference(args, ws, rank)
    elif args.config5:
        out = run_config5(args, local) if rank == 0 else None
    elif args.replicas > 0:
        out = run_replicas(args, rank, local)
    else:
        out = run_fsd(args, ws, rank, local)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
