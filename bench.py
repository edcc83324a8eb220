#!/usr/bin/env python
"""Zone-updates/s of the 3D relativistic jet on B200.

Workload (per GPU): 3D relativistic jet, 512^3 interior cells (+3 ghosts per
side), Gamma = 4/3, WENOZ + HLLC, SSP-RK3, CFL 0.4 (dt = 0.4 / (3/dx)).
Ambient rho = 1 with 3% seeded multiplicative noise (as the reference's jet
example adds, examples/Jet3D/HARM_jet_breakout.jl:91-94), p = 1e-3, v = 0; a
nozzle of radius 16 cells on the x = 0 face injects rho = 0.01, p = 1e-3,
Lorentz factor 10 along +x; outflow elsewhere. Synthetic, generated on the
device. Inputs (5.6 GB of primitives per array) exceed L2 (126 MB).

Headline (`value`): the FP32-bulk form (FP32 reconstruction/flux/divergence,
FP64 conserved variables and con2prim) with the learned con2prim guess when the
network is available, else the previous-state guess; reported next to the plain
FP64 path on the same workload and the L1 rho/p error of the fast path against
it. `e2e`: the same fast path through the public API with host buffers
(pinned FP64 AoS primitives in, K steps, primitives out).

--impl reference: the reference has no runnable CPU path here (it is Julia and
its 2D/3D drivers need CUDA.jl); the oracle's C restatement of the same scheme
is timed on all host cores on a bounded sub-box of the workload instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s on 1 B200, 3D jet: learned+FP32 vs plain FP64 at fixed L1 error"
UNIT = "zone-updates/s"
GAMMA = 4.0 / 3.0
RECON = "wenoz"  # reconstruction of the 3D jet's solvers (--recon; the headline workload is WENOZ)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512, help="interior cells per axis")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-guess-compare", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip configs 1, 2, 3 and 5 next to the headline")
    ap.add_argument("--config2-steps", type=int, default=200,
                    help="steps of the 2D jet (config 2: 200)")
    ap.add_argument("--path", default="both", choices=["both", "fast", "fp64"],
                    help="fp64: time only the plain FP64 path (profiling runs)")
    ap.add_argument("--fp64-contract", type=int, default=0, choices=[0, 1],
                    help="with --path fp64: the FMA-contracted FP64 kernels (vb_tuning.fp64_contract)")
    ap.add_argument("--guess", default="auto", choices=["auto", "learned", "previous"],
                    help="con2prim guess of the fast path (auto: learned when the network is available)")
    ap.add_argument("--learned-form", default="fused", choices=["fused", "two"],
                    help="learned con2prim as one kernel (guess + Newton) or as a guess kernel + con2prim kernel")
    ap.add_argument("--stencil", default="pairs", choices=["pairs", "scalar"],
                    help="FP32 stencil kernel: two cells per thread on packed FP32 pairs, or one cell per thread")
    ap.add_argument("--planes", default="tma", choices=["tma", "cp-async"],
                    help="z-pair stencil: planes staged as TMA tiles, or by per-thread loads and cp.async halo copies")
    ap.add_argument("--dump", action="store_true",
                    help="also time an asynchronous dump of the interior (vb_dump_begin) overlapped with K steps")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--recon", default="wenoz", choices=["wenoz", "ppm", "minmod"],
                    help="reconstruction of the 3D jet (the headline workload: wenoz; profiling of the others)")
    ap.add_argument("--workload", default="jet3d", choices=["jet3d", "batch", "jet2d"],
                    help="batch: 256 uneven 1D/2D Riemann problems in one persistent launch (not the headline)")
    return ap.parse_args()


def workload_config(n, guess):
    return {
        "workload": f"3D relativistic jet {n}^3, {RECON.upper()}+HLLC, SSP-RK3, CFL 0.4, gamma 4/3, nozzle r=16 Gamma=10",
        "grid": [n, n, n],
        "recon": RECON.upper(),
        "riemann": "HLLC",
        "rk": 3,
        "precision": "fp32 bulk (fp64 U, RK accumulation, con2prim)",
        "con2prim_guess": guess,
        "ic": "ambient rho=1 (3% seeded noise), p=1e-3, v=0; nozzle rho=0.01 p=1e-3 Gamma=10",
        "l2": "inputs larger than L2 (5.6 GB per primitive array)",
        "parallelism": "replicas",
    }


# ---- shared problem setup -------------------------------------------------------
def nozzle(n):
    import math

    return [16.0, n / 2, n / 2, 0.01, 1e-3 / (GAMMA - 1), math.sqrt(99.0), 0.0, 0.0]


def device_ic(n, seed, noise=0.03):
    """Primitive AoS array of the workload on the device (torch, reversed shape):
    ambient rho = 1 with `noise` relative seeded density noise, p = 1e-3, v = 0."""
    import torch

    m = n + 6
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    P = torch.zeros((m, m, m, 5), dtype=torch.float64, device="cuda")
    P[..., 0] = 1.0
    if noise:
        P[..., 0] += noise * torch.randn((m, m, m), generator=gen, dtype=torch.float64, device="cuda")
    P[..., 1] = 1e-3 / (GAMMA - 1)
    return P


def make_solver(n, precision, guess, stats=0, c2p_fp32=1):
    from verona_b200 import Solver

    dx = 1.0 / n
    s = Solver(3, (n, n, n), GAMMA, (dx, dx, dx), recon=RECON, riemann="hllc", rk=3, precision=precision,
               guess=guess, n_iter=50, tol=1e-12, floor=1e-8, stats=stats, c2p_fp32=c2p_fp32)
    s.set_boundary(0, 2, nozzle(n))
    return s


def dt_of(n):
    return 0.4 / (3.0 * n)


# ---- clocks -----------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = str(index)
        try:
            import torch

            self.index = "GPU-" + str(torch.cuda.get_device_properties(index).uuid)
        except Exception:
            pass
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", self.index, f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is None:
            self.summary = None
            return
        time.sleep(0.25)
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nme, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nme)
        self.summary = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                        "reasons": sorted(reasons), "samples": len(sm)}


# ---- timing -------------------------------------------------------------------------
def timed_steps(s, dt, warmup, steps, dist=None):
    import torch

    stream = torch.cuda.current_stream()
    s.step(dt, warmup)
    torch.cuda.synchronize()
    s.profile(True)
    s.profile_read()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step(dt, steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    stage_ms, stencil_ms, stage_launches, launches = s.profile_read2()
    s.profile(False)
    timed_steps.stencil_ms = stencil_ms
    return ms, stage_ms, stage_launches, launches


def guess_comparison(n, P0, dt, W, K, dist, learned, stencil_ms_learned, stage_ms_learned, ms_learned, P64=None,
                     err_learned=None):
    """The learned guess against the method without it, on the same FP32-bulk
    workload, each timed like the headline (stencil and con2prim kernel timed
    apart by the library's profiling events) and run again with iteration
    statistics (W steps, counters reset, 3 steps):
    - learned (the headline): the network's guess with the precision gate of
      the con2prim (options.c2p_fp32, the default: FP32 pressure Newton where
      the guess has Lorentz factor below sqrt 2 and kinetic energy below 10 x
      the pressure, the FP64 W Newton for the rest in a second pass);
    - learned_ungated: the same with the FP64 W Newton on every cell;
    - previous_w: the FP64 W Newton warm-started from the previous state's W
      instead of the network (the network's contribution alone; ungated, its
      faster form: the gate in the one-cell-per-thread con2prim kernel runs
      the FP64 fallback inline and costs time there);
    - previous: the reference's con2prim cascade from the previous state
      (src/3dim/structs.jl:277-287); its counter records the cascade stage that
      converged (1 = the 1DW Newton), not Newton iterations."""
    import torch

    from verona_b200 import mlp

    out = {}
    arms = (("learned", "learned"), ("learned_ungated", "learned"), ("previous_w", "previous_w"),
            ("previous", "previous"))
    for name, guess in arms:
        if guess == "learned" and not learned:
            continue
        gate = int(name == "learned")
        if name == "learned":
            out[name] = {"ms_per_step": ms_learned / K, "value": n**3 * K / (ms_learned / 1e3),
                         "stencil_ms_per_stage": stencil_ms_learned,
                         "c2p_ms_per_stage": stage_ms_learned - stencil_ms_learned,
                         "l1_error_vs_fp64": err_learned,
                         "c2p_kernels": "k_c2p_learned (U from the divergence, network guess, FP32 pressure "
                                        "Newton where the gate admits the cell) + k_c2p_deferred (FP64 W Newton of "
                                        "the cells the gate leaves)"}
        else:
            s = make_solver(n, "fp32", guess, c2p_fp32=gate)
            if guess == "learned":
                mlp.attach(s)
            s.load_prims(P0)
            ms, st_ms, st_l, _ = timed_steps(s, dt, W, K, dist)
            sten = timed_steps.stencil_ms / max(st_l, 1)
            err = None
            if P64 is not None:
                Pa = s.store_prims()
                torch.cuda.synchronize()
                err = l1_errors(Pa, P64)
                del Pa
            s.close()
            kern = {"learned_ungated": "k_c2p_learned with the FP64 W Newton on every cell",
                    "previous_w": "k_c2p (the FP64 W Newton from the previous state's W)",
                    "previous": "k_c2p (the reference cascade from the previous primitive state)"}[name]
            out[name] = {"ms_per_step": ms / K, "value": n**3 * K / (ms / 1e3), "stencil_ms_per_stage": sten,
                         "c2p_ms_per_stage": st_ms / max(st_l, 1) - sten, "l1_error_vs_fp64": err,
                         "c2p_kernels": kern}
        s = make_solver(n, "fp32", guess, stats=1, c2p_fp32=gate)
        if guess == "learned":
            mlp.attach(s)
        s.load_prims(P0)
        s.step(dt, W)
        s.reset_counters()
        s.step(dt, 3)
        torch.cuda.synchronize()
        c = s.counters()
        s.close()
        cells = max(int(c[3]), 1)
        stat = {"fallbacks_per_cell": float(c[1]) / cells, "fp64_cell_fraction": float(c[6]) / cells,
                "failures": int(c[0]), "cell_solves_counted": int(c[3])}
        if name == "previous":
            stat["mean_cascade_stage"] = float(c[2]) / cells
        else:
            stat["newton_iters_per_cell"] = float(c[2]) / cells
        out[name].update(stat)
    if learned:
        for base in ("learned_ungated", "previous_w", "previous"):
            out[f"step_speedup_learned_vs_{base}"] = out[base]["ms_per_step"] / out["learned"]["ms_per_step"]
            out[f"c2p_speedup_learned_vs_{base}"] = out[base]["c2p_ms_per_stage"] / out["learned"]["c2p_ms_per_stage"]
    return out


def l1_errors(a, b):
    """L1 relative error of rho and p (interior) of run a against run b."""
    import torch

    ai, bi = a[3:-3, 3:-3, 3:-3], b[3:-3, 3:-3, 3:-3]
    out = {}
    for name, v in (("rho", 0), ("p", 1)):
        out[name] = float((ai[..., v] - bi[..., v]).abs().mean() / bi[..., v].abs().mean())
    la = torch.sqrt(1 + (ai[..., 2:] ** 2).sum(-1))
    lb = torch.sqrt(1 + (bi[..., 2:] ** 2).sum(-1))
    out["lorentz_max_abs"] = float((la - lb).abs().max())
    return out


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp32_roofline(cells, stencil_ms, pair_stencil):
    """Compute roofline of the FP32 stencil kernel, the binding resource of the
    headline stage (its HBM fraction is small by construction): FP32 operations
    per cell (2 fma + add + mul over all lanes, ncu op counters of one launch)
    over the kernel's live CUDA-event time per launch, against SGEMM."""
    flop = read_traffic("fp32_pairs_stencil_flop")
    if not (pair_stencil and flop):
        return None
    peak = fp32_gemm_tflops()
    ach = flop * cells / (stencil_ms / 1e3) / 1e12
    return {"bound": "fp32", "kernel": "k_stage_zp", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
            "frac": ach / peak, "flop_per_cell": flop, "kernel_ms_per_launch": stencil_ms,
            "peak_kind": "measured in this run: cuBLAS SGEMM 8192^3 (torch, TF32 off)"}


MLP_FLOP_PER_CELL = 2 * (4 * 64 + 64 * 64 + 64 * 64 + 64 * 1)  # one inference of the 4-64-64-64-1 network


def tensor_roofline(cells, stage_ms, stencil_ms, learned_fused):
    """Tensor-core roofline of the network inside the fused learned con2prim
    kernel: algorithmic MLP FLOPs per cell (17,024) times the cells of one
    stage launch over that kernel's live time (the stage group's time minus
    the stencil's), against the sustained BF16 peak. The kernel also forms U
    and runs the W Newton, and is bound by latency, not by the tensor cores."""
    try:
        c2p_ms = stage_ms - stencil_ms
        if not learned_fused or not (stencil_ms > 0 and c2p_ms > 0):
            return None
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peak, kind = float(json.load(f)["bf16_tflops_sustained"]), "measured (sustained)"
        except Exception:
            peak, kind = 1400.0, "fallback (sustained)"
        ach = MLP_FLOP_PER_CELL * cells / (c2p_ms / 1e3) / 1e12
        return {"bound": "tensor", "kernel": "k_c2p_learned (network part)", "achieved": ach, "peak": peak,
                "unit": "TFLOP/s", "frac": ach / peak, "flop_per_cell": MLP_FLOP_PER_CELL,
                "kernel_ms_per_launch": c2p_ms, "peak_kind": kind}
    except Exception:
        return None


def fp32_gemm_tflops():
    """FP32 denominator of the stencil's compute roofline: cuBLAS SGEMM 8192^3
    on the CUDA cores (TF32 off), best of 3 after one warm-up."""
    import torch

    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn((n, n), dtype=torch.float32, device="cuda")
    b = torch.randn((n, n), dtype=torch.float32, device="cuda")
    c = a @ b
    best = None
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n**3 / (best / 1e3) / 1e12


def fp64_gemm_tflops():
    """FP64 denominator of the plain path's roofline: cuBLAS DGEMM 8192^3
    through torch, best of 3 after one warm-up (B200's FP64 vector and tensor
    rates are nominally equal)."""
    import torch

    n = 8192
    a = torch.randn((n, n), dtype=torch.float64, device="cuda")
    b = torch.randn((n, n), dtype=torch.float64, device="cuda")
    c = a @ b
    best = None
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n**3 / (best / 1e3) / 1e12


def read_traffic(key):
    """DRAM bytes per cell of one RK-stage kernel group (the stage kernel plus
    its con2prim kernel where split) from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_traffic.txt")
    try:
        for line in open(path):
            f = line.split()
            if len(f) >= 2 and f[0] == key:
                return float(f[1])
    except OSError:
        pass
    return None


# ---- CPU baseline (the oracle, test infrastructure, timed on the host cores) -----------
def cpu_baseline(seconds):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np

    from oracle import oracle as O

    S = 96
    n = (S, S, S)
    rng = np.random.default_rng(42)
    P = np.zeros((5, S + 6, S + 6, S + 6), order="F")
    P[0] = 1.0 + 0.03 * rng.standard_normal(P.shape[1:])
    P[1] = 1e-3 / (GAMMA - 1)
    s = O.SolverND(3, n, P, GAMMA, 1e-8, 50, 1e-12, O.WENOZ, O.HLLC, 3)
    s.set_grid(1.0 / S, 1.0 / S, 1.0 / S)
    s.set_boundary(0, O.BC_NOZZLE, [16.0 * S / 512, S / 2, S / 2, 0.01, 3e-3, 99 ** 0.5, 0, 0])
    dt = dt_of(S)
    t0 = time.perf_counter()
    s.step(dt, 1)
    one = time.perf_counter() - t0
    k = max(1, int(seconds / max(one, 1e-3)))
    t0 = time.perf_counter()
    s.step(dt, k)
    el = time.perf_counter() - t0
    return {
        "value": S**3 * k / el,
        "unit": UNIT,
        "cores": O.num_threads(),
        "kind": "port",
        "sample": f"oracle (C FP64 restatement, OpenMP) on a {S}^3 sub-box of the same jet workload "
                  f"(WENOZ+HLLC+RK3, FP64), {k} steps after 1 warm-up step, {el:.1f} s",
    }


# ---- arms ------------------------------------------------------------------------------
def run_reference(args, rank):
    if rank != 0:
        return
    cb = cpu_baseline(args.cpu_seconds * max(1, args.steps) / 10.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.n, "previous state (reference)"),
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (Julia/CUDA.jl) does not run here; its scheme is timed as the oracle's C restatement",
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, dist):
    import torch

    import verona_b200  # noqa: F401  (fails loudly if the CUDA library is missing)
    from verona_b200 import _lib

    n, K, W = args.n, args.steps, args.warmup
    dt = dt_of(n)
    cells = n**3
    learned_ok = False
    try:
        from verona_b200 import mlp  # noqa: F401

        learned_ok = mlp.available()
    except Exception:
        learned_ok = False
    if args.guess == "learned" and not learned_ok:
        raise RuntimeError("--guess learned: the learned con2prim guess is unavailable")
    if args.guess == "previous":
        learned_ok = False
    guess = "learned" if learned_ok else "previous"
    info = {}
    if learned_ok:
        t0 = time.time()
        src = "loaded" if os.path.exists(mlp.DEFAULT_WEIGHTS) else "trained"
        mlp.trained()
        info["mlp"] = {"weights": src, "seconds": round(time.time() - t0, 2), "params": mlp.n_params()}
    P0 = device_ic(n, 42 + rank)

    # plain FP64 path (same scheme, reference con2prim)
    fp64 = None
    if args.path == "fp64":
        s = make_solver(n, "fp64", "previous")
        s.set_tuning(fp64_contract=args.fp64_contract)
        s.load_prims(P0)
        ms, st_ms, st_l, ln = timed_steps(s, dt, W, K, dist)
        print(json.dumps({"path": "fp64", "zone_updates_per_s": cells * K / (ms / 1e3), "ms_per_step": ms / K,
                          "stage_ms_per_launch": st_ms / max(st_l, 1), "launches": ln}), flush=True)
        s.close()
        return
    fp64_forms = {}
    if not args.no_fp64 and args.path == "both":
        peak64 = fp64_gemm_tflops()
        hbm_peak, hbm_kind = read_peaks()
        for form, contract in (("bitexact", 0), ("contracted", 1)):
            s = make_solver(n, "fp64", "previous")
            s.set_tuning(fp64_contract=contract)
            s.load_prims(P0)
            ms, st_ms, st_l, ln = timed_steps(s, dt, W, K, dist)
            r = {"value": cells * K / (ms / 1e3), "ms_per_step": ms / K, "stage_ms_per_launch": st_ms / max(st_l, 1),
                 "fma_contraction": bool(contract)}
            # HBM roofline of the plain path: 560 B of compulsory traffic per
            # zone-update of an FP64 SSP-RK3 step (14 passes of 5 FP64 arrays)
            # at the measured step rate
            ach_hbm = r["value"] * 560.0 / 1e9
            r["roofline_hbm"] = {"bound": "hbm", "achieved": ach_hbm, "peak": hbm_peak, "unit": "GB/s",
                                 "frac": ach_hbm / hbm_peak, "bytes_per_zone_update": 560.0, "peak_kind": hbm_kind}
            # FP64 roofline of the stage group (k_stage_zm<double> + k_c2p<double>):
            # FP64 operations per cell (2 dfma + dadd + dmul, ncu counters of one
            # RK-stage launch pair) over the group's live time, against DGEMM
            flop = read_traffic(f"fp64_previous_stage_group_flop{'_contracted' if contract else ''}")
            if flop:
                ach = flop * cells / (r["stage_ms_per_launch"] / 1e3) / 1e12
                r["roofline"] = {"bound": "fp64", "achieved": ach, "peak": peak64, "unit": "TFLOP/s",
                                 "frac": ach / peak64, "flop_per_cell": flop,
                                 "peak_kind": "measured in this run: cuBLAS DGEMM 8192^3 (torch)"}
            Pout = s.store_prims()
            torch.cuda.synchronize()
            info[f"fp64_{form}_counters"] = s.counters().tolist()
            s.close()
            del s
            fp64_forms[form] = (r, Pout)
        P64 = fp64_forms["bitexact"][1]
        # the contracted form against the bit-exact one (which equals the
        # oracle bit for bit at small sizes): max difference per field over
        # the field's max magnitude, on the full grid after W + K steps
        Pc = fp64_forms["contracted"][1]
        fp64_forms["contracted"][0]["max_rel_vs_bitexact"] = [
            float((Pc[..., v] - P64[..., v]).abs().max() / P64[..., v].abs().max()) for v in range(5)]
        del Pc
        ok = max(fp64_forms["contracted"][0]["max_rel_vs_bitexact"]) <= 1e-10
        fp64 = dict(fp64_forms["contracted" if ok else "bitexact"][0])
        fp64["form"] = "contracted" if ok else "bitexact"
        fp64["forms"] = {k: v[0] for k, v in fp64_forms.items()}
        fp64_forms = {}

    # headline: FP32 bulk (+ learned guess when available)
    s = make_solver(n, "fp32", guess)
    if learned_ok:
        mlp.attach(s)
    s.set_tuning(learned_fused=int(args.learned_form == "fused"), fp32_pairs=int(args.stencil == "pairs"),
                 tma_tiles=int(args.planes == "tma"))
    tma_active = s.tma_tiles_active
    s.load_prims(P0)
    with Clocks(torch.cuda.current_device()) as clk:
        ms, st_ms, st_l, launches = timed_steps(s, dt, W, K, dist)
    stencil_ms = timed_steps.stencil_ms / max(st_l, 1)
    Pf = s.store_prims()
    torch.cuda.synchronize()
    info["fast_counters"] = s.counters().tolist()
    err = l1_errors(Pf, P64) if fp64 else None
    del Pf
    guesses = None
    if args.path == "both" and not args.no_guess_compare:
        guesses = guess_comparison(n, P0, dt, W, K, dist, learned_ok, stencil_ms, st_ms / max(st_l, 1), ms,
                                   P64=P64 if fp64 else None, err_learned=err)
    if fp64:
        del P64

    t_tensor = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_tensor, op=dist.ReduceOp.MAX)
    ms_max = float(t_tensor.item())
    value = world * cells * K / (ms_max / 1e3)

    # asynchronous dump of the interior, overlapped with the next K steps
    dump = None
    if args.dump:
        shp = s.interior_shape
        keep = torch.empty(tuple(reversed(shp)), dtype=torch.float64, pin_memory=True)
        out = keep.numpy().transpose(3, 2, 1, 0)
        s.dump_begin(out)
        s.dump_wait()  # first dump allocates the snapshot buffer and the copy stream
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.dump_begin(out)
        nan = s.dump_wait()
        alone = (time.perf_counter() - t0) * 1e3
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        s.dump_begin(out)
        s.step(dt, K)
        e1.record(stream)
        s.dump_wait()
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        dump = {"interior_bytes": out.nbytes, "nan_count": nan, "copy_alone_ms": alone,
                "steps_with_dump_ms": e0.elapsed_time(e1), "wall_with_dump_ms": wall, "steps_without_dump_ms": ms,
                "note": f"dump_begin then {K} steps on the compute stream while the snapshot crosses PCIe on the "
                        "handle's copy stream; steps_without_dump_ms is the timed region of the headline"}
        del out, keep

    # e2e through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.empty(P0.shape, dtype=torch.float64, pin_memory=True)
        host.copy_(P0)
        del P0
        torch.cuda.synchronize()
        s.load_prims(host.numpy().transpose(3, 2, 1, 0))  # warm the staging buffer
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        s.load_prims(host.numpy().transpose(3, 2, 1, 0))
        s.step(dt, K)
        s.prims_into(host.numpy().transpose(3, 2, 1, 0))
        el = time.perf_counter() - t0
        tt = torch.tensor([el], dtype=torch.float64, device="cuda")
        if dist is not None:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        el = float(tt.item())
        nbytes = host.numel() * 8
        e2e = {"value": world * cells * K / el, "unit": UNIT, "h2d_bytes_per_step": nbytes / K,
               "d2h_bytes_per_step": nbytes / K,
               "note": f"one H2D of the FP64 AoS primitives, {K} steps, one D2H (the HARM_HLL call pattern)"}
    s.close()
    del s
    torch.cuda.empty_cache()
    configs = None
    if args.path == "both" and not args.no_configs:
        configs = configs_measure(args, rank, world, dist)

    if rank != 0:
        return
    # roofline of the dominant kernel group (one RK stage: the z-marching stage
    # kernel and its con2prim kernel). Algorithmic bytes per zone-update of an
    # FP32-bulk SSP-RK3 step: P read and written once per stage, 3 * 2 * 5 * 4 B
    # = 120 B, and the FP64 conserved arrays, 8 passes of 5 * 8 B (stage 1: U^n
    # in, U^1 out; stages 2, 3: U^n and U^(k-1) in, U^k out) = 320 B; 440 B in
    # all, 440/3 B per cell per stage launch.
    peak, peak_kind = read_peaks()
    bytes_per_cell_step = 440.0
    stage_ms_per_launch = st_ms / max(st_l, 1)
    achieved = cells * bytes_per_cell_step / 3.0 / (stage_ms_per_launch / 1e3) / 1e9
    form = "_fused" if learned_ok and args.learned_form == "fused" else ""
    form += "_pairs" if args.stencil == "pairs" else ""
    form += "_gated" if learned_ok else ""  # options.c2p_fp32 = 1, the default
    traffic = read_traffic(f"fp32_{guess}{form}_stage_group")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 bulk + f64 (U, con2prim)", "data": "synthetic",
        "config": dict(workload_config(n, guess), learned_form=args.learned_form if learned_ok else None,
                       stencil=args.stencil, planes=args.planes if args.stencil == "pairs" else None,
                       tma_tiles_active=tma_active),
        "fp64_plain": fp64,
        "speedup_vs_fp64": (value / world) / fp64["value"] if fp64 else None,
        "speedup_vs_fp64_denominator": (f"fp64_plain.forms.{fp64['form']}: the faster plain FP64 form within the "
                                        "parity bar (1e-10 per field)") if fp64 else None,
        "l1_error_vs_fp64": err,
        "guess_comparison": guesses,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic * cells if traffic else None, "peak_kind": peak_kind,
                     "per": "one RK-stage launch of the kernel group over the full grid",
                     "kernel": ("k_stage_zp (z-pair FP32 reconstruct+HLLC+divergence) + k_c2p_learned "
                                "(RK combination, tensor-core guess, gated Newton) + k_c2p_deferred" if learned_ok and
                                args.learned_form == "fused" else "stencil kernel + con2prim kernel(s)"),
                     "algorithmic_bytes_per_launch": bytes_per_cell_step / 3.0 * cells,
                     "stage_ms_per_launch": stage_ms_per_launch},
        "roofline_fp32": fp32_roofline(cells, stencil_ms, learned_ok and args.learned_form == "fused"
                                       and args.stencil == "pairs"),
        "roofline_tensor": tensor_roofline(cells, stage_ms_per_launch, stencil_ms,
                                           learned_ok and args.learned_form == "fused"),
        "gpu_launches": launches,
        "clocks": clk.summary,
        "e2e": e2e,
        "counters": info,
        "configs": configs,
    }
    if dump is not None:
        line["dump"] = dump
    if not os.environ.get("VB_BENCH_NO_CPU"):
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
    print(json.dumps(line), flush=True)


# ---- batch of uneven problems -------------------------------------------------------------
BATCH_GAMMA = 5.0 / 3.0


def batch_measure(K, W, rank, world, dist, e2e_on=True, single_on=True):
    """192 1D tubes (N in [256, 8192]) and 64 2D quadrant problems (side in
    [128, 1024]) from seed 42, MINMOD/PPM/WENOZ per problem, HLLC, SSP-RK3,
    FP32 bulk, gamma 5/3: K steps of every problem as one persistent launch."""
    import numpy as np
    import torch

    from verona_b200 import Solver
    from verona_b200.autotune import tune_batch
    from verona_b200.batch import Batch, riemann_problems

    opts = dict(riemann="hllc", rk=3, precision="fp32", n_iter=50, tol=1e-12, floor=1e-8)
    specs, prims = riemann_problems(42 + rank, gamma=BATCH_GAMMA)
    b = Batch(specs, BATCH_GAMMA, **opts)
    for i, P in enumerate(prims):
        b.load_prims(i, P)
    info = b.info()
    cells = info["interior_cells"]
    tune = tune_batch(b, steps=2, use_cache=False)
    stream = torch.cuda.current_stream()
    b.step(W)
    b.reset_counters()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    with Clocks(torch.cuda.current_device()) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.step(K)  # one graph launch: K steps of all problems in one persistent kernel
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cnt = b.counters()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    value = world * cells * K / (ms / 1e3)

    # the same problems one grid at a time (a Solver per problem, its own launches)
    ks = max(1, min(K, 3))
    single = None
    solvers = []
    for spec, P in (zip(specs, prims) if single_on else ()):
        d = spec["dims"]
        dx = (spec["dx"],) if d == 1 else (spec["dx"], spec["dy"])
        s_ = Solver(d, spec["n"][:d], BATCH_GAMMA, dx, recon=spec["recon"], **opts)
        s_.load_prims(P)
        solvers.append((s_, spec["dt"]))
    for s_, dt in solvers:
        s_.step(dt, 1)
    torch.cuda.synchronize()
    e0.record(stream)
    for s_, dt in solvers:
        s_.step(dt, ks)
    e1.record(stream)
    torch.cuda.synchronize()
    if single_on:
        single = cells * ks / (e0.elapsed_time(e1) / 1e3)
    for s_, _ in solvers:
        s_.close()

    # e2e: host primitives in, K steps, host primitives out, through the public API
    e2e = None
    if e2e_on:
        host = [torch.from_numpy(np.ascontiguousarray(P.transpose(tuple(range(P.ndim - 1, -1, -1))))).pin_memory()
                for P in prims]
        dev = [torch.empty(h.shape, dtype=torch.float64, device="cuda") for h in host]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i, (h, d) in enumerate(zip(host, dev)):
            d.copy_(h, non_blocking=True)
            b.load_prims(i, d)
        b.step(K)
        for i, (h, d) in enumerate(zip(host, dev)):
            b.store_prims(i, d)
            h.copy_(d, non_blocking=True)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        nbytes = sum(h.numel() * 8 for h in host)
        e2e = {"value": world * cells * K / el, "unit": UNIT, "h2d_bytes_per_step": nbytes / K,
               "d2h_bytes_per_step": nbytes / K}
    b.close()
    peak, peak_kind = read_peaks()
    # algorithmic bytes per zone-update, FP32-bulk SSP-RK3: 6 passes of P (4 B)
    # and 8 of U (8 B) per variable; 3 variables in 1D, 4 in 2D
    c1 = sum(q["n"][0] for q in specs if q["dims"] == 1)
    alg = (c1 * (6 * 3 * 4 + 8 * 3 * 8) + (cells - c1) * (6 * 4 * 4 + 8 * 4 * 8)) / cells
    achieved = value / world * alg / 1e9
    line = {
        "metric": "zone-updates/s on 1 B200, 256 uneven 1D/2D Riemann problems in one persistent launch",
        "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 bulk + f64 (U, con2prim)",
        "data": "synthetic (seeded states)",
        "config": {"workload": "192 1D tubes N~U[256,8192] + 64 2D quadrant problems side~U[128,1024], seed 42, "
                               "MINMOD/PPM/WENOZ per problem, HLLC, SSP-RK3, CFL 0.4, gamma 5/3",
                   "interior_cells": cells, "tiles_per_stage": info["tiles_per_stage"],
                   "l2": "inputs larger than L2 (%.2f GB of state)" % (info["device_bytes"] / 1e9),
                   "tuning": {k: tune[k] for k in ("variant", "ctas_per_sm", "shape", "ms_per_step")}},
        "one_grid_at_a_time": {"value": single, "unit": UNIT, "steps": ks,
                               "note": "the same problems through one Solver each, launched one after another"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "algorithmic_bytes_per_zone_update": alg},
        "gpu_launches": 1,
        "counters": [int(x) for x in cnt],
        "clocks": clk.summary,
        "e2e": e2e,
    }
    return line


def run_batch(args, rank, world, dist):
    line = batch_measure(args.steps, args.warmup, rank, world, dist, e2e_on=not args.no_e2e)
    if rank == 0:
        print(json.dumps(line), flush=True)


def jet2d_measure(n, K, W, rank, world, dist, planes="tma", forms=("fp64", "fp64c", "fp32", "fp32w")):
    """2D relativistic jet n^2, WENOZ + HLLC, SSP-RK3, CFL 0.4, gamma 4/3:
    ambient rho = 1 (3 % seeded noise), p = 1e-3, v = 0; nozzle of radius 32
    cells on the x-lo face (rho 0.01, p 1e-3, Lorentz factor 10 along +x),
    outflow elsewhere. Each form timed over K steps on the device after W:
    fp64 (the plain method, the reference's rounding), fp64c (the plain
    method with FMA contraction), fp32 (the FP32-bulk form with the
    reference's 2D con2prim), fp32w (the FP32-bulk form with the previous
    state's W through the gated W Newton, VB_GUESS_PREVIOUS_W)."""
    import math

    import torch

    from verona_b200 import Solver

    dx = 1.0 / n
    dt = 0.4 / (2.0 * n)
    tma = int(planes == "tma")
    hbm_peak, hbm_kind = read_peaks()
    res = {}
    with Clocks(torch.cuda.current_device()) as clk:
        for form in forms:
            prec = "fp32" if form.startswith("fp32") else "fp64"
            s = Solver(2, (n, n), GAMMA, (dx, dx), recon="wenoz", riemann="hllc", rk=3, precision=prec, n_iter=50,
                       tol=1e-12, floor=1e-8, guess="previous_w" if form == "fp32w" else "previous")
            s.set_tuning(tma_tiles=tma, fp64_contract=int(form == "fp64c"))
            tma_active = s.tma_tiles_active
            s.set_boundary(0, 2, [32.0, n / 2, 0.0, 0.01, 1e-3 / (GAMMA - 1), math.sqrt(99.0), 0.0, 0.0])
            s.init_prims("ambient", seed=7 + rank, noise=0.03, rho=1.0, u=1e-3 / (GAMMA - 1))
            ms, st_ms, st_l, launches = timed_steps(s, dt, W, K, dist)
            t = torch.tensor([ms], device="cuda")
            if dist is not None:
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
            c = s.counters()
            v = world * n * n * K / (t.item() / 1e3)
            # compulsory traffic per zone-update of an SSP-RK3 step in 2D: 14
            # passes of 4 arrays, P in FP32 for the FP32-bulk form (6 passes)
            bpz = 6 * 4 * 4 + 8 * 4 * 8 if prec == "fp32" else 448.0
            res[form] = {"value": v, "ms_per_step": t.item() / K, "stage_ms_per_launch": st_ms / max(st_l, 1),
                         "c2p_failures": int(c[0]), "tma_tiles_active": tma_active, "tma_timeouts": int(c[4]),
                         "roofline_hbm": {"achieved": v / world * bpz / 1e9, "peak": hbm_peak, "unit": "GB/s",
                                          "frac": v / world * bpz / 1e9 / hbm_peak, "bytes_per_zone_update": bpz,
                                          "peak_kind": hbm_kind}}
            s.close()
            del s
    return res, clk.summary


def run_jet2d(args, rank, world, dist):
    """The 2D jet (config 2) alone: 4096^2 unless --n is above 512."""
    n = args.n if args.n > 512 else 4096
    K, W = args.steps, args.warmup
    res, clocks = jet2d_measure(n, K, W, rank, world, dist, planes=args.planes)
    if rank != 0:
        return
    line = {
        "metric": "zone-updates/s on 1 B200, 2D jet (plain FP64 method)", "value": res["fp64"]["value"],
        "unit": "zone-updates/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": res["fp64"]["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"2D relativistic jet {n}^2, WENOZ+HLLC, SSP-RK3, CFL 0.4, gamma 4/3, nozzle r=32 "
                               "Gamma=10", "grid": [n, n], "tiles": args.planes,
                   "l2": "inputs larger than L2" if n * n * 4 * 8 > 126e6 else "inputs smaller than L2",
                   "parallelism": "replicas"},
        "fp64": res["fp64"], "fp64_contracted": res["fp64c"], "fp32_bulk": res["fp32"],
        "fp32_bulk_previous_w": res["fp32w"], "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def config1_measure(rank):
    """Config 1, Marti & Mueller problem 1 on N = 1024 cells to t = 0.4 (1024
    steps, CFL 0.4, gamma 5/3): the reference's own 1D scheme
    (Verona1D.HARM_HLL: MINMOD, HLL, midpoint RK2, no ghosts) on the GPU (one
    persistent CTA runs every step) and as the oracle's C restatement on one
    host core; and the configured form (MINMOD + HLLC, RK2, outflow ghosts)
    through the ghosted 1D solver on the GPU and the oracle. zone-updates/s =
    1024 cells x steps / time of the whole run."""
    import numpy as np
    import torch

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import mm1_ghosted, n_steps, shock_tube_1d
    from oracle import oracle as O
    from verona_b200 import Solver

    g, N = 5.0 / 3.0, 1024
    dx = 1.0 / N
    dt = 0.4 * dx
    steps, _ = n_steps(dt, 0.4)
    out = {"cells": N, "steps": steps}
    stream = torch.cuda.current_stream()

    def gpu_time(s, P0):
        s.load_prims(P0)
        s.step(dt, 2)  # warm-up (module load, first launches)
        s.load_prims(P0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(dt, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    x, rho, u, ux = shock_tube_1d(N, gamma=g)
    s = Solver(1, (N,), g, (dx,), nghost=0, recon="minmod", n_iter=50, tol=1e-12)
    el = gpu_time(s, np.asfortranarray(np.stack([rho, u, ux])))
    s.close()
    t0 = time.perf_counter()
    o = O.Solver1DRef(rho, u, ux, g, "minmod", 50, 1e-12)
    o.step(dt, dx, steps)
    el_cpu = time.perf_counter() - t0
    out["reference_scheme_hll_rk2"] = {
        "gpu": {"value": N * steps / el, "seconds": el, "kernel": "k_ref1d_steps (one persistent CTA)"},
        "cpu_oracle": {"value": N * steps / el_cpu, "seconds": el_cpu, "cores": 1,
                       "note": "the oracle's C restatement of Verona1D.HARM_HLL (the reference's CPU path)"}}
    xg, P0 = mm1_ghosted(N, g)
    s = Solver(1, (N,), g, (dx,), recon="minmod", riemann="hllc", rk=2, n_iter=50, tol=1e-12, floor=1e-10)
    el = gpu_time(s, P0)
    s.close()
    t0 = time.perf_counter()
    o = O.SolverND(1, (N,), P0, g, 1e-10, 50, 1e-12, O.MINMOD, O.HLLC, 2)
    o.set_grid(dx)
    o.step(dt, steps)
    el_cpu = time.perf_counter() - t0
    out["configured_minmod_hllc_rk2"] = {
        "gpu": {"value": N * steps / el, "seconds": el, "kernel": "k_stage (box tiles), one launch per stage"},
        "cpu_oracle": {"value": N * steps / el_cpu, "seconds": el_cpu, "cores": O.num_threads()}}
    return out


def config3_measure(n, K, W, rank, world, dist, recon="ppm", noise=0.03, learned=False):
    """A precision form on the 3D jet n^3 with `recon` + HLLC (SSP-RK3, gamma
    4/3, nozzle radius 16 cells, Lorentz 10; config 3 is PPM): the FP32-bulk
    form (with the learned guess if `learned`) and the plain FP64 path
    (FMA-contracted) over the same K steps after W from the same state, with
    the L1 rho / p and max Lorentz-factor errors of the FP32-bulk result
    against the FP64 one."""
    import torch

    from verona_b200 import Solver, mlp

    dx = 1.0 / n
    dt = dt_of(n)
    P0 = device_ic(n, 42 + rank, noise)
    hbm_peak, hbm_kind = read_peaks()
    res, outs = {}, {}
    for prec in ("fp32", "fp64"):
        guess = "learned" if (learned and prec == "fp32") else "previous"
        s = Solver(3, (n, n, n), GAMMA, (dx, dx, dx), recon=recon, riemann="hllc", rk=3, precision=prec,
                   guess=guess, n_iter=50, tol=1e-12, floor=1e-8)
        s.set_tuning(fp64_contract=int(prec == "fp64"))
        s.set_boundary(0, 2, nozzle(n))
        if guess == "learned":
            mlp.attach(s)
        s.load_prims(P0)
        ms, st_ms, st_l, _ = timed_steps(s, dt, W, K, dist)
        v = world * n**3 * K / (ms / 1e3)
        bpz = 440.0 if prec == "fp32" else 560.0
        res[prec] = {"value": v, "ms_per_step": ms / K, "stage_ms_per_launch": st_ms / max(st_l, 1),
                     "c2p_failures": int(s.counters()[0]),
                     "roofline_hbm": {"achieved": v / world * bpz / 1e9, "peak": hbm_peak, "unit": "GB/s",
                                      "frac": v / world * bpz / 1e9 / hbm_peak, "bytes_per_zone_update": bpz,
                                      "peak_kind": hbm_kind}}
        outs[prec] = s.store_prims()
        torch.cuda.synchronize()
        s.close()
        del s
    del P0
    res["l1_error_fp32_vs_fp64"] = l1_errors(outs["fp32"], outs["fp64"])
    res["steps"] = K
    res["speedup_fp32_vs_fp64"] = res["fp32"]["value"] / res["fp64"]["value"]
    del outs
    torch.cuda.empty_cache()
    return res


def configs_measure(args, rank, world, dist):
    """Configs 1, 2, 3 and 5 of the task next to the headline (config 4)."""
    import torch

    out = {}
    K, W = args.steps, args.warmup
    out["config1_1d_shock_tube_1024"] = config1_measure(rank)
    torch.cuda.empty_cache()
    res, _ = jet2d_measure(4096, args.config2_steps, W, rank, world, dist)
    out["config2_2d_jet_4096"] = dict(res, steps=args.config2_steps,
                                      workload="2D jet 4096^2, WENOZ+HLLC, SSP-RK3, nozzle r=32 Gamma=10")
    torch.cuda.empty_cache()
    out["config3_3d_jet_512_ppm"] = dict(config3_measure(args.n, K, W, rank, world, dist),
                                         workload=f"3D jet {args.n}^3, PPM+HLLC, SSP-RK3, nozzle r=16 Gamma=10")
    torch.cuda.empty_cache()
    # the headline workload on the configured noise-free ambient
    out["config4_noise_free"] = dict(config3_measure(args.n, K, W, rank, world, dist, recon="wenoz", noise=0.0,
                                                     learned=True),
                                     workload=f"3D jet {args.n}^3, WENOZ+HLLC, SSP-RK3, nozzle r=16 Gamma=10, "
                                              "ambient rho=1 p=1e-3 without noise; fp32 = learned guess")
    torch.cuda.empty_cache()
    b = batch_measure(K, W, rank, world, dist, e2e_on=False, single_on=False)
    out["config5_batch_256"] = {k: b[k] for k in ("value", "ms_per_step", "roofline", "counters", "config")}
    out["config5_batch_256"]["steps"] = K
    torch.cuda.empty_cache()
    return out


def main():
    global RECON
    args = parse()
    RECON = args.recon
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as D

        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
        dist = D
    try:
        if args.workload == "batch":
            run_batch(args, rank, world, dist)
        elif args.workload == "jet2d":
            run_jet2d(args, rank, world, dist)
        else:
            run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
