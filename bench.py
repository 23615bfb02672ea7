#!/usr/bin/env python
"""Benchmark of the D3Q27 colour-gradient step (one JSON line on rank 0).

Workload: the round jet, 128x256x128 (y streamwise), D=16, U=0.05,
tau=0.52, sigma=0.005, beta=0.8, jet inlet + convective outlet, radial
statistics on (the accumulating half of the 20000-step run).  A step is one
full lattice update (moments + boundary + collision).  Synthetic data: the
reference's initial condition with seeded noise; no dataset is involved.

  value      MLUPS = NX*NY*NZ*steps/t/1e6 (ghost shell counted, like
             utilities/countmlups.cuh:42-48), device time of exactly K steps
             (CUDA events on the launching stream), populations resident in HBM.
  e2e        the same metric through the public API with host buffers, copies
             inside the timed region.  The job is a run as the reference's
             main loop makes one: the initial fields come from pinned host
             memory and the populations are their equilibrium, formed on the
             device (mcg_init_equilibrium, the reference's initial states being
             feq of their fields), then K steps, then the fields are
             downloaded.  `e2e.restart` is the same with the whole state
             uploaded instead (mcg_set_fields + mcg_set_populations, 990 MB).
  roofline   live per-launch event times of the dominant kernel against its
             algorithmic bytes (216 B/node of populations per pass in float32,
             108 B in float16) and the measured HBM copy peak.
  cpu_baseline  the float64 OpenMP oracle (oracle/) on a bounded sample of the
             same workload, rank 0 only.

--impl reference runs the reference's own CUDA build (oracle/_ref, compiled
from the reference sources for this case) through its launch API on the same
GPU and workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS & % HBM roofline, FP16-store vs FP32 at stated error; adjoint/fwd cost"
DEFAULT_CASE = "jet_128x256x128"


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_launch(cells: int, kernel: str):
    """DRAM bytes (read + write) of one launch of `kernel` (e.g.
    "k_fused_pipe<CodecF32>"): the per-node figure of its ncu capture in
    profiles/traffic.json scaled to `cells` nodes, with the capture it came
    from; (None, None) when the kernel has no capture there."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            rec = json.load(fh)["kernels"][kernel]
        return int(float(rec["dram_bytes_per_node"]) * cells), rec.get("workload")
    except (OSError, KeyError, ValueError):
        return None, None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
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
        self._t.join(timeout=2)
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, v: float) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(case_name: str, seconds: float):
    """Float64 OpenMP oracle on a sample of the same workload (rank 0 only):
    whole steps until `seconds` of host time have passed."""
    from multicomponent_color_gradient_b200 import get_case
    from oracle.oracle import Oracle, num_threads

    case = get_case(case_name, NSTATS_START_STEP=0)
    O = Oracle(case, 64)
    O.init_jet()
    O.step(1)  # warm-up (first touch of the arrays)
    steps = 0
    t0 = time.perf_counter()
    while True:
        O.step(1)
        steps += 1
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    cells = case["NX"] * case["NY"] * case["NZ"]
    return {"value": round(cells * steps / dt / 1e6, 3), "unit": "MLUPS", "cores": num_threads(), "kind": "port",
            "sample": f"{steps} steps of {case_name} (float64 OpenMP oracle, radial statistics on), {dt:.1f} s"}


def adjoint_cost(steps: int, snapshots: int):
    """The bubble adjoint at its configuration: 96^3 periodic box, R = 20, tau
    0.7, sigma 0.01; initial velocity a seeded sum of divergence-free Fourier
    modes with wave numbers up to 8 per axis (4912 amplitudes) scaled to a
    peak of 0.01; J = sum (psi_T - psi*)^2 against psi* of a run with sigma =
    0.012 from the same state; `snapshots` held states (binomial
    checkpointing, its innermost segments reversed from a tape of at most 20
    moment records, the library's default).  Device time of one forward +
    reverse sweep against `steps` plain forward steps."""
    import numpy as np

    from multicomponent_color_gradient_b200.adjoint import BubbleProblem

    P = BubbleProblem("adjoint_bubble_96", nsteps=steps, snapshots=snapshots, max_mode=8, seed=1, relax_steps=50)
    try:
        a = np.random.default_rng(2).normal(size=P.modes.count)
        a *= 0.01 / np.abs(P.modes.velocity(a)).max()
        u = P.initial_velocity(a)
        T = P.solver(0.012, P.case["taub"])
        T.init_equilibrium(P.rhor, P.rhob, u[0], u[1], u[2])
        T.step(steps)
        fr, fb = T.get_populations()
        rr, rb = fr.reshape(27, -1).sum(0, dtype=np.float64), fb.reshape(27, -1).sum(0, dtype=np.float64)
        # psi of the target run; ghost nodes (no populations) enter no sum and stay 0
        P.target = np.divide(rr - rb, rr + rb, out=np.zeros_like(rr), where=(rr + rb) > 0).astype(np.float32)
        P.evaluate(a)  # warm-up
        r = P.evaluate(a)
        S = P.solver(P.case["sigma"], P.case["taub"])
        S.init_equilibrium(P.rhor, P.rhob, u[0], u[1], u[2])
        S.step(3)
        fwd = S.step_timed(steps)
        return {"value": round(r["ms"] / fwd, 3), "unit": "adjoint sweep / forward run", "workload": "adjoint_bubble_96",
                "steps": steps, "snapshots": snapshots, "tape_records": 20,
                "sweep_ms": round(r["ms"], 3), "forward_ms": round(fwd, 3),
                "forward_steps_in_sweep": r["forward_steps"], "J": r["J"], "dJ_dsigma": r["dJ_dsigma"],
                "dJ_dtau": r["dJ_dtau"], "amplitudes": int(P.modes.count),
                "objective": "sum (psi_T - psi*)^2, psi* from sigma = 0.012"}
    finally:
        P.close()


def jet_adjoint_cost(steps: int, segment: int, storage: str):
    """The jet adjoint at its configuration: jet 128x256x128, inlet profile of
    8 Bessel coefficients seeded around the top-hat (N(0, 0.02)), T = `steps`,
    J = the misfit of the time-averaged centreline velocity and half-width over
    the second half of the run for 2 <= y/D <= 10, against the profiles of a
    run with the coefficients perturbed by N(0, 0.05); forward states stored in
    `storage`, float32 adjoint, a snapshot every `segment` steps, as many
    segment tapes as device memory allows (the library's default).  Device
    time of one sweep against `steps` plain forward steps of the same storage
    (and of float32 storage)."""
    import numpy as np

    from multicomponent_color_gradient_b200 import Solver, get_case

    rng = np.random.default_rng(5)
    c0 = rng.normal(scale=0.02, size=8).astype(np.float32)
    ct = (c0 + rng.normal(scale=0.05, size=8)).astype(np.float32)
    t_begin, t_end = steps // 2, steps - 1
    case = get_case(DEFAULT_CASE, storage=storage, NSTATS_START_STEP=t_begin)
    D = 2 * int(case["jet_radius"])
    y_lo, y_hi = 2 * D, min(10 * D, case["NY"] - 2)
    with Solver(case) as S:
        S.set_inlet_bessel(ct)
        S.init_jet()
        S.step(t_end + 1)
        uc_t, rh_t = S.jet_profile_metrics()
        S.set_inlet_bessel(c0)
        S.init_jet()
        r = S.adjoint_jet_profile_run(steps, t_begin, t_end, y_lo, y_hi, uc_t, rh_t, segment=segment)
        S.init_jet()
        S.step(3)
        fwd = S.step_timed(steps)
    with Solver(get_case(DEFAULT_CASE, NSTATS_START_STEP=10 ** 9)) as S32:
        S32.init_jet()
        S32.step(3)
        fwd32 = S32.step_timed(steps)
    return {"value": round(r["ms"] / fwd, 3), "unit": "adjoint sweep / forward run", "workload": DEFAULT_CASE,
            "storage": storage, "steps": steps, "segment": segment, "sweep_ms": round(r["ms"], 3),
            "forward_ms": round(fwd, 3), "vs_float32_forward": round(r["ms"] / fwd32, 3),
            "forward_ms_float32": round(fwd32, 3), "forward_steps_in_sweep": r["forward_steps"], "J": r["J"],
            "dJ_dc": [round(float(v), 9) for v in r["dJ_dc"]],
            "objective": f"time-averaged centreline uy and half-width misfit, steps {t_begin}..{t_end}, "
                         f"y {y_lo}..{y_hi}",
            "gradient": "inlet-profile Bessel coefficients"}


def run_reference(args, world, rank):
    if world > 1 and rank != 0:
        return
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_" + args.case)
    base = {"metric": METRIC, "impl": "reference", "unit": "MLUPS", "n_gpus": 1, "higher_is_better": True}
    if not os.path.exists(binary):
        print(json.dumps(dict(base, unavailable=f"reference build {os.path.relpath(binary, ROOT)} not present "
                                                 "(built by oracle/build_ref.sh from the reference sources)")))
        return
    from multicomponent_color_gradient_b200 import get_case

    case = get_case(args.case)
    mode = "jet" if case["boundary"] == "jet" else "bubble"
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    out = subprocess.run([binary, "time", mode, str(args.warmup), str(args.steps), "1"], capture_output=True,
                         text=True, timeout=1800)
    clocks = sampler.stop()
    if out.returncode != 0:
        print(json.dumps(dict(base, unavailable=f"reference build exited {out.returncode}: {out.stderr[-200:]}")))
        return
    r = json.loads(out.stdout.strip().splitlines()[-1])
    v = r["mlups"]
    line = dict(base, value=round(v, 3), steps=args.steps, warmup=args.warmup,
                ms_per_step=round(r["ms_per_step"], 6), scaling="weak", vs_baseline=None, dtype="f32",
                data="synthetic",
                config={"workload": args.case, "shape": [case["NX"], case["NY"], case["NZ"]],
                        "implementation": "reference kernels.cu/launch.cuh compiled for sm_100a (oracle/_ref)",
                        "radial_statistics": "on", "l2": "inputs larger than L2"},
                cpu_baseline={"value": round(v, 3), "unit": "MLUPS", "kind": "reference", "cores": 0,
                              "sample": f"{args.steps} steps on the GPU: the reference has no CPU implementation"},
                e2e={"value": round(v, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                clocks=clocks)
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default=DEFAULT_CASE)
    ap.add_argument("--storage", default="f32", choices=["f32", "f16"])
    ap.add_argument("--repeats", type=int, default=5, help="least number of timed regions of `steps` steps")
    ap.add_argument("--seconds", type=float, default=1.0, help="least device time over all timed regions")
    ap.add_argument("--no-f16", action="store_true", help="skip the float16-storage companion measurement")
    ap.add_argument("--s3", type=int, default=1, help="also measure the 256x512x256 jet (float32 and float16)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="host time of the cpu_baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-cost measurement")
    ap.add_argument("--adjoint-steps", type=int, default=400, help="steps of the bubble adjoint (96^3)")
    ap.add_argument("--adjoint-snapshots", type=int, default=20, help="held states of the bubble adjoint")
    ap.add_argument("--jet-adjoint-steps", type=int, default=4000, help="steps of the jet adjoint (128x256x128)")
    ap.add_argument("--jet-adjoint-segment", type=int, default=200, help="checkpoint segment of the jet adjoint")
    ap.add_argument("--jet-adjoint-storage", default="f16", choices=["f32", "f16"],
                    help="storage of the jet adjoint's forward states")
    ap.add_argument("--shape", default=None,
                    help="NXxNYxNZ override of the case grid (smaller profiling captures); not a bench line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import numpy as np
    import torch

    from multicomponent_color_gradient_b200 import Solver, get_case

    torch.cuda.set_device(local)
    hbm_peak, peak_kind = load_peaks()

    def measure(storage: str, case_name: str, repeats_min: int, seconds_min: float):
        """Device time of exactly `args.steps` steps (CUDA events on the solver
        stream), in several timed regions: at least `repeats_min`, and about
        `seconds_min` seconds in all so that the clock sampler sees the run.
        Every rank runs the same number of regions (set from the max over
        ranks of the first region)."""
        over = {}
        if args.shape:
            over = dict(zip(("NX", "NY", "NZ"), (int(v) for v in args.shape.lower().split("x"))))
        case = get_case(case_name, storage=storage, NSTATS_START_STEP=0, seed=20260101 + rank, inlet_noise=0.01,
                        **over)
        S = Solver(case)
        S.init_jet() if case["boundary"] == "jet" else S.init_bubble()
        S.step(args.warmup)
        S.synchronize()
        barrier(world)
        sampler = ClockSampler(local)
        sampler.start()
        regions, kernel_ms = [], {"fused": 0.0, "boundary": 0.0}
        launches = n_regions = None
        while n_regions is None or len(regions) < n_regions:
            barrier(world)
            S.synchronize()
            l0 = S.launches
            ms, per_kernel = S.step_profiled(args.steps)
            if launches is None:
                launches = S.launches - l0
            for k in kernel_ms:
                kernel_ms[k] += per_kernel[k]
            regions.append(max_over_ranks(world, ms))
            if n_regions is None:
                n_regions = max(repeats_min, min(200, int(seconds_min * 1e3 / max(regions[0], 1e-3)) + 1))
        clocks = sampler.stop()
        cells = case["NX"] * case["NY"] * case["NZ"]
        ms = float(np.median(regions))
        step_bytes = 432 if storage == "f32" else 216  # algorithmic bytes per lattice update
        n_launch = args.steps * len(regions)
        r = {"case": case, "cells": cells, "ms": ms, "mlups": world * cells * args.steps / (ms * 1e3),
             "step_bytes": step_bytes, "t_fused": kernel_ms["fused"] / n_launch,
             "t_bc": kernel_ms["boundary"] / n_launch, "launches": launches, "clocks": clocks,
             "tiling": S.tiling(),
             "spread": {"regions": len(regions), "min_ms_per_step": round(min(regions) / args.steps, 6),
                        "max_ms_per_step": round(max(regions) / args.steps, 6)}}
        r["achieved"] = step_bytes * cells / (r["t_fused"] * 1e-3) / 1e9  # GB/s of the fused kernel
        r["step_gbs"] = step_bytes * cells / (ms / args.steps * 1e-3) / 1e9
        return S, r

    S, m = measure(args.storage, args.case, args.repeats, args.seconds)
    case, cells, ms, mlups = m["case"], m["cells"], m["ms"], m["mlups"]
    tiling = m["tiling"]
    kname = "k_fused_pipe" if tiling["pipelined"] else "k_fused"  # the fused-step kernel that ran
    codec = "CodecF32" if args.storage == "f32" else "CodecF16"
    traffic, traffic_src = traffic_per_launch(cells, f"{kname}<{codec}>")
    roofline = {"bound": "hbm", "kernel": kname, "achieved": round(m["achieved"], 1), "peak": hbm_peak,
                "unit": "GB/s", "frac": round(m["achieved"] / hbm_peak, 4), "peak_kind": peak_kind,
                "traffic": traffic, "traffic_capture": traffic_src, "algorithmic_bytes_per_node": m["step_bytes"],
                "step_achieved": round(m["step_gbs"], 1), "step_frac": round(m["step_gbs"] / hbm_peak, 4),
                "tiling": tiling,
                "kernels": {kname: {"ms_per_launch": round(m["t_fused"], 6)}}}
    if m["t_bc"] > 0:  # a separate boundary launch (the fused step writes the jet's boundary itself by default)
        roofline["kernels"]["k_boundary"] = {"ms_per_launch": round(m["t_bc"], 6)}

    # end to end through the public API, pinned host buffers on both sides;
    # each job runs three times and the median is kept.  The headline job
    # starts the run from host fields (the populations are their equilibrium,
    # formed on the device); `restart` uploads the whole state instead.
    e2e = None
    try:
        if args.no_e2e:
            raise RuntimeError("skipped (--no-e2e)")
        keys = ("rhor", "rhob", "ux", "uy", "uz")
        fr_h = torch.empty(27 * cells, dtype=torch.float32, pin_memory=True)
        fb_h = torch.empty(27 * cells, dtype=torch.float32, pin_memory=True)
        fl_h = {k: torch.empty(cells, dtype=torch.float32, pin_memory=True) for k in keys}
        out_h = {k: torch.empty(cells, dtype=torch.float32, pin_memory=True) for k in keys}
        fr_np, fb_np = S.get_populations()
        fr_h.numpy()[:] = fr_np
        fb_h.numpy()[:] = fb_np
        F = S.get_fields()
        for k in keys:
            fl_h[k].numpy()[:] = F[k]
        del fr_np, fb_np
        fields = {k: fl_h[k].numpy() for k in keys}
        outs = {k: out_h[k].numpy() for k in keys}

        def job(upload):
            times = []
            for _ in range(3):
                barrier(world)
                S.synchronize()
                t0 = time.perf_counter()  # every API call below that returns host data synchronises its stream
                upload()
                t1 = time.perf_counter()
                S.step(args.steps)
                S.synchronize()
                t2 = time.perf_counter()
                S.get_fields(out=outs)
                t3 = time.perf_counter()
                times.append((max_over_ranks(world, t3 - t0), t1 - t0, t2 - t1, t3 - t2))
            assert np.isfinite(outs["uy"]).all()
            times.sort()
            return times[len(times) // 2]

        def restart_upload():
            S.set_fields(**fields)
            S.set_populations(fr_h.numpy(), fb_h.numpy())

        d2h = 5 * cells * 4
        wall, t_in, t_steps, t_out = job(lambda: S.init_equilibrium(**fields))
        h2d = 5 * cells * 4
        rwall, r_in, r_steps, r_out = job(restart_upload)
        rh2d = (2 * 27 * cells + 5 * cells) * 4
        e2e = {"value": round(world * cells * args.steps / (wall * 1e6), 3), "unit": "MLUPS",
               "h2d_bytes_per_step": int(h2d // args.steps), "d2h_bytes_per_step": int(d2h // args.steps),
               "job": f"run from host fields: upload 5 fields ({h2d / 1e6:.0f} MB) and form their equilibrium "
                      f"populations on the device (mcg_init_equilibrium) + {args.steps} steps + download fields "
                      f"({d2h / 1e6:.0f} MB), pinned host buffers; median of 3 jobs",
               "seconds": round(wall, 5),
               "split_ms": {"init_equilibrium": round(t_in * 1e3, 3), "steps": round(t_steps * 1e3, 3),
                            "get_fields": round(t_out * 1e3, 3)},
               "d2h_gbs": round(d2h / t_out / 1e9, 2),
               "restart": {"value": round(world * cells * args.steps / (rwall * 1e6), 3), "unit": "MLUPS",
                           "h2d_bytes_per_step": int(rh2d // args.steps),
                           "d2h_bytes_per_step": int(d2h // args.steps),
                           "job": f"upload the whole state ({rh2d / 1e6:.0f} MB: 5 fields + 54 populations per "
                                  f"node; mcg_set_fields + mcg_set_populations) + {args.steps} steps + download "
                                  f"fields, pinned host buffers; median of 3 jobs",
                           "seconds": round(rwall, 5),
                           "split_ms": {"upload": round(r_in * 1e3, 3), "steps": round(r_steps * 1e3, 3),
                                        "get_fields": round(r_out * 1e3, 3)},
                           "h2d_gbs": round(rh2d / r_in / 1e9, 2)}}
    except Exception as exc:  # keep the device-timed number; report why e2e is missing
        e2e = {"value": None, "unit": "MLUPS", "error": str(exc)[:200]}
    S.close()

    f16 = None
    if not args.no_f16 and args.storage == "f32":
        S16, m16 = measure("f16", args.case, 3, 0.3)
        f16 = {"value": round(m16["mlups"], 3), "unit": "MLUPS", "ratio_vs_f32": round(m16["mlups"] / mlups, 3),
               "kernel_frac_216B": round(m16["achieved"] / hbm_peak, 4),
               "step_frac_216B": round(m16["step_gbs"] / hbm_peak, 4),
               "kernel_ms_per_launch": round(m16["t_fused"], 6), "tiling": m16["tiling"], "spread": m16["spread"]}
        S16.close()

    s3 = None
    if args.s3 and not args.shape and args.case == DEFAULT_CASE:
        s3 = {"workload": "jet_256x512x256", "steps": args.steps}
        try:
            for st in ("f32", "f16"):
                S3, m3 = measure(st, "jet_256x512x256", 3, 0.3)
                S3.close()
                s3[st] = {"value": round(m3["mlups"], 3), "unit": "MLUPS",
                          "kernel_ms_per_launch": round(m3["t_fused"], 6),
                          "kernel_frac": round(m3["achieved"] / hbm_peak, 4),
                          "step_frac": round(m3["step_gbs"] / hbm_peak, 4),
                          "algorithmic_bytes_per_node": m3["step_bytes"], "tiling": m3["tiling"],
                          "spread": m3["spread"]}
            s3["f16_ratio_vs_f32"] = round(s3["f16"]["value"] / s3["f32"]["value"], 3)
        except Exception as exc:
            s3["error"] = str(exc)[:200]

    adjoint = jet_adjoint = None
    if not args.no_adjoint:
        try:
            adjoint = adjoint_cost(args.adjoint_steps, args.adjoint_snapshots)
        except Exception as exc:
            adjoint = {"value": None, "error": str(exc)[:200]}
        try:
            jet_adjoint = jet_adjoint_cost(args.jet_adjoint_steps, args.jet_adjoint_segment,
                                           args.jet_adjoint_storage)
        except Exception as exc:
            jet_adjoint = {"value": None, "error": str(exc)[:200]}

    if rank != 0:
        return
    cpu = None
    if not args.no_cpu:
        try:
            cpu = cpu_baseline(args.case, args.cpu_seconds)
        except Exception as exc:
            cpu = {"value": None, "error": str(exc)[:200]}
    line = {
        "metric": METRIC, "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 6), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.case, "shape": [case["NX"], case["NY"], case["NZ"]], "storage": args.storage,
                   "tau": round(case["taub"], 6), "sigma": round(case["sigma"], 6), "beta": case["beta_recolor"],
                   "radial_statistics": "on", "inlet_noise": 0.01,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (%.0f MB of populations per buffer)" % (m["step_bytes"] / 2 * cells / 1e6)},
        "timing": {"statistic": "median over timed regions of exactly `steps` steps", **m["spread"]},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": m["launches"],
        "gpu_launches_scope": "per timed region of `steps` steps", "clocks": m["clocks"],
        "f16_store": f16, "s3": s3, "adjoint": adjoint, "jet_adjoint": jet_adjoint,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
