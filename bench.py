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
  e2e        the same metric through the public API with host buffers: upload
             the state from pinned host memory (mcg_set_fields +
             mcg_set_populations), K steps, download the fields; copies inside
             the timed region.
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
    """DRAM bytes (read + write) of one launch of `kernel` scaled from its
    committed ncu summary (profiles/<kernel>_jet_*.md, line
    `dram_bytes_per_node: <value>`), or None."""
    import glob
    import re

    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", f"{kernel}_jet_*.md"))):
        m = re.search(r"dram_bytes_per_node:\s*([0-9.]+)", open(path).read())
        if m:
            return int(float(m.group(1)) * cells)
    return None


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


def adjoint_cost(steps: int):
    """Discrete-adjoint cost on the 96^3 periodic bubble (R=20, tau 0.7, sigma
    0.01): device time of one forward + reverse sweep over `steps` steps (a
    moment record per state) against `steps` plain forward steps."""
    import numpy as np

    from multicomponent_color_gradient_b200.adjoint import BubbleProblem

    P = BubbleProblem("adjoint_bubble_96", nsteps=steps, max_mode=1, seed=1, relax_steps=0)
    try:
        a = np.random.default_rng(2).normal(scale=2e-3, size=P.modes.count)
        P.evaluate(a)
        r = P.evaluate(a)
        S = P.solver(P.case["sigma"], P.case["taub"])
        u = P.initial_velocity(a)
        S.init_equilibrium(P.rhor, P.rhob, u[0], u[1], u[2])
        S.step(3)
        fwd = S.step_timed(steps)
        return {"value": round(r["ms"] / fwd, 3), "unit": "adjoint sweep / forward run", "workload": "adjoint_bubble_96",
                "steps": steps, "sweep_ms": round(r["ms"], 3), "forward_ms": round(fwd, 3),
                "forward_steps_in_sweep": r["forward_steps"]}
    finally:
        P.close()


def jet_adjoint_cost(steps: int, segment: int):
    """Jet adjoint cost on the bench jet (128x256x128): one forward + reverse
    sweep over `steps` steps (objective over the second half, y >= 64, inlet
    profile gradient) against `steps` plain forward steps."""
    import numpy as np

    from multicomponent_color_gradient_b200 import Solver, get_case

    with Solver(get_case(DEFAULT_CASE, NSTATS_START_STEP=10 ** 9)) as S:
        S.set_inlet_bessel(np.zeros(8, np.float32))
        S.init_jet()
        S.adjoint_jet_run(20, 10, 19, 64)  # warm-up
        r = S.adjoint_jet_run(steps, steps // 2, steps - 1, 64, segment=segment)
        S.init_jet()
        S.step(3)
        fwd = S.step_timed(steps)
    return {"value": round(r["ms"] / fwd, 3), "unit": "adjoint sweep / forward run", "workload": DEFAULT_CASE,
            "steps": steps, "segment": segment, "sweep_ms": round(r["ms"], 3), "forward_ms": round(fwd, 3),
            "forward_steps_in_sweep": r["forward_steps"], "gradient": "inlet-profile Bessel coefficients"}


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
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default=DEFAULT_CASE)
    ap.add_argument("--storage", default="f32", choices=["f32", "f16"])
    ap.add_argument("--no-f16", action="store_true", help="skip the float16-storage companion measurement")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="host time of the cpu_baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-cost measurement")
    ap.add_argument("--adjoint-steps", type=int, default=100)
    ap.add_argument("--jet-adjoint-steps", type=int, default=400, help="steps of the jet-adjoint cost measurement")
    ap.add_argument("--jet-adjoint-segment", type=int, default=100, help="checkpoint segment of the jet adjoint")
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

    def measure(storage: str):
        over = {}
        if args.shape:
            over = dict(zip(("NX", "NY", "NZ"), (int(v) for v in args.shape.lower().split("x"))))
        case = get_case(args.case, storage=storage, NSTATS_START_STEP=0, seed=20260101 + rank, inlet_noise=0.01,
                        **over)
        S = Solver(case)
        S.init_jet() if case["boundary"] == "jet" else S.init_bubble()
        S.step(args.warmup)
        S.synchronize()
        barrier(world)
        l0 = S.launches
        sampler = ClockSampler(local)
        sampler.start()
        ms, per_kernel = S.step_profiled(args.steps)
        clocks = sampler.stop()
        launches = S.launches - l0
        ms = max_over_ranks(world, ms)
        return case, S, ms, per_kernel, launches, clocks

    case, S, ms, per_kernel, launches, clocks = measure(args.storage)
    cells = case["NX"] * case["NY"] * case["NZ"]
    mlups = world * cells * args.steps / (ms * 1e3)
    step_bytes = 432 if args.storage == "f32" else 216  # algorithmic bytes per lattice update
    t_fused = per_kernel["fused"] / args.steps  # ms per launch
    t_bc = per_kernel["boundary"] / args.steps
    ach = step_bytes * cells / (t_fused * 1e-3) / 1e9
    step_gbps = step_bytes * cells / (ms / args.steps * 1e-3) / 1e9
    tiling = S.tiling()
    kname = "k_fused_pipe" if tiling["pipelined"] else "k_fused"  # the fused-step kernel that ran
    roofline = {"bound": "hbm", "kernel": kname, "achieved": round(ach, 1), "peak": hbm_peak, "unit": "GB/s",
                "frac": round(ach / hbm_peak, 4), "peak_kind": peak_kind, "traffic": traffic_per_launch(cells, kname),
                "algorithmic_bytes_per_node": step_bytes,
                "step_achieved": round(step_gbps, 1), "step_frac": round(step_gbps / hbm_peak, 4),
                "tiling": tiling,
                "kernels": {kname: {"ms_per_launch": round(t_fused, 6)},
                            "k_boundary": {"ms_per_launch": round(t_bc, 6)}}}

    # end to end through the public API: host state in, K steps, fields out
    e2e = None
    try:
        if args.no_e2e:
            raise RuntimeError("skipped (--no-e2e)")
        fr_h = torch.empty(27 * cells, dtype=torch.float32, pin_memory=True)
        fb_h = torch.empty(27 * cells, dtype=torch.float32, pin_memory=True)
        fl_h = {k: torch.empty(cells, dtype=torch.float32, pin_memory=True) for k in ("rhor", "rhob", "ux", "uy", "uz")}
        fr_np, fb_np = S.get_populations()
        fr_h.numpy()[:] = fr_np
        fb_h.numpy()[:] = fb_np
        F = S.get_fields()
        for k in fl_h:
            fl_h[k].numpy()[:] = F[k]
        del fr_np, fb_np
        barrier(world)
        S.synchronize()
        t0 = time.perf_counter()  # every API call below that returns host data synchronises its stream
        S.set_fields(**{k: fl_h[k].numpy() for k in fl_h})
        S.set_populations(fr_h.numpy(), fb_h.numpy())
        S.step(args.steps)
        out = S.get_fields()
        wall = time.perf_counter() - t0
        e2e_s = max_over_ranks(world, wall)
        h2d = (2 * 27 * cells + 5 * cells) * 4
        d2h = 5 * cells * 4
        e2e = {"value": round(world * cells * args.steps / (e2e_s * 1e6), 3), "unit": "MLUPS",
               "h2d_bytes_per_step": int(h2d // args.steps), "d2h_bytes_per_step": int(d2h // args.steps),
               "job": f"upload state ({h2d / 1e6:.0f} MB) + {args.steps} steps + download fields ({d2h / 1e6:.0f} MB)",
               "seconds": round(e2e_s, 4)}
        assert np.isfinite(out["uy"]).all()
    except Exception as exc:  # keep the device-timed number; report why e2e is missing
        e2e = {"value": None, "unit": "MLUPS", "error": str(exc)[:200]}
    S.close()

    f16 = None
    if not args.no_f16 and args.storage == "f32":
        c16, S16, ms16, pk16, _, _ = measure("f16")
        m16 = world * cells * args.steps / (ms16 * 1e3)
        f16 = {"value": round(m16, 3), "unit": "MLUPS", "ratio_vs_f32": round(m16 / mlups, 3),
               "step_frac_216B": round(216 * cells / (ms16 / args.steps * 1e-3) / 1e9 / hbm_peak, 4)}
        S16.close()

    adjoint = jet_adjoint = None
    if not args.no_adjoint:
        try:
            adjoint = adjoint_cost(args.adjoint_steps)
        except Exception as exc:
            adjoint = {"value": None, "error": str(exc)[:200]}
        try:
            jet_adjoint = jet_adjoint_cost(args.jet_adjoint_steps, args.jet_adjoint_segment)
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
                   "l2": "inputs larger than L2 (%.0f MB of populations per buffer)" % (step_bytes / 2 * cells / 1e6)},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
        "f16_store": f16, "adjoint": adjoint, "jet_adjoint": jet_adjoint,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
