"""Shared helpers for the parity tests (initial states, comparisons, reference runs)."""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8, dtype=np.float64).astype(np.float32)
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1])


def grid(case):
    return int(case["NX"]), int(case["NY"]), int(case["NZ"])


def interior(case):
    NX, NY, NZ = grid(case)
    m = np.zeros((NZ, NY, NX), bool)
    m[1:-1, 1:-1, 1:-1] = True
    return m.reshape(-1)


def initial_state(case, noise=0.0, seed=1234):
    """Reference initial condition (jet/jetIn.cuh:13-62 or bubble/bubbleIn.cuh:10-39)
    in reference layout, with optional seeded multiplicative noise on f."""
    NX, NY, NZ = grid(case)
    N = NX * NY * NZ
    z, y, x = np.meshgrid(np.arange(NZ), np.arange(NY), np.arange(NX), indexing="ij")
    x = x.reshape(-1); y = y.reshape(-1); z = z.reshape(-1)
    f32 = np.float32
    if case["boundary"] == "jet":
        rr = np.full(N, f32(case["rhor0"]), f32)
        rb = np.zeros(N, f32)
        dx = x.astype(f32) - f32(case["jet_x0"])
        dz = z.astype(f32) - f32(case["jet_z0"])
        jet = (dx * dx + dz * dz) <= f32(case["jet_radius"]) * f32(case["jet_radius"])
        col = (y == 0) & (x >= 1) & (x <= NX - 2) & (z >= 1) & (z <= NZ - 2)
        rr[col] = np.where(jet[col], f32(0), f32(case["rhor0"]))
        rb[col] = np.where(jet[col], f32(case["rhob0"]), f32(0))
    else:
        dx = x.astype(f32) - f32(case["bubble_x0"])
        dy = y.astype(f32) - f32(case["bubble_y0"])
        dz = z.astype(f32) - f32(case["bubble_z0"])
        inside = (dx * dx + dy * dy + dz * dz) <= f32(case["bubble_radius"]) * f32(case["bubble_radius"])
        if case.get("bubble_red_inside", 0):
            rr = np.where(inside, f32(case["rhor0"]), f32(0)).astype(f32)
            rb = np.where(inside, f32(0), f32(case["rhob0"])).astype(f32)
        else:
            rr = np.where(inside, f32(0), f32(case["rhor0"])).astype(f32)
            rb = np.where(inside, f32(case["rhob0"]), f32(0)).astype(f32)
    fr = (W[:, None] * rr[None, :]).astype(f32)
    fb = (W[:, None] * rb[None, :]).astype(f32)
    if noise:
        rng = np.random.default_rng(seed)
        eps = rng.uniform(-noise, noise, size=(2, 27, N)).astype(f32)
        fr = (fr * (f32(1) + eps[0])).astype(f32)
        fb = (fb * (f32(1) + eps[1])).astype(f32)
    zeros = np.zeros(N, f32)
    fields = dict(rhor=rr, rhob=rb, ux=zeros.copy(), uy=zeros.copy(), uz=zeros.copy())
    return fr.reshape(-1), fb.reshape(-1), fields


def run_reference(case_name, case, steps, stats_from, state=None):
    """Run the reference's own CUDA build (oracle/_ref) and load its dump."""
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_" + case_name)
    NX, NY, NZ = grid(case)
    N = NX * NY * NZ
    M = NY * (NX // 2)
    with tempfile.TemporaryDirectory() as td:
        args = [binary, "run", "jet" if case["boundary"] == "jet" else "bubble", str(steps), str(stats_from), td]
        if state is not None:
            fr, fb, fields = state
            sd = os.path.join(td, "in")
            os.makedirs(sd)
            np.asarray(fr, np.float32).tofile(os.path.join(sd, "fr.bin"))
            np.asarray(fb, np.float32).tofile(os.path.join(sd, "fb.bin"))
            np.concatenate([np.asarray(fields[k], np.float32) for k in ("rhor", "rhob", "ux", "uy", "uz")]).tofile(
                os.path.join(sd, "fields.bin"))
            args.append(sd)
        subprocess.run(args, check=True, capture_output=True, timeout=600)
        out = {
            "fr": np.fromfile(os.path.join(td, "fr.bin"), np.float32),
            "fb": np.fromfile(os.path.join(td, "fb.bin"), np.float32),
        }
        fields = np.fromfile(os.path.join(td, "fields.bin"), np.float32).reshape(5, N)
        for k, key in enumerate(("rhor", "rhob", "ux", "uy", "uz")):
            out[key] = fields[k]
        out["pi"] = np.fromfile(os.path.join(td, "pi.bin"), np.float32)
        radial = np.fromfile(os.path.join(td, "radial.bin"), np.float64).reshape(5, M)
        for k, key in enumerate(("sum_uy", "sum_uy2", "sum_ur", "sum_ur2", "sum_uruy")):
            out[key] = radial[k]
        out["count"] = np.fromfile(os.path.join(td, "count.bin"), np.uint64)
        out["tke"] = float(open(os.path.join(td, "tke.txt")).read())
    return out


def pops_interior(f, case):
    m = interior(case)
    return np.asarray(f).reshape(27, -1)[:, m]


def maxabs(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))


def psi_of(rr, rb):
    rr = np.asarray(rr, np.float64)
    rb = np.asarray(rb, np.float64)
    return (rr - rb) / (rr + rb)


def feq64(rho, ux, uy, uz):
    """Third-order Hermite equilibrium (lbm.cuh:16-35) in float64, reference
    layout (Q, Ncells)."""
    w = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8, np.float64)
    cs2 = 1.0 / 3.0
    rho, ux, uy, uz = (np.asarray(a, np.float64) for a in (rho, ux, uy, uz))
    cu = CX[:, None] * ux[None, :] + CY[:, None] * uy[None, :] + CZ[:, None] * uz[None, :]
    usq = (ux * ux + uy * uy + uz * uz)[None, :]
    a2 = cu * cu / (2 * cs2 * cs2) - usq / (2 * cs2) + cu / cs2
    a3 = cu * (cu * cu / (6 * cs2 ** 3) - usq / (2 * cs2 * cs2))
    return w[:, None] * rho[None, :] * (1.0 + a2 + a3)


def pop_maxabs(a, b, case, mask=None):
    """max |a - b| over the interior nodes of two reference-layout population
    arrays (27 x Ncells), one direction at a time so that the largest grids
    (33.5 M nodes) compare without float64 copies of the whole arrays."""
    m = interior(case) if mask is None else mask
    a = np.asarray(a).reshape(27, -1)
    b = np.asarray(b).reshape(27, -1)
    err = 0.0
    for i in range(27):
        d = np.abs(a[i][m].astype(np.float64) - b[i][m].astype(np.float64))
        err = max(err, float(d.max()))
    return err
