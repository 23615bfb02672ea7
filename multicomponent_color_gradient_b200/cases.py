"""Named cases (shapes and physics) for the D3Q27 colour-gradient solver.

Every run parameter of the reference is a compile-time constant in
constants.cuh:8-76.  A case here is the same set of names as a plain dict, so
one table feeds the solver (``Solver(case)``), the constants.cuh generator and
the tests.  ``derive`` repeats the float32 arithmetic of constants.cuh:59-76
so derived values (nu, tau, sigma) are bit-identical to what the reference
computes for the same Re, We and jet scales.
"""
from __future__ import annotations

import copy

import numpy as np

f32 = np.float32

BOUNDARY = {"jet": 0, "closed": 1, "periodic": 2}
STORAGE = {"f32": 0, "f16": 1}

# constants.cuh as shipped (constants.cuh:8-76)
REFERENCE_DEFAULT = dict(
    NX=128, NY=400, NZ=128,
    NSTEP=200000, NOUTPUT=2000, NSTATS_START_STEP=6000, write_vti_output=1,
    sponge_cells=34,
    jet_radius=7.0, jet_velocity=0.05,
    bubble_radius=10.0,
    rhor0=1.0, rhob0=1.0,
    Re=5000.0, We=2000.0,
    beta_recolor=0.80, sponge_K=0.0,
    boundary="jet", storage="f32", seed=0, init_noise=0.0, inlet_noise=0.0,
    bubble_red_inside=0,
)

CS2 = f32(1.0 / 3.0)  # constants.cuh:45


def derive(case: dict) -> dict:
    """Fill jet/bubble centres and nu, taur, taub, sigma like constants.cuh.

    If the case gives ``tau`` (and optionally ``sigma``) directly, those win:
    nu = (tau - 0.5) * cs2, taur = taub = tau.  Otherwise
    nu = 2 R U / Re, tau = 0.5 + nu / cs2, sigma = rhob0 U^2 2R / We
    (constants.cuh:60-73), all in float32.
    """
    c = dict(REFERENCE_DEFAULT)
    c.update(case)
    NX, NY, NZ = int(c["NX"]), int(c["NY"]), int(c["NZ"])
    half = f32(2)
    c.setdefault("jet_x0", float(f32(NX - 1) / half))
    c.setdefault("jet_z0", float(f32(NZ - 1) / half))
    c.setdefault("bubble_x0", float(f32(NX - 1) / half))
    c.setdefault("bubble_y0", float(f32(NY - 1) / half))
    c.setdefault("bubble_z0", float(f32(NZ - 1) / half))
    R = f32(c["jet_radius"])
    U = f32(c["jet_velocity"])
    if "tau" in c:
        tau = f32(c["tau"])
        nu = (tau - f32(0.5)) * CS2
        c["nu"], c["taur"], c["taub"] = float(nu), float(tau), float(tau)
    else:
        nu = (f32(2) * R * U) / f32(c["Re"])
        tau = f32(0.5) + nu / CS2
        c["nu"], c["taur"], c["taub"] = float(nu), float(tau), float(tau)
    if "sigma" not in c:
        c["sigma"] = float((f32(c["rhob0"]) * U * U * f32(2.0) * R) / f32(c["We"]))
    return c


# ---------------------------------------------------------------------------
# The workloads.  Sizes count the ghost shell like the reference.
# ---------------------------------------------------------------------------
CASES = {
    # Static bubble: 64^3, radius 16, tau 0.8, sigma 0.01, beta 0.7, 2000 steps.
    # "periodic" is the physics run (Laplace jump, spurious currents);
    # "bubble_64_ref" is the same case under the reference's own bubble
    # semantics (x,z wrap, y ghost planes frozen) for parity with its build.
    "bubble_64": dict(NX=64, NY=64, NZ=64, bubble_radius=16.0, tau=0.8, sigma=0.01, beta_recolor=0.7,
                      NSTEP=2000, NOUTPUT=500, NSTATS_START_STEP=10**9, boundary="periodic",
                      bubble_red_inside=1, seed=20260101, init_noise=1e-6, Re=1.0, We=1.0),
    "bubble_64_ref": dict(NX=64, NY=64, NZ=64, bubble_radius=16.0, tau=0.8, sigma=0.01, beta_recolor=0.7,
                          NSTEP=2000, NOUTPUT=500, NSTATS_START_STEP=10**9, boundary="closed",
                          Re=1.0, We=1.0),
    # Round jet: 128x256x128, D=16, U=0.05, tau=0.52 (Re=120), sigma=0.005 (We=8),
    # beta 0.8, stats from step 10000 of 20000.
    "jet_128x256x128": dict(NX=128, NY=256, NZ=128, jet_radius=8.0, jet_velocity=0.05, Re=120.0, We=8.0,
                            beta_recolor=0.8, NSTEP=20000, NOUTPUT=2000, NSTATS_START_STEP=10000,
                            boundary="jet"),
    # Same jet, 256x512x256, D=32 (Re=240, We=16), 40000 steps, stats from 20000.
    "jet_256x512x256": dict(NX=256, NY=512, NZ=256, jet_radius=16.0, jet_velocity=0.05, Re=240.0, We=16.0,
                            beta_recolor=0.8, NSTEP=40000, NOUTPUT=4000, NSTATS_START_STEP=20000,
                            boundary="jet"),
    # 64x128x64 crop of the large jet with the same tau and sigma (D=8).
    "jet_64x128x64": dict(NX=64, NY=128, NZ=64, jet_radius=4.0, jet_velocity=0.05, Re=60.0, We=4.0,
                          beta_recolor=0.8, NSTEP=10000, NOUTPUT=1000, NSTATS_START_STEP=5000,
                          boundary="jet"),
    # Deforming bubble for the adjoint: 96^3 periodic, radius 20, tau 0.7, sigma 0.01.
    "adjoint_bubble_96": dict(NX=96, NY=96, NZ=96, bubble_radius=20.0, tau=0.7, sigma=0.01, beta_recolor=0.7,
                              NSTEP=400, NOUTPUT=400, NSTATS_START_STEP=10**9, boundary="periodic",
                              bubble_red_inside=1, Re=1.0, We=1.0),
    # Small cases the CPU oracle finishes in seconds.
    "bubble_24_ref": dict(NX=24, NY=24, NZ=24, bubble_radius=6.0, tau=0.8, sigma=0.01, beta_recolor=0.7,
                          NSTEP=100, NOUTPUT=100, NSTATS_START_STEP=10**9, boundary="closed", Re=1.0, We=1.0),
    "jet_24x40x24": dict(NX=24, NY=40, NZ=24, jet_radius=3.0, jet_velocity=0.05, Re=45.0, We=3.0,
                         beta_recolor=0.8, NSTEP=100, NOUTPUT=50, NSTATS_START_STEP=20, boundary="jet"),
    "jet_32x48x32": dict(NX=32, NY=48, NZ=32, jet_radius=4.0, jet_velocity=0.05, Re=60.0, We=4.0,
                         beta_recolor=0.8, NSTEP=100, NOUTPUT=50, NSTATS_START_STEP=20, boundary="jet"),
}


def get_case(name: str, **overrides) -> dict:
    """Derived parameter dict of a named case, with overrides applied first."""
    c = copy.deepcopy(CASES[name])
    c.update(overrides)
    out = derive(c)
    out["name"] = name
    return out
