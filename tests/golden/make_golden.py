"""Generate golden fixtures from the reference's own CUDA build.

The reference ships no tests or golden vectors.  These fixtures are outputs of
the reference itself: its kernels.cu / launch.cuh compiled for sm_100a per
case by oracle/build_ref.sh (binaries oracle/_ref/ref_<case>), run on a B200
from the reference's own initial condition (launch_bubble, or launch_jetDensity
+ launch_Injet) through the launch sequence of main.cu:52-82.  Run on a
machine with a GPU and the reference build present:

    python tests/golden/make_golden.py [out_dir]

Each fixture keeps, for interior nodes, rhor, rhob, ux, uy, uz (float32), a
seeded sample of 4096 population entries per colour, the radial sums and
counts, and the total kinetic energy.  tests/test_oracle.py checks the CPU
oracle against them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from helpers import interior, run_reference  # noqa: E402
from multicomponent_color_gradient_b200 import get_case  # noqa: E402

# (case, steps, first statistics step)
GOLDEN = [("bubble_24_ref", 100, 10**9), ("jet_24x40x24", 100, 20), ("jet_32x48x32", 60, 10)]


def sample_index(case, n=4096, seed=99):
    m = np.flatnonzero(interior(case))
    rng = np.random.default_rng(seed)
    nodes = rng.choice(m, size=n, replace=True)
    dirs = rng.integers(0, 27, size=n)
    return dirs.astype(np.int64) * (case["NX"] * case["NY"] * case["NZ"]) + nodes.astype(np.int64)


def main(out_dir=HERE):
    for name, steps, stats_from in GOLDEN:
        case = get_case(name)
        R = run_reference(name, case, steps, stats_from)
        m = interior(case)
        idx = sample_index(case)
        np.savez_compressed(
            os.path.join(out_dir, f"ref_{name}.npz"),
            steps=steps, stats_from=stats_from,
            rhor=R["rhor"][m], rhob=R["rhob"][m], ux=R["ux"][m], uy=R["uy"][m], uz=R["uz"][m],
            pop_index=idx, fr_sample=R["fr"][idx], fb_sample=R["fb"][idx],
            sum_uy=R["sum_uy"], sum_uy2=R["sum_uy2"], sum_ur=R["sum_ur"], sum_ur2=R["sum_ur2"],
            sum_uruy=R["sum_uruy"], count=R["count"], tke=R["tke"])
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
