"""Case headers for compiling the reference's own CUDA sources (test infrastructure).

The reference is configured only through compile-time constants
(constants.cuh:8-76).  To build it for one of this project's cases without
touching its sources, build_ref.sh pre-includes (nvcc ``-include``) a header
generated here.  The header defines the reference's include guard
``CONSTANTS_CUH`` and every name constants.cuh defines, so the reference's own
constants.cuh is skipped and all its files see the case values.  Derived
quantities (nu, taur, taub, sigma) are written as exact float literals taken
from ``multicomponent_color_gradient_b200.cases.derive`` so the reference build
and this project's solver use bit-identical constants.

Usage: python oracle/ref_constants.py <case> <out_header>
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from multicomponent_color_gradient_b200.cases import get_case  # noqa: E402

# Cases the reference is compiled for (one binary each, shapes are compile-time).
REF_CASES = ["bubble_24_ref", "jet_24x40x24", "jet_32x48x32", "bubble_64_ref", "jet_128x256x128",
             "jet_256x512x256"]


def flt(v: float) -> str:
    """Float literal that round-trips float32 exactly."""
    return f"static_cast<real_t>({float(np.float32(v)).hex()})"


def header_text(c: dict) -> str:
    L = []
    a = L.append
    a("// Generated by oracle/ref_constants.py for case '%s'. Test infrastructure only." % c["name"])
    a("#ifndef CONSTANTS_CUH")
    a("#define CONSTANTS_CUH")
    a("#include <array>")
    a("#include <cstddef>")
    a('#include "utilities/types.cuh"')
    a("inline constexpr int NSTEP = %d;" % int(c["NSTEP"]))
    a("inline constexpr int NOUTPUT = %d;" % int(c["NOUTPUT"]))
    a("inline constexpr int NSTATS_START_STEP = %d;" % int(min(c["NSTATS_START_STEP"], 2**31 - 1)))
    a("inline constexpr bool write_vti_output = %s;" % ("true" if c["write_vti_output"] else "false"))
    a("inline constexpr label_t NX = static_cast<label_t>(%d);" % c["NX"])
    a("inline constexpr label_t NZ = static_cast<label_t>(%d);" % c["NZ"])
    a("inline constexpr label_t NY = static_cast<label_t>(%d);" % c["NY"])
    a("inline constexpr label_t sponge_cells = static_cast<label_t>(%d);" % c["sponge_cells"])
    a("inline constexpr label_t Ncells = NX * NY * NZ;")
    a("inline constexpr label_t NR_BINS = NX / static_cast<label_t>(2);")
    a("inline constexpr label_t NradialProfileCells = NY * NR_BINS;")
    a("inline constexpr label_t Q = 27;")
    a("inline constexpr std::size_t bytesCell = std::size_t(Ncells) * sizeof(real_t);")
    a("inline constexpr std::size_t fSize = std::size_t(Ncells) * (std::size_t)Q;")
    a("inline constexpr std::size_t bytesF = fSize * sizeof(pop_t);")
    for k in ("jet_radius", "jet_x0", "jet_z0", "jet_velocity", "bubble_radius", "bubble_x0", "bubble_y0",
              "bubble_z0"):
        a("inline constexpr real_t %s = %s;" % (k, flt(c[k])))
    a("inline constexpr real_t pi = static_cast<real_t>(3.141592653589793);")
    # lattice constants: same expressions as the reference so they fold identically
    a("inline constexpr real_t cs2 = static_cast<real_t>(1.0 / 3.0);")
    a("inline constexpr real_t cs4 = cs2 * cs2;")
    a("inline constexpr real_t cs6 = cs4 * cs2;")
    a("inline constexpr real_t inv_cs2 = static_cast<real_t>(1) / cs2;")
    a("inline constexpr real_t inv_2cs2 = static_cast<real_t>(1) / (static_cast<real_t>(2) * cs2);")
    a("inline constexpr real_t inv_2cs4 = static_cast<real_t>(1) / (static_cast<real_t>(2) * cs4);")
    a("inline constexpr real_t inv_6cs6 = static_cast<real_t>(1.0) / (static_cast<real_t>(6.0) * cs6);")
    a("inline constexpr real_t inv_2cs6 = static_cast<real_t>(1.0) / (static_cast<real_t>(2.0) * cs6);")
    for k in ("rhor0", "rhob0", "Re", "nu", "taur", "taub"):
        a("inline constexpr real_t %s = %s;" % (k, flt(c[k])))
    a("inline constexpr real_t omegar = static_cast<real_t>(1) / taur;")
    a("inline constexpr real_t omegab = static_cast<real_t>(1) / taub;")
    for k in ("We", "sigma", "beta_recolor"):
        a("inline constexpr real_t %s = %s;" % (k, flt(c[k])))
    a("inline constexpr real_t sigma_over_4cs4 = sigma / (static_cast<real_t>(4) * cs4);")
    a("#endif")
    return "\n".join(L) + "\n"


def main() -> None:
    name, out = sys.argv[1], sys.argv[2]
    c = get_case(name)
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    text = header_text(c)
    if os.path.exists(out) and open(out).read() == text:
        return  # unchanged: keep the timestamp so build_ref.sh does not rebuild
    with open(out, "w") as fh:
        fh.write(text)


if __name__ == "__main__":
    if len(sys.argv) == 2 and sys.argv[1] == "--list":
        print(" ".join(REF_CASES))
    else:
        main()
