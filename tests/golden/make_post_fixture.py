"""Writes the output tree of a short jet run with this solver, the fixture that
tests/test_post_compat.py feeds to the reference's post/ readers.

Needs a GPU.  jet 24x40x24 (Re 45, We 3), NOUTPUT 20, statistics from step 10,
61 steps as main.cu:52-104 runs them, then the radial outputs and three
update_uy_average samples.  VTI output is off (the VTI text is covered by
tests/test_outputs.py).

    python tests/golden/make_post_fixture.py OUT_ROOT
    # then copy OUT_ROOT/JET_VTK to tests/golden/post_jet_24x40x24/JET_VTK
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from multicomponent_color_gradient_b200 import Solver, get_case  # noqa: E402


def main(out_root: str) -> None:
    case = get_case("jet_24x40x24", NOUTPUT=20, NSTATS_START_STEP=10, write_vti_output=0, NSTEP=61)
    with Solver(case) as S:
        S.output_open(out_root)
        S.init_jet()
        for step in range(case["NSTEP"]):
            S.step(1)
            if step % case["NOUTPUT"] == 0:
                S.output_step(step)
        S.write_radial_outputs()
        for _ in range(3):
            S.launch_update_uy_average()
        S.write_uy_average()
        print("wrote", S.output_dirs()[0])


if __name__ == "__main__":
    main(sys.argv[1])
