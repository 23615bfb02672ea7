"""The output files against the reference's own writers, compiled from the
reference sources into oracle/_ref (oracle/ref_dump.cu modes `vti` and
`outputs`).

* VTI: write_vti (io/save_data.cuh:137-200) and mcg_write_vti on the same five
  float32 fields give byte-identical files.
* The whole output tree of the jet main loop (main.cu:17-120; jet 24x40x24,
  NSTEP 100, NOUTPUT 50, statistics from step 20): the reference binary run
  with its own writers (meanF/meanFieldsRT.cuh:93-381) against this
  package's C++ driver bin/mcg_jet with the same constants.  The same files
  by the same relative paths; case_info.txt, radial_profile_metadata.txt and
  radial_count.bin byte for byte; the VTI files byte for byte outside their
  base64 payloads, whose decoded fields agree within 2e-5; the radial sums
  within 2e-5 per sample; the kinetic-energy files within 1e-4 relative.
"""
import base64
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from conftest import ref_binary
from multicomponent_color_gradient_b200 import Solver, get_case

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NAME = "jet_24x40x24"
PAYLOAD = re.compile(rb"(format=\"binary\">\n)([A-Za-z0-9+/=]+)(\n)")


def _binary():
    b = ref_binary(NAME)
    if b is None:
        pytest.skip(f"reference build oracle/_ref/ref_{NAME} not present")
    return b


def _split_vti(data: bytes):
    """(text with the base64 payloads blanked, decoded float32 arrays)."""
    arrays = []

    def blank(m):
        raw = base64.b64decode(m.group(2), validate=True)
        n = struct.unpack("<Q", raw[:8])[0]
        assert n == len(raw) - 8
        arrays.append(np.frombuffer(raw[8:], np.float32))
        return m.group(1) + b"<payload>" + m.group(3)

    return PAYLOAD.sub(blank, data), arrays


def test_vti_bytes_equal_reference_writer(tmp_path):
    binary = _binary()
    case = get_case(NAME)
    N = case["NX"] * case["NY"] * case["NZ"]
    rng = np.random.default_rng(23)
    fields = {"rhor": rng.uniform(0, 1, N), "rhob": rng.uniform(0, 1, N), "ux": rng.normal(0, 0.01, N),
              "uy": rng.normal(0.02, 0.01, N), "uz": rng.normal(0, 0.01, N)}
    fields = {k: v.astype(np.float32) for k, v in fields.items()}
    np.concatenate([fields[k] for k in ("rhor", "rhob", "ux", "uy", "uz")]).tofile(tmp_path / "fields.bin")
    subprocess.run([binary, "vti", str(tmp_path / "fields.bin"), str(tmp_path / "ref.vti")], check=True, timeout=120)
    with Solver(case) as S:
        S.set_fields(**fields)
        S.write_vti(str(tmp_path / "ours.vti"))
    ref = (tmp_path / "ref.vti").read_bytes()
    ours = (tmp_path / "ours.vti").read_bytes()
    assert len(ref) > 100000
    assert ours == ref


def _tree(root):
    return sorted(os.path.relpath(os.path.join(d, f), root) for d, _, fs in os.walk(root) for f in fs)


def test_output_tree_matches_reference_main_loop(tmp_path):
    binary = _binary()
    exe = os.path.join(ROOT, "multicomponent_color_gradient_b200", "bin", "mcg_jet")
    if not os.path.exists(exe):
        pytest.skip("bin/mcg_jet not built")
    case = get_case(NAME)
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    ref_dir.mkdir()
    subprocess.run([binary, "outputs", str(ref_dir)], check=True, capture_output=True, timeout=300)
    args = [exe, "--NX", "24", "--NY", "40", "--NZ", "24", "--jet_radius", "3", "--Re", "45", "--We", "3",
            "--NSTEP", str(case["NSTEP"]), "--NOUTPUT", str(case["NOUTPUT"]), "--NSTATS_START_STEP",
            str(case["NSTATS_START_STEP"]), "--out", str(our_dir)]
    out = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    files = _tree(ref_dir)
    assert files == _tree(our_dir)
    assert "JET_VTK/Re45_We3/case_info.txt" in files and "JET_VTK/Re45_We3/vti_data/lbm_00000050.vti" in files
    NY, NRB = case["NY"], case["NX"] // 2
    count = np.fromfile(ref_dir / "JET_VTK/Re45_We3/mean_profiles/radial_count.bin", np.uint64)
    assert count.size == NY * NRB and count.max() > 0
    cnt = np.maximum(count.astype(np.float64), 1.0)
    for f in files:
        a, b = (ref_dir / f).read_bytes(), (our_dir / f).read_bytes()
        name = os.path.basename(f)
        if name in ("case_info.txt", "radial_profile_metadata.txt", "radial_count.bin"):
            assert a == b, f
        elif name.startswith("radial_sum_"):
            x, y = np.frombuffer(a, np.float64), np.frombuffer(b, np.float64)
            assert x.shape == y.shape == (NY * NRB,), f
            assert np.max(np.abs(x - y) / cnt) <= 2e-5, f
        elif name.startswith("tke_"):
            x, y = np.frombuffer(a, np.float32), np.frombuffer(b, np.float32)
            assert x.shape == y.shape and x.size == case["NSTEP"] // case["NOUTPUT"], f
            scale = np.max(np.abs(np.frombuffer((ref_dir / f).with_name("tke_total.bin").read_bytes(), np.float32)))
            np.testing.assert_allclose(y, x, rtol=1e-4, atol=1e-4 * scale, err_msg=f)
        elif name.endswith(".vti"):
            ta, xa = _split_vti(a)
            tb, xb = _split_vti(b)
            assert ta == tb, f
            assert len(xa) == len(xb) == 4
            for u, v in zip(xa, xb):
                assert u.shape == v.shape and np.max(np.abs(u.astype(np.float64) - v)) <= 2e-5, f
        else:
            pytest.fail(f"unexpected file {f}")
