"""Output files: names, layouts and contents the reference writes and its post/
scripts read (meanF/meanFieldsRT.cuh:93-381, io/save_data.cuh:137-215,
post/mean_profile_io.py:139-179, post/binConversionVti.py:22-28)."""
import base64
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from multicomponent_color_gradient_b200 import Solver, get_case
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def read_kv(path):
    out = {}
    for line in open(path).read().splitlines():
        parts = line.split(maxsplit=1)
        if len(parts) == 2:
            out[parts[0]] = parts[1]
    return out


def read_radial(mean_dir, NY, NRB):
    """The reader of post/mean_profile_io.py:139-179, restated: (NY, NR_BINS) arrays."""
    out = {}
    for k in ("uy", "uy2", "ur", "ur2", "uruy"):
        a = np.fromfile(os.path.join(mean_dir, f"radial_sum_{k}.bin"), np.float64)
        assert a.size == NY * NRB
        out["sum_" + k] = a.reshape(NY, NRB)
    c = np.fromfile(os.path.join(mean_dir, "radial_count.bin"), np.uint64)
    assert c.size == NY * NRB
    out["count"] = c.reshape(NY, NRB)
    return out


def decode_vti(path):
    text = open(path, "rb").read().decode()
    assert text.startswith('<?xml version="1.0"?>\n<VTKFile type="ImageData" version="1.0" '
                           'byte_order="LittleEndian" header_type="UInt64">\n')
    arrays = {}
    for m in re.finditer(r'<DataArray type="Float32" Name="(\w+)"(?: NumberOfComponents="3")? format="binary">\n'
                         r'([A-Za-z0-9+/=]+)\n        </DataArray>', text):
        raw = base64.b64decode(m.group(2), validate=True)
        assert base64.b64encode(raw).decode() == m.group(2)  # canonical text, '=' padding
        n = struct.unpack("<Q", raw[:8])[0]
        assert n == len(raw) - 8
        arrays[m.group(1)] = np.frombuffer(raw[8:], np.float32)
    ext = re.search(r'WholeExtent="0 (\d+) 0 (\d+) 0 (\d+)"', text)
    return arrays, tuple(int(v) + 1 for v in ext.groups())


def test_output_files_match_reference_layout(tmp_path):
    case = get_case("jet_24x40x24", NOUTPUT=20, NSTATS_START_STEP=10, write_vti_output=1, NSTEP=61)
    NX, NY, NZ, N, NRB = case["NX"], case["NY"], case["NZ"], case["NX"] * case["NY"] * case["NZ"], case["NX"] // 2
    S = Solver(case)
    S.output_open(str(tmp_path))
    S.init_jet()
    O = Oracle(case, 64)
    O.init_jet()
    tke_o = []
    for step in range(61):  # main.cu:52-104
        S.step(1)
        O.step(1)
        if step % case["NOUTPUT"] == 0:
            S.output_step(step)
            tke_o.append(O.total_tke())
            F = S.get_fields()
    S.write_radial_outputs()
    # uy_avg: the running mean of kernels.cu:168-186 over three different
    # states (steps 61, 68, 75), restated in float32 numpy
    m = np.zeros((NZ, NY, NX), bool)
    m[1:-1, 1:-1, 1:-1] = True
    m = m.ravel()
    expect = np.zeros(N, np.float32)
    samples_uy = []
    for k in range(3):
        if k:
            S.step(7)
        S.launch_update_uy_average()
        uy = S.get_fields()["uy"]
        samples_uy.append(uy)
        c = np.float32(k)
        expect = np.where(m, (expect * c + uy) / (c + np.float32(1)), np.float32(0)).astype(np.float32)
    S.write_uy_average()
    case_dir, mean_dir, vti_dir = S.output_dirs()
    assert case_dir.endswith(os.path.join("JET_VTK", "Re45_We3"))
    info = read_kv(os.path.join(case_dir, "case_info.txt"))
    assert (info["NX"], info["NY"], info["NZ"], info["NOUTPUT"], info["NR_BINS"]) == ("24", "40", "24", "20", "12")
    assert float(info["jet_diameter"]) == 6.0
    # tke files: one float32 per output step (steps 0, 20, 40, 60)
    tot = np.fromfile(os.path.join(mean_dir, "tke_total.bin"), np.float32)
    avg = np.fromfile(os.path.join(mean_dir, "tke_avg.bin"), np.float32)
    diff = np.fromfile(os.path.join(mean_dir, "tke_diff.bin"), np.float32)
    assert tot.size == avg.size == diff.size == 4
    np.testing.assert_allclose(tot, tke_o, rtol=1e-4)
    assert diff[0] == 0.0
    # radial moments: post/mean_profile_io.py layout, counts = samples x columns
    R = read_radial(mean_dir, NY, NRB)
    meta = read_kv(os.path.join(mean_dir, "radial_profile_metadata.txt"))
    samples = int(meta["radial_sample_count"])
    assert samples == 51 and int(meta["uy_avg_start_step"]) == 10 and int(meta["uy_avg_last_sample_step"]) == 60
    assert R["count"][0].sum() == 0 and R["count"][-1].sum() == 0
    assert np.all(R["count"][1:-1] % samples == 0)
    OR = O.get_radial()
    np.testing.assert_array_equal(R["count"].ravel(), OR["count"])
    cnt = np.maximum(OR["count"].astype(np.float64), 1.0)
    assert np.max(np.abs(R["sum_uy"].ravel() - OR["sum_uy"]) / cnt) <= 2e-5
    # VTI of the last output step: arrays equal the fields at that step
    arrays, dims = decode_vti(os.path.join(vti_dir, "lbm_00000060.vti"))
    assert dims == (NX, NY, NZ)
    np.testing.assert_array_equal(arrays["rhor"], F["rhor"])
    np.testing.assert_array_equal(arrays["rhob"], F["rhob"])
    np.testing.assert_array_equal(arrays["rho"], F["rhor"] + F["rhob"])
    u = arrays["u"].reshape(N, 3)
    np.testing.assert_array_equal(u[:, 1], F["uy"])
    assert sorted(os.listdir(vti_dir)) == [f"lbm_{s:08d}.vti" for s in (0, 20, 40, 60)]
    # uy_avg.bin: float32 Ncells as post/binConversionVti.py:22-28 reads it
    uy_avg = np.fromfile(os.path.join(mean_dir, "uy_avg.bin"), np.float32)
    assert uy_avg.size == N
    assert not np.any(uy_avg[~m])  # ghost nodes are not averaged
    np.testing.assert_allclose(uy_avg[m], expect[m], rtol=1e-6, atol=1e-9)
    # the three samples differ, so a wrong weighting would show: the mean is
    # neither the last sample nor the first
    for u in (samples_uy[0], samples_uy[-1]):
        assert np.max(np.abs(uy_avg[m] - u[m])) > 100 * (1e-6 * np.max(np.abs(expect[m])) + 1e-9)


@pytest.mark.parametrize("async_output", ["0", "1"])
def test_cpp_driver_runs_the_main_loop(tmp_path, async_output):
    exe = os.path.join(ROOT, "multicomponent_color_gradient_b200", "bin", "mcg_jet")
    if not os.path.exists(exe):
        pytest.skip("bin/mcg_jet not built")
    out = subprocess.run([exe, "--NX", "24", "--NY", "40", "--NZ", "24", "--jet_radius", "3", "--Re", "45", "--We",
                          "3", "--NSTEP", "200", "--NOUTPUT", "100", "--NSTATS_START_STEP", "50", "--out",
                          str(tmp_path), "--async_output", async_output], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    assert "MLUPS" in out.stdout and "tke_avg" in out.stdout
    mean = tmp_path / "JET_VTK" / "Re45_We3" / "mean_profiles"
    assert (mean / "radial_sum_uy.bin").stat().st_size == 40 * 12 * 8
    assert (tmp_path / "JET_VTK" / "Re45_We3" / "vti_data" / "lbm_00000100.vti").exists()


def _run_outputs(root, asynchronous):
    case = get_case("jet_24x40x24", NOUTPUT=20, NSTATS_START_STEP=10, write_vti_output=1, NSTEP=61)
    with Solver(case) as S:
        S.output_open(str(root))
        S.init_jet()
        for step in range(61):
            S.step(1)
            if step % case["NOUTPUT"] == 0:
                S.output_step_async(step) if asynchronous else S.output_step(step)
        if asynchronous:
            S.output_flush()
        S.write_radial_outputs()
        case_dir, _, _ = S.output_dirs()
    return case_dir


def test_async_outputs_equal_sync_outputs(tmp_path):
    """mcg_output_step_async writes the same files as mcg_output_step (tke,
    radial sums and metadata, VTI) while stepping on.  The fields, VTI text and
    metadata are deterministic and compared byte for byte.  The radial sums
    and the kinetic energy are float64 atomic sums whose order changes from
    run to run, so those files are compared within a reordering tolerance."""
    a = _run_outputs(tmp_path / "sync", False)
    b = _run_outputs(tmp_path / "async", True)
    files_a = sorted(os.path.relpath(os.path.join(d, f), a) for d, _, fs in os.walk(a) for f in fs)
    files_b = sorted(os.path.relpath(os.path.join(d, f), b) for d, _, fs in os.walk(b) for f in fs)
    assert files_a == files_b and len(files_a) > 10
    for f in files_a:
        fa, fb = os.path.join(a, f), os.path.join(b, f)
        name = os.path.basename(f)
        if name.startswith("radial_sum_"):
            x, y = np.fromfile(fa, np.float64), np.fromfile(fb, np.float64)
            assert x.shape == y.shape and np.max(np.abs(x - y)) <= 1e-10 * max(np.max(np.abs(x)), 1e-30), f
        elif name.startswith("tke_"):
            x, y = np.fromfile(fa, np.float32), np.fromfile(fb, np.float32)
            np.testing.assert_allclose(x, y, rtol=1e-6, atol=1e-12, err_msg=f)
        else:
            assert open(fa, "rb").read() == open(fb, "rb").read(), f


def test_async_output_reports_a_writer_error_once(tmp_path):
    """A file the worker thread cannot write (here: the VTI directory removed
    after mcg_output_open) comes back from mcg_output_flush as an I/O error;
    the next flush is clean and later output steps write again."""
    import shutil

    from multicomponent_color_gradient_b200._lib import McgError

    case = get_case("jet_24x40x24", NOUTPUT=20, NSTATS_START_STEP=10, write_vti_output=1, NSTEP=61)
    with Solver(case) as S:
        S.output_open(str(tmp_path))
        _, _, vti_dir = S.output_dirs()
        S.init_jet()
        S.step(5)
        shutil.rmtree(vti_dir)
        S.output_step_async(5)
        with pytest.raises(McgError, match="vti"):
            S.output_flush()
        S.output_flush()  # the error was reported once
        os.makedirs(vti_dir)
        S.step(5)
        S.output_step_async(10)
        S.output_flush()
        assert os.path.exists(os.path.join(vti_dir, "lbm_00000010.vti"))
