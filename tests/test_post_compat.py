"""The post/ file contract end to end, on the CPU: the output tree of a short
jet run with this solver (tests/golden/post_jet_24x40x24, written by
tests/golden/make_post_fixture.py on a GPU) read back

* by the reference's own post/mean_profile_io.py (read_metadata,
  read_radial_moments, require_samples, averaged_radial_fields,
  fit_virtual_origin: post/mean_profile_io.py:61-239), imported from the
  reference checkout (MCG_REFERENCE_DIR, or the one oracle/build_ref.sh
  compiled from), when one is present, else skipped;
* by the package's plain-XML replacement of post/binConversionVti.py, which
  needs no vtk package.
"""
import base64
import importlib
import os
import re
import struct
import sys

import numpy as np
import pytest

from conftest import reference_dir
from multicomponent_color_gradient_b200.post import read_case_info, write_uy_avg_vti

HERE = os.path.dirname(os.path.abspath(__file__))
CASE_DIR = os.path.join(HERE, "golden", "post_jet_24x40x24", "JET_VTK", "Re45_We3")
MEAN_DIR = os.path.join(CASE_DIR, "mean_profiles")
REF_DIR = reference_dir()
REF_POST = os.path.join(REF_DIR, "post") if REF_DIR else None
NX, NY, NZ, NRB = 24, 40, 24, 12
SAMPLES = 51  # statistics from step 10 to step 60


@pytest.fixture(scope="module")
def ref_post():
    if REF_POST is None or not os.path.isfile(os.path.join(REF_POST, "mean_profile_io.py")):
        pytest.skip("the reference's post/ scripts are not present")
    sys.path.insert(0, REF_POST)
    try:
        yield importlib.import_module("mean_profile_io")
    finally:
        sys.path.remove(REF_POST)


def test_reference_reader_accepts_the_radial_files(ref_post):
    meta = ref_post.read_metadata(MEAN_DIR)
    assert (meta["NY"], meta["NR_BINS"], meta["radial_sample_count"]) == (NY, NRB, SAMPLES)
    assert meta["D"] == 6.0 and meta["uy_avg_start_step"] == 10 and meta["uy_avg_last_sample_step"] == 60
    mom = ref_post.read_radial_moments(MEAN_DIR)
    ref_post.require_samples(mom)
    for k in ("sum_uy", "sum_uy2", "sum_ur", "sum_ur2", "sum_uruy", "count"):
        assert mom[k].shape == (NY, NRB), k
    # counts: every fluid plane y = 1..NY-2 holds samples x (its columns per bin);
    # columns whose radius lies beyond the last bin (the corners) are not counted
    cnt = mom["count"].astype(np.int64)
    assert cnt[0].sum() == 0 and cnt[-1].sum() == 0
    assert np.all(cnt[1:-1] % SAMPLES == 0)
    per_plane = cnt[1:-1].sum(axis=1)
    assert np.all(per_plane == per_plane[0]) and 0 < per_plane[0] <= SAMPLES * (NX - 2) * (NZ - 2)
    f = ref_post.averaged_radial_fields(mom)
    valid = cnt > 0
    np.testing.assert_allclose(f["uy"][valid], mom["sum_uy"][valid] / cnt[valid])
    assert np.all(np.isfinite(f["uy_rms"][valid])) and np.all(f["uy_rms"][valid] >= 0)
    # the jet enters at y = 0: the centreline mean velocity is positive in the near field
    uc = f["uy"][:, 0]
    assert np.all(uc[1:12] > 0)
    y = np.arange(NY, dtype=np.float64)
    spread, y0, *_ = ref_post.fit_virtual_origin(y, uc, meta["D"], meta["U_jet"], yi_over_d=0.5, yf_over_d=1.8)
    assert np.isfinite(spread) and np.isfinite(y0)


def test_restated_reader_matches_the_reference_reader(ref_post):
    """The reader that tests/test_outputs.py uses (post/mean_profile_io.py:139-179
    restated) returns what the reference's reader returns."""
    mom = ref_post.read_radial_moments(MEAN_DIR)
    for k in ("uy", "uy2", "ur", "ur2", "uruy"):
        a = np.fromfile(os.path.join(MEAN_DIR, f"radial_sum_{k}.bin"), np.float64).reshape(NY, NRB)
        np.testing.assert_array_equal(a, mom["sum_" + k])
    c = np.fromfile(os.path.join(MEAN_DIR, "radial_count.bin"), np.uint64).reshape(NY, NRB)
    np.testing.assert_array_equal(c, mom["count"])


def test_uy_avg_vti_without_vtk(tmp_path):
    """write_uy_avg_vti writes the ImageData that post/binConversionVti.py:12-51
    writes with the vtk package: dimensions NX x NY x NZ, unit spacing, origin 0,
    one Float32 point array `uy_avg` equal to uy_avg.bin."""
    info = read_case_info(CASE_DIR)
    assert (int(info["NX"]), int(info["NY"]), int(info["NZ"])) == (NX, NY, NZ)
    out = write_uy_avg_vti(CASE_DIR, tmp_path)
    assert out == tmp_path / "uy_avg.vti"
    text = out.read_text()
    assert 'WholeExtent="0 23 0 39 0 23"' in text and 'Origin="0 0 0" Spacing="1 1 1"' in text
    m = re.search(r'<DataArray type="Float32" Name="uy_avg" format="binary">\n([A-Za-z0-9+/=]+)\n', text)
    raw = base64.b64decode(m.group(1), validate=True)
    n = struct.unpack("<Q", raw[:8])[0]
    assert n == NX * NY * NZ * 4 == len(raw) - 8
    np.testing.assert_array_equal(np.frombuffer(raw[8:], "<f4"),
                                  np.fromfile(os.path.join(MEAN_DIR, "uy_avg.bin"), "<f4"))


def test_uy_avg_vti_rejects_a_short_file(tmp_path):
    import shutil
    case = tmp_path / "case"
    shutil.copytree(CASE_DIR, case)
    with open(case / "mean_profiles" / "uy_avg.bin", "r+b") as fh:
        fh.truncate(100)
    with pytest.raises(ValueError, match="expected"):
        write_uy_avg_vti(case)


def test_vti_text_several_arrays():
    """vti_text writes the VTI layout the solver's lbm_*.vti files have: one
    Float32 point array per name, each base64 of [UInt64 byte count][payload],
    the first array named as the Scalars attribute."""
    from multicomponent_color_gradient_b200.post import vti_text

    nx, ny, nz = 3, 4, 2
    rng = np.random.default_rng(5)
    arrays = {"rhor": rng.random(nx * ny * nz, dtype=np.float32),
              "rhob": rng.random(nx * ny * nz, dtype=np.float32)}
    text = vti_text(nx, ny, nz, arrays)
    assert text.startswith('<?xml version="1.0"?>\n<VTKFile type="ImageData" version="1.0" '
                           'byte_order="LittleEndian" header_type="UInt64">\n')
    assert 'WholeExtent="0 2 0 3 0 1"' in text and '<PointData Scalars="rhor">' in text
    found = re.findall(r'<DataArray type="Float32" Name="(\w+)" format="binary">\n([A-Za-z0-9+/=]+)\n', text)
    assert [n for n, _ in found] == ["rhor", "rhob"]
    for name, b64 in found:
        raw = base64.b64decode(b64, validate=True)
        assert struct.unpack("<Q", raw[:8])[0] == len(raw) - 8
        np.testing.assert_array_equal(np.frombuffer(raw[8:], "<f4"), arrays[name])
