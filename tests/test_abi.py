"""C ABI checks that need no GPU: the library loads, exports every symbol
include/mcg.h declares, the params struct matches the C layout, parameter
derivation matches constants.cuh, and calls fail cleanly without a device."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from multicomponent_color_gradient_b200 import _lib, get_case
from multicomponent_color_gradient_b200.cases import derive
from multicomponent_color_gradient_b200.solver import params_struct

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mcg.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mcg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 40
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\sT\s+(mcg_\w+)", out.stdout))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(lib, n)
    # every declared function has a ctypes signature in the binding
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_params_struct_layout_matches_c():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "mcg.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(mcg_params), offsetof(mcg_params, jet_radius),
         offsetof(mcg_params, boundary), offsetof(mcg_params, seed), offsetof(mcg_params, bubble_red_inside),
         offsetof(mcg_params, reserved));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as td:
        cfile = os.path.join(td, "t.c")
        open(cfile, "w").write(src)
        exe = os.path.join(td, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), cfile, "-o", exe], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    P = _lib.McgParams
    assert vals == [C.sizeof(P), P.jet_radius.offset, P.boundary.offset, P.seed.offset,
                    P.bubble_red_inside.offset, P.reserved.offset]


def test_default_params_are_constants_cuh():
    lib = _lib.load()
    p = _lib.McgParams()
    assert lib.mcg_params_default(C.byref(p)) == 0
    assert (p.NX, p.NY, p.NZ, p.NSTEP, p.NOUTPUT, p.NSTATS_START_STEP) == (128, 400, 128, 200000, 2000, 6000)
    # constants.cuh:60-73 in float32
    f = np.float32
    nu = (f(2) * f(7.0) * f(0.05)) / f(5000)
    assert np.float32(p.nu) == nu
    assert np.float32(p.taub) == f(0.5) + nu / f(1.0 / 3.0)
    assert np.float32(p.sigma) == (f(1) * f(0.05) * f(0.05) * f(2.0) * f(7.0)) / f(2000)
    assert np.float32(p.jet_x0) == f(127) / f(2)


@pytest.mark.parametrize("name", ["jet_128x256x128", "jet_256x512x256", "jet_64x128x64", "jet_24x40x24"])
def test_python_derivation_matches_c(name):
    """cases.derive (used for the reference build's constants) == mcg_params_derive."""
    lib = _lib.load()
    c = get_case(name)
    p = params_struct(c)
    q = _lib.McgParams.from_buffer_copy(p)
    assert lib.mcg_params_derive(C.byref(q)) == 0
    for k in ("nu", "taur", "taub", "sigma", "jet_x0", "jet_z0", "bubble_x0", "bubble_y0", "bubble_z0"):
        assert np.float32(getattr(q, k)) == np.float32(c[k]), k


def test_tau_cases_give_the_requested_tau():
    c = get_case("bubble_64")
    assert np.float32(c["taub"]) == np.float32(0.8)
    assert np.float32(c["sigma"]) == np.float32(0.01)
    lib = _lib.load()
    p = params_struct(c)
    assert lib.mcg_params_set_tau(C.byref(p), C.c_float(0.8)) == 0
    assert np.float32(p.nu) == np.float32(c["nu"])
    assert lib.mcg_params_set_tau(C.byref(p), C.c_float(0.5)) == 1  # tau <= 0.5 rejected


def test_jet_config_maps_to_reference_constants():
    """128x256x128, D=16, tau=0.52, sigma=0.005 <=> jet_radius 8, Re 120, We 8."""
    c = get_case("jet_128x256x128")
    assert abs(c["taub"] - 0.52) < 1e-6
    assert abs(c["sigma"] - 0.005) < 1e-9
    c = get_case("jet_256x512x256")
    assert abs(c["taub"] - 0.52) < 1e-6 and abs(c["sigma"] - 0.005) < 1e-9


def test_constants_header_is_parsed_by_post_regex():
    """post/case_config.py:30-35 and post/mean_profile_io.py:12-18 regex-parse constants.cuh."""
    lib = _lib.load()
    c = get_case("jet_128x256x128")
    p = params_struct(c)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "constants.cuh")
        assert lib.mcg_write_constants_header(C.byref(p), path.encode()) == 0
        text = open(path).read()

    def parse(name):
        m = re.search(rf"{name}\s*=\s*(?:static_cast<[^>]+>\()?([0-9.+\-eE]+)", text)
        return float(m.group(1))

    assert parse("NX") == 128 and parse("NY") == 256 and parse("NZ") == 128
    assert parse("jet_radius") == 8.0 and abs(parse("jet_velocity") - 0.05) < 1e-9
    assert round(parse("Re")) == 120 and round(parse("We")) == 8
    assert parse("NOUTPUT") == 2000
    assert np.float32(parse("taub")) == np.float32(c["taub"])


def test_calls_fail_cleanly_without_device():
    lib = _lib.load()
    if lib.mcg_device_count() > 0:
        pytest.skip("a GPU is visible")
    p = params_struct(get_case("bubble_24_ref"))
    h = C.c_void_p()
    st = lib.mcg_create(C.byref(p), C.byref(h))
    assert st == 9 and not h.value
    assert b"device" in lib.mcg_last_error_string()


def test_invalid_params_rejected():
    lib = _lib.load()
    c = get_case("bubble_24_ref")
    for k, v in (("NX", 2), ("taub", 0.5), ("beta_recolor", 1.5), ("boundary", 7), ("storage", 3)):
        p = params_struct(c)
        setattr(p, k, v)
        h = C.c_void_p()
        assert lib.mcg_create(C.byref(p), C.byref(h)) == 1, k
        assert not h.value
    assert lib.mcg_create(None, None) == 1
    assert lib.mcg_status_string(4) == b"non-finite value"
    assert lib.mcg_abi_version() == 1
