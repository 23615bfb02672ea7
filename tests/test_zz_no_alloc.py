"""mcg_conservation_sums_static: the float64 population sums for callers that
cannot let the library allocate (they own all device memory and allow no
cudaMalloc/cudaFree inside their time loop).  Called through the C ABI on
device buffers the test owns, and checked against the handle-based
mcg_conservation_sums on two calls in a row; the second call must not see the
first call's scratch contents.  The calls leave the device's free memory
unchanged, also run on a non-default stream, and a call on a grid with fewer
z planes than the one before reads only the slots it wrote itself."""
import ctypes as C

import numpy as np
import pytest

from multicomponent_color_gradient_b200 import Solver, _lib, get_case

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-12, 1e-9  # float64 sums of the same float32 values, different order


def _static_sums(lib, fr_d, fb_d, case, out_d, stream=None):
    import torch

    handle = None if stream is None else C.c_void_p(stream.cuda_stream)
    st = lib.mcg_conservation_sums_static(C.c_void_p(fr_d.data_ptr()), C.c_void_p(fb_d.data_ptr()),
                                          int(case["NX"]), int(case["NY"]), int(case["NZ"]),
                                          C.c_void_p(out_d.data_ptr()), handle)
    assert st == 0, lib.mcg_last_error_string()
    torch.cuda.synchronize()
    return out_d.cpu().numpy()


def _device_state(S):
    import torch

    fr, fb = S.get_populations()
    fr_d = torch.from_numpy(fr).cuda()
    fb_d = torch.from_numpy(fb).cuda()
    torch.cuda.synchronize()
    return fr_d, fb_d


def test_static_scratch_sums_match_handle_sums_twice():
    import torch

    lib = _lib.load()
    case = get_case("jet_32x48x32", NSTATS_START_STEP=10)
    S = Solver(case)
    S.init_jet()
    out_d = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
    previous = None
    for _ in range(2):
        S.step(25)
        expected = S.conservation_sums()
        fr_d, fb_d = _device_state(S)
        got = _static_sums(lib, fr_d, fb_d, case, out_d)
        np.testing.assert_allclose(got, expected, rtol=RTOL, atol=ATOL)
        if previous is not None:
            assert not np.array_equal(got, previous)  # a fresh result, not the last call's
        previous = got
    S.close()


def test_static_scratch_allocates_nothing_and_runs_on_a_stream():
    """After a first call (which looks up the scratch address and loads the
    kernels), further calls change the device's free memory by nothing; a call
    on a non-default stream gives the same sums."""
    import torch

    lib = _lib.load()
    case = get_case("jet_32x48x32", NSTATS_START_STEP=10)
    with Solver(case) as S:
        S.init_jet()
        S.step(20)
        expected = S.conservation_sums()
        fr_d, fb_d = _device_state(S)
    out_d = torch.zeros(5, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    _static_sums(lib, fr_d, fb_d, case, out_d)
    _static_sums(lib, fr_d, fb_d, case, out_d, stream=side)
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        got = _static_sums(lib, fr_d, fb_d, case, out_d)
        np.testing.assert_allclose(got, expected, rtol=RTOL, atol=ATOL)
    out_d.fill_(float("nan"))
    torch.cuda.synchronize()
    got = _static_sums(lib, fr_d, fb_d, case, out_d, stream=side)
    np.testing.assert_allclose(got, expected, rtol=RTOL, atol=ATOL)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_static_scratch_smaller_grid_after_larger_grid():
    """A grid of 30 interior planes, then one of 22: the second call folds
    only the 22 slots it wrote (slots 22..29 still hold the first call's
    partials) and matches its own handle sums."""
    import torch

    lib = _lib.load()
    out_d = torch.zeros(5, dtype=torch.float64, device="cuda")
    for name in ("jet_32x48x32", "jet_24x40x24"):
        case = get_case(name, NSTATS_START_STEP=5)
        with Solver(case) as S:
            S.init_jet()
            S.step(15)
            expected = S.conservation_sums()
            fr_d, fb_d = _device_state(S)
        got = _static_sums(lib, fr_d, fb_d, case, out_d)
        np.testing.assert_allclose(got, expected, rtol=RTOL, atol=ATOL)


def test_static_scratch_rejects_too_many_planes():
    import torch

    lib = _lib.load()
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    out_d = torch.zeros(5, dtype=torch.float64, device="cuda")
    nz = 4096 + 3  # NZ - 2 = 4097 interior planes > MCG_STATIC_SCRATCH_PLANES
    st = lib.mcg_conservation_sums_static(C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), 4, 4, nz,
                                          C.c_void_p(out_d.data_ptr()), None)
    assert st == 1
    assert b"static scratch" in lib.mcg_last_error_string()
    assert lib.mcg_conservation_sums_static(None, None, 8, 8, 8, None, None) == 1
