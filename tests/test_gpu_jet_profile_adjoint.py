"""The jet adjoint for the misfit of time-averaged profiles, and the float32
adjoint over a float16-stored forward run.

Profile objective (mcg_adjoint_jet_profile_run), on the jet 24x40x24 (D = 6,
Re 45, We 3) with inlet-profile coefficients c = (0.1, -0.05, 0.02, 0, ...):
T = 160 steps, the radial statistics of steps 80..159 give the mean profiles
U(y, r), their centreline velocity uc(y) and half-width r_half(y) as the
reference's post/plot_profiles.py:53-91 forms them, and
  J = 1/2 sum_{2 <= y <= 7} ((uc - uc*)/U)^2 + ((r_half - r_half*)/D)^2
against the profiles of a target run with c* = (0.16, -0.02, 0.05, 0.03, 0, ...).
Checks: the C ABI's metrics equal the Python restatement on the same sums;
J equals the objective of the GPU's own forward run (1e-5) and of the
float64 oracle (1e-3: the half-width divides small velocity differences);
dJ/dc_k equals float64 central differences of the oracle's J (steps 0.02
and 0.01, Richardson extrapolation) within 1e-3 relative.

Float16 storage (mcg_adjoint_jet_run on a float16 handle): the forward states
are stored in float16 and the reverse sweep is the float32 adjoint of the
step at those states; J and dJ/dc within 1 % of the all-float32 adjoint.
"""
import numpy as np
import pytest

from multicomponent_color_gradient_b200 import Solver, get_case
from multicomponent_color_gradient_b200.post import profile_metrics, profile_objective
from oracle.oracle import Oracle
from test_gpu_jet_adjoint import multipliers

pytestmark = pytest.mark.gpu

T, T0, T1 = 160, 80, 159
Y_LO, Y_HI = 2, 7
C0 = np.array([0.1, -0.05, 0.02, 0, 0, 0, 0, 0], np.float64)
C_TARGET = np.array([0.16, -0.02, 0.05, 0.03, 0, 0, 0, 0], np.float64)


def case(**kw):
    return get_case("jet_24x40x24", NSTATS_START_STEP=T0, **kw)


def scales(c):
    return float(c["jet_velocity"]), 2.0 * float(c["jet_radius"])


def metrics_of(radial, c):
    return profile_metrics(radial["sum_uy"], radial["count"], c["NX"], c["NZ"], c["jet_x0"], c["jet_z0"])


def gpu_profiles(coeffs, storage="f32"):
    c = case(storage=storage)
    with Solver(c) as S:
        S.set_inlet_bessel(np.asarray(coeffs, np.float32))
        S.init_jet()
        S.step(T1 + 1)
        uc, rh = S.jet_profile_metrics()
        radial = S.get_radial()
    return uc, rh, radial


def oracle_profiles(coeffs):
    c = case()
    O = Oracle(c, 64)
    O.set_inlet_profile(multipliers(coeffs))
    O.init_jet()
    O.step(T1 + 1)
    return metrics_of(O.get_radial(), c)


@pytest.fixture(scope="module")
def target():
    uc, rh, _ = gpu_profiles(C_TARGET)
    return uc, rh


@pytest.fixture(scope="module")
def adjoint(target):
    with Solver(case()) as S:
        S.set_inlet_bessel(C0.astype(np.float32))
        S.init_jet()
        return S.adjoint_jet_profile_run(T, T0, T1, Y_LO, Y_HI, target[0], target[1])


def test_profile_metrics_match_python_restatement():
    uc, rh, radial = gpu_profiles(C0)
    puc, prh = metrics_of(radial, case())
    print("uc", uc[Y_LO:Y_HI + 1], "r_half", rh[Y_LO:Y_HI + 1])
    assert np.isfinite(uc[Y_LO:Y_HI + 1]).all() and np.isfinite(rh[Y_LO:Y_HI + 1]).all()
    np.testing.assert_allclose(uc, puc, rtol=1e-6, atol=1e-12, equal_nan=True)
    np.testing.assert_allclose(rh, prh, rtol=1e-5, atol=1e-9, equal_nan=True)


def test_profile_J_matches_forward_runs(adjoint, target):
    c = case()
    U, D = scales(c)
    uc, rh, _ = gpu_profiles(C0)
    J = profile_objective(uc, rh, target[0], target[1], Y_LO, Y_HI, U, D)
    ouc, orh = oracle_profiles(C0)
    Jo = profile_objective(ouc, orh, target[0], target[1], Y_LO, Y_HI, U, D)
    print(f"profile J adjoint={adjoint['J']:.8e} forward={J:.8e} fp64 oracle={Jo:.8e}")
    assert J > 0
    assert abs(adjoint["J"] - J) <= 1e-5 * J
    assert abs(adjoint["J"] - Jo) <= 1e-3 * Jo


@pytest.mark.parametrize("k", [0, 1, 3])
def test_profile_dJ_dc_matches_fp64_central_differences(adjoint, target, k):
    c = case()
    U, D = scales(c)

    def J_of(coeffs):
        uc, rh = oracle_profiles(coeffs)
        return profile_objective(uc, rh, target[0], target[1], Y_LO, Y_HI, U, D)

    def d(h):
        cp, cm = C0.copy(), C0.copy()
        cp[k] += h
        cm[k] -= h
        return (J_of(cp) - J_of(cm)) / (2 * h)

    d1, d2 = d(0.02), d(0.01)
    fd = (4.0 * d2 - d1) / 3.0
    g = adjoint["dJ_dc"][k]
    print(f"profile dJ/dc[{k}] adjoint={g:.7e} fd={fd:.7e} (h=0.02: {d1:.7e}, h=0.01: {d2:.7e})")
    assert abs(g - fd) <= 1e-3 * abs(fd), (k, g, fd)


@pytest.mark.parametrize("tapes", [1, 2])
def test_profile_segments_give_the_same_gradients(adjoint, target, tapes):
    """Snapshots every 48 steps (segments of 48, 48, 48, 16).  The first pass
    runs through the window's end, the last step, so the last `tapes` segments
    are recorded there and only the others are re-run."""
    with Solver(case()) as S:
        S.set_inlet_bessel(C0.astype(np.float32))
        S.init_jet()
        S.set_jet_adjoint_tapes(tapes)
        r = S.adjoint_jet_profile_run(T, T0, T1, Y_LO, Y_HI, target[0], target[1], segment=48)
    lengths = [48, 48, 48, 16]
    assert r["forward_steps"] == T + sum(lengths[:len(lengths) - tapes])
    assert abs(r["J"] - adjoint["J"]) <= 1e-12 * adjoint["J"]
    np.testing.assert_allclose(r["dJ_dc"], adjoint["dJ_dc"], rtol=1e-6, atol=1e-15)


def test_float16_forward_under_float32_adjoint():
    out = {}
    for storage in ("f32", "f16"):
        with Solver(case(storage=storage)) as S:
            S.set_inlet_bessel(C0.astype(np.float32))
            S.init_jet()
            out[storage] = S.adjoint_jet_run(40, 20, 39, 20)
    a, b = out["f32"], out["f16"]
    print(f"J f32 {a['J']:.6e} f16 {b['J']:.6e}; dJ/dc f32 {a['dJ_dc'][:3]} f16 {b['dJ_dc'][:3]}")
    assert abs(b["J"] - a["J"]) <= 1e-2 * a["J"]
    for k in (0, 1, 2, 5):
        assert abs(b["dJ_dc"][k] - a["dJ_dc"][k]) <= 1e-2 * abs(a["dJ_dc"][k]), k
