"""Radial inlet profile (Bessel series around the top-hat) on the GPU:
the per-column multipliers against scipy's J0 and its zeros, the zero series
reproducing the top-hat step exactly, and the jet step with a profile against
the oracle given the same multipliers (tolerances of the parity tests)."""
import numpy as np
import pytest
from scipy import special

from helpers import initial_state, interior, maxabs
from multicomponent_color_gradient_b200 import Solver, get_case
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

COEFFS = np.array([0.12, -0.05, 0.03, 0.0, 0.01, -0.004, 0.002, 0.001], np.float32)


def expected_profile(case, coeffs):
    NX, NZ = case["NX"], case["NZ"]
    x = np.arange(NX, dtype=np.float32) - np.float32(case["jet_x0"])
    z = np.arange(NZ, dtype=np.float32) - np.float32(case["jet_z0"])
    r = np.sqrt(x.astype(np.float64)[None, :] ** 2 + z.astype(np.float64)[:, None] ** 2)
    alpha = special.jn_zeros(0, len(coeffs))
    m = np.ones_like(r)
    for c, a in zip(coeffs, alpha):
        m += float(c) * special.j0(a * r / case["jet_radius"])
    return m


def test_profile_multipliers_match_scipy():
    case = get_case("jet_32x48x32")
    with Solver(case) as S:
        np.testing.assert_array_equal(S.inlet_profile(), 1.0)
        S.set_inlet_bessel(COEFFS)
        np.testing.assert_allclose(S.inlet_profile(), expected_profile(case, COEFFS), rtol=1e-6, atol=1e-7)
        S.set_inlet_bessel([])
        np.testing.assert_array_equal(S.inlet_profile(), 1.0)


def test_zero_series_is_the_top_hat():
    case = get_case("jet_24x40x24", NSTATS_START_STEP=0)
    out = []
    for coeffs in (None, np.zeros(8, np.float32)):
        with Solver(case) as S:
            if coeffs is not None:
                S.set_inlet_bessel(coeffs)
            S.init_jet()
            S.step(30)
            out.append(S.get_populations())
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("precision", [32, 64])
def test_jet_with_profile_matches_oracle(precision):
    case = get_case("jet_32x48x32", NSTATS_START_STEP=20)
    fr, fb, fields = initial_state(case)
    with Solver(case) as S:
        S.set_inlet_bessel(COEFFS)
        prof = S.inlet_profile()
        S.set_fields(**fields)
        S.set_populations(fr, fb)
        O = Oracle(case, precision)
        O.set_inlet_profile(prof)
        O.set_fields(**fields)
        O.set_populations(fr, fb)
        S.step(60)
        O.step(60)
        F, OF = S.get_fields(), O.get_fields()
        m = interior(case)
        e = {k: maxabs(F[k][m], OF[k][m]) for k in ("rhor", "rhob", "ux", "uy", "uz")}
        print(f"fp{precision}: {e}")
        for k, v in e.items():
            assert v <= 2e-5, (k, v)
        # the profile changes the flow: the inlet plane's uy follows m(r)
        NX, NY, NZ = case["NX"], case["NY"], case["NZ"]
        uy1 = F["uy"].reshape(NZ, NY, NX)[:, 1, :]
        top = Solver(case)
        top.set_fields(**fields)
        top.set_populations(fr, fb)
        top.step(60)
        uy1_top = top.get_fields()["uy"].reshape(NZ, NY, NX)[:, 1, :]
        top.close()
        assert np.max(np.abs(uy1 - uy1_top)) > 1e-4
