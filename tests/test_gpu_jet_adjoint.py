"""Discrete adjoint of the jet (inlet with its radial profile, convective outlet)
on the GPU against central finite differences of the float64 CPU oracle:
jet 24x40x24 (D=6, Re 45, We 3), profile coefficients c = (0.1, -0.05, 0.02,
0, ...), T = 40 steps, J = sum over steps 20..39 of (1/2) sum of uy^2 over
y >= 20.  dJ/dc_k within 1e-4 relative of float64 central differences
(steps 0.02 and 0.01 combined by Richardson extrapolation, which removes the
O(h^2) truncation error); J within 1e-5 of the GPU's own forward run and
1e-4 of the float64 oracle."""
import numpy as np
import pytest
from scipy import special

from multicomponent_color_gradient_b200 import Solver, get_case
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

CASE = get_case("jet_24x40x24", NSTATS_START_STEP=10 ** 9)
C0 = np.array([0.1, -0.05, 0.02, 0, 0, 0, 0, 0], np.float64)
T, T0, T1, YOBS = 40, 20, 39, 20


def multipliers(c):
    NX, NZ = CASE["NX"], CASE["NZ"]
    x = np.arange(NX, dtype=np.float32) - np.float32(CASE["jet_x0"])
    z = np.arange(NZ, dtype=np.float32) - np.float32(CASE["jet_z0"])
    r = np.sqrt(x.astype(np.float64)[None, :] ** 2 + z.astype(np.float64)[:, None] ** 2)
    m = np.ones_like(r)
    for ck, a in zip(c, special.jn_zeros(0, len(c))):
        m += ck * special.j0(a * r / CASE["jet_radius"])
    return m


def objective(F):
    NX, NY, NZ = CASE["NX"], CASE["NY"], CASE["NZ"]
    uy = np.asarray(F["uy"], np.float64).reshape(NZ, NY, NX)[1:-1, YOBS:-1, 1:-1]
    return 0.5 * float(np.sum(uy * uy))


def oracle_J(c):
    O = Oracle(CASE, 64)
    O.set_inlet_profile(multipliers(c))
    O.init_jet()
    J = 0.0
    for t in range(T):
        O.step(1)
        if T0 <= t <= T1:
            J += objective(O.get_fields())
    return J


@pytest.fixture(scope="module")
def adjoint():
    with Solver(CASE) as S:
        S.set_inlet_bessel(C0.astype(np.float32))
        S.init_jet()
        return S.adjoint_jet_run(T, T0, T1, YOBS)


def test_J_matches_forward_runs(adjoint):
    with Solver(CASE) as S:
        S.set_inlet_bessel(C0.astype(np.float32))
        S.init_jet()
        J = 0.0
        for t in range(T):
            S.step(1)
            if T0 <= t <= T1:
                J += objective(S.get_fields())
    Jo = oracle_J(C0)
    print(f"J adjoint={adjoint['J']:.8e} forward={J:.8e} fp64 oracle={Jo:.8e}")
    assert abs(adjoint["J"] - J) <= 1e-5 * J
    assert abs(adjoint["J"] - Jo) <= 1e-4 * Jo


def central_difference(J_of, c0, k, h):
    cp, cm = c0.copy(), c0.copy()
    cp[k] += h
    cm[k] -= h
    return (J_of(cp) - J_of(cm)) / (2 * h)


@pytest.mark.parametrize("k", [0, 1, 2, 5])
def test_dJ_dc_matches_fp64_central_differences(adjoint, k):
    d1 = central_difference(oracle_J, C0, k, 0.02)
    d2 = central_difference(oracle_J, C0, k, 0.01)
    fd = (4.0 * d2 - d1) / 3.0
    g = adjoint["dJ_dc"][k]
    print(f"dJ/dc[{k}] adjoint={g:.7e} fd={fd:.7e} (h=0.02: {d1:.7e}, h=0.01: {d2:.7e})")
    assert abs(g - fd) <= 1e-4 * abs(fd), (k, g, fd)


@pytest.mark.parametrize("segment", [7, 16])
@pytest.mark.parametrize("tapes", [1, 3])
def test_segments_give_the_same_gradients(adjoint, segment, tapes):
    """Snapshots every `segment` steps, one segment tape (every segment re-run
    once from its snapshot) or three (the two last segments of the first pass,
    which stops before the last one, reversed from their pass-1 tapes): the
    gradients of the all-steps tape."""
    with Solver(CASE) as S:
        S.set_inlet_bessel(C0.astype(np.float32))
        S.init_jet()
        S.set_jet_adjoint_tapes(tapes)
        r = S.adjoint_jet_run(T, T0, T1, YOBS, segment=segment)
    nseg = -(-T // segment)
    rerun = T - (min(tapes, nseg) - 1) * segment  # segments nseg-2 .. nseg-tapes come from pass 1
    assert r["forward_steps"] == (nseg - 1) * segment + rerun
    assert abs(r["J"] - adjoint["J"]) <= 1e-12 * adjoint["J"]
    np.testing.assert_allclose(r["dJ_dc"], adjoint["dJ_dc"], rtol=1e-9, atol=1e-15)


def test_state_is_left_unchanged():
    with Solver(CASE) as S:
        S.set_inlet_bessel(C0.astype(np.float32))
        S.init_jet()
        S.step(5)
        before = S.get_populations(), S.get_fields(), S.current_step
        S.adjoint_jet_run(10, 0, 9, YOBS)
        after = S.get_populations(), S.get_fields(), S.current_step
        np.testing.assert_array_equal(before[0][0], after[0][0])
        np.testing.assert_array_equal(before[0][1], after[0][1])
        for key in before[1]:
            np.testing.assert_array_equal(before[1][key], after[1][key])
        assert before[2] == after[2] == 5
