"""Discrete adjoint on the GPU against central finite differences of the
float64 CPU oracle, for the periodic bubble (22^3 interior, R = 6, tau 0.7,
sigma 0.01, beta 0.7) started from feq(rho_c, u0) with u0 a sum of 26
divergence-free Fourier modes, J = sum (psi_T - psi*)^2 after T = 24 steps.

Tolerances: the adjoint runs in float32; the finite differences are float64
central differences with steps h and h/2 (1 % and 0.5 % of sigma, 0.002 and
0.001 of tau, 1 % and 0.5 % of the largest amplitude) combined by Richardson
extrapolation, (4 D(h/2) - D(h))/3, which removes the O(h^2) truncation
error.  Gradients agree within 1e-4 relative; J within 1e-4 relative."""
import numpy as np
import pytest

from helpers import feq64, interior
from multicomponent_color_gradient_b200 import Solver, derive
from multicomponent_color_gradient_b200.adjoint import BubbleObjective, BubbleProblem
from multicomponent_color_gradient_b200.solver import adjoint_plan
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

CASE = dict(NX=24, NY=24, NZ=24, bubble_radius=6.0, tau=0.7, sigma=0.01, beta_recolor=0.7, boundary="periodic",
            bubble_red_inside=1, NSTATS_START_STEP=10 ** 9, NSTEP=100, NOUTPUT=100, Re=1.0, We=1.0)
T = 24


@pytest.fixture(scope="module")
def problem():
    P = BubbleProblem(CASE, nsteps=T, max_mode=1, seed=3, relax_steps=40)
    a0 = np.random.default_rng(11).normal(scale=4e-3, size=P.modes.count)
    yield P, a0
    P.close()


def oracle_J(P, a, sigma, tau):
    case = derive(dict(P.case, sigma=sigma, tau=tau))
    O = Oracle(case, 64)
    u = P.modes.velocity(a)
    rr, rb = P.rhor.astype(np.float64), P.rhob.astype(np.float64)
    O.set_fields(rr, rb, u[0], u[1], u[2])
    O.set_populations(feq64(rr, u[0], u[1], u[2]).reshape(-1), feq64(rb, u[0], u[1], u[2]).reshape(-1))
    O.step(T)
    fr, fb = O.get_populations()
    N = P.modes.N
    r, b = fr.reshape(27, N).sum(0), fb.reshape(27, N).sum(0)
    m = interior(case)
    d = (r - b)[m] / (r + b)[m] - P.target[m].astype(np.float64)
    return float(np.sum(d * d))


def test_J_matches_the_forward_run(problem):
    P, a0 = problem
    r = P.evaluate(a0)
    S = P.solver(P.case["sigma"], P.case["taub"])
    u = P.initial_velocity(a0)
    S.init_equilibrium(P.rhor, P.rhob, u[0], u[1], u[2])
    S.step(T)
    fr, fb = S.get_populations()
    rr, rb = fr.reshape(27, S.N).sum(0, dtype=np.float64), fb.reshape(27, S.N).sum(0, dtype=np.float64)
    m = interior(P.case)
    J = float(np.sum(((rr - rb)[m] / (rr + rb)[m] - P.target[m]) ** 2))
    assert abs(r["J"] - J) <= 1e-5 * J, (r["J"], J)
    Jo = oracle_J(P, a0, P.case["sigma"], P.case["taub"])
    print(f"J gpu={r['J']:.8e} forward={J:.8e} fp64 oracle={Jo:.8e}")
    assert abs(r["J"] - Jo) <= 1e-4 * Jo


def _richardson(d_h, d_h2):
    """(4 D(h/2) - D(h)) / 3: central differences with the O(h^2) term removed."""
    return (4.0 * d_h2 - d_h) / 3.0


def test_gradients_match_fp64_central_differences(problem):
    P, a0 = problem
    r = P.evaluate(a0)
    sigma, tau = P.case["sigma"], P.case["taub"]
    f32 = np.float32

    def d_sigma(frac):
        # the parameters reach both solvers as float32: difference the rounded values
        sp, sm = float(f32((1 + frac) * sigma)), float(f32((1 - frac) * sigma))
        return (oracle_J(P, a0, sp, tau) - oracle_J(P, a0, sm, tau)) / (sp - sm)

    def d_tau(step):
        tp, tm = float(f32(tau + step)), float(f32(tau - step))
        return (oracle_J(P, a0, sigma, tp) - oracle_J(P, a0, sigma, tm)) / (tp - tm)

    fd_s = _richardson(d_sigma(0.01), d_sigma(0.005))
    fd_t = _richardson(d_tau(0.002), d_tau(0.001))
    print(f"dJ/dsigma adjoint={r['dJ_dsigma']:.7e} fd={fd_s:.7e}; dJ/dtau adjoint={r['dJ_dtau']:.7e} fd={fd_t:.7e}")
    assert abs(r["dJ_dsigma"] - fd_s) <= 1e-4 * abs(fd_s)
    assert abs(r["dJ_dtau"] - fd_t) <= 1e-4 * abs(fd_t)
    g = r["dJ_da"]
    for k in np.argsort(-np.abs(g))[:3]:

        def d_a(h):
            ap, am = a0.copy(), a0.copy()
            ap[k] += h
            am[k] -= h
            return (oracle_J(P, ap, sigma, tau) - oracle_J(P, am, sigma, tau)) / (2 * h)

        h = 0.01 * np.abs(a0).max()
        fd = _richardson(d_a(h), d_a(h / 2))
        print(f"dJ/da[{k}] adjoint={g[k]:.7e} fd={fd:.7e}")
        assert abs(g[k] - fd) <= 1e-4 * abs(fd), (k, g[k], fd)


def test_matches_fp64_cpu_adjoint(problem):
    """The float32 GPU adjoint against the oracle's float64 adjoint (the
    reference step's push form, direction by direction): the whole dJ/du0
    field within 1e-4 of its largest value (measured 1.1e-6), J and the
    parameter gradients within 1e-4 relative (measured 8e-7, 5e-6, 2e-7)."""
    P, a0 = problem
    r = P.evaluate(a0)
    O = Oracle(P.case, 64)
    u = P.modes.velocity(a0)
    rr, rb = P.rhor.astype(np.float64), P.rhob.astype(np.float64)
    O.set_fields(rr, rb, u[0], u[1], u[2])
    O.set_populations(feq64(rr, u[0], u[1], u[2]).reshape(-1), feq64(rb, u[0], u[1], u[2]).reshape(-1))
    o = O.adjoint_periodic(P.target, T)
    scale = np.abs(o["dJ_du0"]).max()
    err = np.abs(r["dJ_du0"] - o["dJ_du0"]).max() / scale
    print(f"J {r['J']:.8e} vs {o['J']:.8e}; dJ/dsigma {r['dJ_dsigma']:.6e} vs {o['dJ_dsigma']:.6e}; "
          f"dJ/dtau {r['dJ_dtau']:.6e} vs {o['dJ_dtau']:.6e}; dJ/du0 max rel err {err:.2e}")
    assert abs(r["J"] - o["J"]) <= 1e-4 * o["J"]
    assert abs(r["dJ_dsigma"] - o["dJ_dsigma"]) <= 1e-4 * abs(o["dJ_dsigma"])
    assert abs(r["dJ_dtau"] - o["dJ_dtau"]) <= 1e-4 * abs(o["dJ_dtau"])
    assert err <= 1e-4


@pytest.mark.parametrize("snapshots", [2, 5])
@pytest.mark.parametrize("tape", [0, 4])
def test_fewer_snapshots_same_gradients(problem, snapshots, tape):
    """Binomial checkpointing with 2 or 5 held states, the innermost segments
    reversed by re-advancing before every op (tape 0) or from a tape of 4
    moment records: the gradients of the all-states tape, bit for bit for
    dJ/du0 (the fused step's records equal the moments kernel's)."""
    P, a0 = problem
    full = P.evaluate(a0)
    P.snapshots, P.tape = snapshots, tape
    try:
        r = P.evaluate(a0)
    finally:
        P.snapshots, P.tape = T + 1, None
    assert r["forward_steps"] == adjoint_plan(T, snapshots, tape)[0] > T
    assert abs(r["J"] - full["J"]) <= 1e-12 * full["J"]
    for k in ("dJ_dsigma", "dJ_dtau"):
        assert abs(r[k] - full[k]) <= 1e-9 * abs(full[k])
    np.testing.assert_array_equal(r["dJ_du0"], full["dJ_du0"])


def test_torch_autograd_function(problem):
    import torch

    P, a0 = problem
    a = torch.tensor(a0, dtype=torch.float64, requires_grad=True)
    sigma = torch.tensor(P.case["sigma"], dtype=torch.float64, requires_grad=True)
    tau = torch.tensor(P.case["taub"], dtype=torch.float64, requires_grad=True)
    J = BubbleObjective.apply(a, sigma, tau, P)
    (3.0 * J).backward()
    r = P.evaluate(a0)
    assert abs(float(J) - r["J"]) <= 1e-12 * r["J"]
    np.testing.assert_allclose(a.grad.numpy(), 3.0 * r["dJ_da"], rtol=1e-12)
    assert abs(float(sigma.grad) - 3.0 * r["dJ_dsigma"]) <= 1e-9 * abs(r["dJ_dsigma"])
    assert abs(float(tau.grad) - 3.0 * r["dJ_dtau"]) <= 1e-9 * abs(r["dJ_dtau"])


def test_state_is_left_unchanged(problem):
    P, a0 = problem
    S = P.solver(P.case["sigma"], P.case["taub"])
    u = P.initial_velocity(a0)
    S.init_equilibrium(P.rhor, P.rhob, u[0], u[1], u[2])
    S.step(3)
    before = S.get_populations(), S.get_fields(), S.current_step
    S.adjoint_run(P.target, 5, 6)
    after = S.get_populations(), S.get_fields(), S.current_step
    np.testing.assert_array_equal(before[0][0], after[0][0])
    np.testing.assert_array_equal(before[0][1], after[0][1])
    for k in before[1]:
        np.testing.assert_array_equal(before[1][k], after[1][k])
    assert before[2] == after[2] == 3


def test_adjoint_cost_within_four_forward_runs():
    """96^3 periodic bubble, 100 steps, a snapshot per state: the whole
    forward + reverse sweep against 100 plain forward steps."""
    P = BubbleProblem("adjoint_bubble_96", nsteps=100, max_mode=1, seed=1, relax_steps=0)
    try:
        a = np.random.default_rng(2).normal(scale=2e-3, size=P.modes.count)
        P.evaluate(a)  # warm-up (allocations, first launches)
        r = P.evaluate(a)
        S = P.solver(P.case["sigma"], P.case["taub"])
        u = P.initial_velocity(a)
        S.init_equilibrium(P.rhor, P.rhob, u[0], u[1], u[2])
        S.step(5)
        fwd = S.step_timed(100)
        print(f"adjoint sweep {r['ms']:.2f} ms vs forward {fwd:.2f} ms: {r['ms'] / fwd:.2f}x")
        assert r["forward_steps"] == 100
        assert r["ms"] <= 4.0 * fwd
    finally:
        P.close()
