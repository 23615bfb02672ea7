"""The float64 CPU adjoint of the oracle (the reference step in its own push
form, periodic box) against central finite differences of the same oracle:
16^3 bubble (R=4) relaxed 15 steps, u0 from 26 Fourier modes, T = 12."""
import numpy as np
import pytest

from helpers import feq64, interior
from multicomponent_color_gradient_b200 import derive
from multicomponent_color_gradient_b200.adjoint import FourierModes
from oracle.oracle import Oracle

CASE = derive(dict(NX=16, NY=16, NZ=16, bubble_radius=4.0, tau=0.7, sigma=0.01, beta_recolor=0.7,
                   boundary="periodic", bubble_red_inside=1, NSTATS_START_STEP=10 ** 9, NSTEP=100, NOUTPUT=100,
                   Re=1.0, We=1.0))
T = 12
N = 16 ** 3


def mirror(a):
    v = a.reshape(16, 16, 16)
    v[:, :, 0], v[:, :, -1] = v[:, :, -2], v[:, :, 1]
    v[:, 0, :], v[:, -1, :] = v[:, -2, :], v[:, 1, :]
    v[0], v[-1] = v[-2].copy(), v[1].copy()


@pytest.fixture(scope="module")
def setup():
    O = Oracle(CASE, 64)
    O.init_bubble()
    O.step(15)
    fr, fb = O.get_populations()
    rr, rb = fr.reshape(27, N).sum(0), fb.reshape(27, N).sum(0)
    mirror(rr)
    mirror(rb)
    M = FourierModes(CASE, 1, 3)
    a0 = np.random.default_rng(1).normal(scale=4e-3, size=M.count)
    return rr, rb, (rr - rb) / (rr + rb), M, a0


def state(setup, sigma, tau, a):
    rr, rb, _, M, _ = setup
    O = Oracle(derive(dict(CASE, sigma=sigma, tau=tau)), 64)
    u = M.velocity(a)
    O.set_fields(rr, rb, u[0], u[1], u[2])
    O.set_populations(feq64(rr, *u).reshape(-1), feq64(rb, *u).reshape(-1))
    return O


def J(setup, sigma, tau, a):
    target = setup[2]
    O = state(setup, sigma, tau, a)
    O.step(T)
    fr, fb = O.get_populations()
    r, b = fr.reshape(27, N).sum(0), fb.reshape(27, N).sum(0)
    m = interior(CASE)
    d = (r - b)[m] / (r + b)[m] - target[m]
    return float(np.sum(d * d))


def test_oracle_adjoint_matches_its_finite_differences(setup):
    _, _, target, M, a0 = setup
    s, t = CASE["sigma"], CASE["taub"]
    res = state(setup, s, t, a0).adjoint_periodic(target, T)
    assert abs(res["J"] - J(setup, s, t, a0)) <= 1e-12 * res["J"]
    f32 = np.float32
    sp, sm = float(f32(1.01 * s)), float(f32(0.99 * s))
    tp, tm = float(f32(t + 0.002)), float(f32(t - 0.002))
    fd_s = (J(setup, sp, t, a0) - J(setup, sm, t, a0)) / (sp - sm)
    fd_t = (J(setup, s, tp, a0) - J(setup, s, tm, a0)) / (tp - tm)
    assert abs(res["dJ_dsigma"] - fd_s) <= 1e-5 * abs(fd_s), (res["dJ_dsigma"], fd_s)
    assert abs(res["dJ_dtau"] - fd_t) <= 1e-4 * abs(fd_t), (res["dJ_dtau"], fd_t)
    g = M.project(res["dJ_du0"])
    for k in np.argsort(-np.abs(g))[:3]:
        h = 1e-4
        ap, am = a0.copy(), a0.copy()
        ap[k] += h
        am[k] -= h
        fd = (J(setup, s, t, ap) - J(setup, s, t, am)) / (2 * h)
        assert abs(g[k] - fd) <= 1e-6 * abs(fd), (k, g[k], fd)
