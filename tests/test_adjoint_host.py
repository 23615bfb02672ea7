"""Host-side pieces of the discrete adjoint (no GPU): the binomial
checkpointing schedule and the Fourier-mode parametrisation of u0."""
import functools

import numpy as np
import pytest

from multicomponent_color_gradient_b200 import get_case
from multicomponent_color_gradient_b200.adjoint import FourierModes
from multicomponent_color_gradient_b200.solver import adjoint_plan


@functools.lru_cache(maxsize=None)
def optimal_forward_steps(n, s):
    """Fewest forward steps that reverse n ops (op t needs state t) holding the
    first state plus s free slots: exhaustive over every split point."""
    if n == 1:
        return 0
    if s == 0:
        return n * (n - 1) // 2
    return min(m + optimal_forward_steps(n - m, s - 1) + optimal_forward_steps(m, s) for m in range(1, n))


@pytest.mark.parametrize("snapshots", [1, 2, 3, 4, 6])
def test_schedule_is_optimal(snapshots):
    for T in range(1, 41):
        fwd, r = adjoint_plan(T, snapshots)
        s = min(snapshots - 1, T)
        assert fwd == optimal_forward_steps(T + 1, s), (T, snapshots, fwd)


def test_schedule_with_a_slot_per_state_runs_each_step_once():
    for T in (1, 7, 100, 1000):
        assert adjoint_plan(T, T + 1) == (T, 1)
        assert adjoint_plan(T, T + 50) == (T, 1)
        assert adjoint_plan(T, 1) == (T * (T + 1) // 2, T)


def test_schedule_depth_is_binomial():
    # r least with C(s + r, s) >= T + 1 (s = snapshots - 1)
    from math import comb
    for T, snaps in ((1000, 4), (500, 10), (64, 2)):
        f, r = adjoint_plan(T, snaps)
        assert comb(snaps + r, snaps) >= T + 1 > comb(snaps + r - 1, snaps)
        # Griewank's minimum: r n - C(s + r, s + 1) forward steps for n = T + 1 ops
        assert f == r * (T + 1) - comb(snaps + r, snaps + 1)


def dense_velocity(M, a):
    """Direct sum of the modes at every interior node (small grids only)."""
    z, y, x = np.meshgrid(np.arange(M.NZ), np.arange(M.NY), np.arange(M.NX), indexing="ij")
    xi = np.stack([(x - 1).ravel(), (y - 1).ravel(), (z - 1).ravel()], 1).astype(np.float64)
    inside = ((x >= 1) & (x <= M.NX - 2) & (y >= 1) & (y <= M.NY - 2) & (z >= 1) & (z <= M.NZ - 2)).ravel()
    u = np.zeros((3, M.N))
    u[:, inside] = ((np.cos(xi[inside] @ M.k.T + M.phase[None, :]) * a[None, :]) @ M.e).T
    return u


def test_fourier_modes_are_divergence_free_and_project_is_the_transpose():
    case = get_case("adjoint_bubble_96", NX=14, NY=12, NZ=10)
    M = FourierModes(case, max_mode=1, seed=5)
    assert M.count == 26
    assert np.allclose(np.einsum("mc,mc->m", M.k, M.e), 0.0)
    rng = np.random.default_rng(0)
    a = rng.normal(size=M.count)
    # the FFT synthesis equals the direct sum of the modes
    np.testing.assert_allclose(M.velocity(a), dense_velocity(M, a), atol=1e-12)
    v = rng.normal(size=(3, M.N))
    lhs = float(np.sum(M.velocity(a) * v))
    rhs = float(a @ M.project(v))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
    u = M.velocity(a).reshape(3, 10, 12, 14)
    assert np.all(u[:, 0] == 0) and np.all(u[:, :, :, -1] == 0)


def test_fourier_modes_eight_per_axis():
    """8 modes per axis on a 22^3 interior: 2456 wave vectors, 4912 amplitudes;
    the spectral divergence k . e vanishes and synthesis/projection stay adjoint."""
    case = get_case("adjoint_bubble_96", NX=24, NY=24, NZ=24)
    M = FourierModes(case, max_mode=8, seed=2)
    assert M.count == 2 * (17 ** 3 - 1) // 2
    assert np.allclose(np.einsum("mc,mc->m", M.k, M.e), 0.0, atol=1e-12)
    rng = np.random.default_rng(3)
    a = rng.normal(size=M.count) * 1e-3
    v = rng.normal(size=(3, M.N))
    lhs = float(np.sum(M.velocity(a) * v))
    rhs = float(a @ M.project(v))
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs)
    with pytest.raises(ValueError):
        FourierModes(case, max_mode=11)


def taped_forward_steps(n, s, K):
    """Forward steps of the treeverse splits with every segment of at most
    K + 1 ops reversed by one taped advance (its length minus one steps)."""
    from math import comb

    def beta(h, r):
        return 0 if r < 0 else comb(h + r, h)

    if n <= 1:
        return 0
    if n <= K + 1:
        return n - 1
    if s == 0:
        return n * (n - 1) // 2
    held = s + 1
    r = 0
    while beta(held, r) < n:
        r += 1
    m = min(max(n - beta(held - 1, r), beta(held, r - 2), 1), n - 1)
    return m + taped_forward_steps(n - m, s - 1, K) + taped_forward_steps(m, s, K)


@pytest.mark.parametrize("tape", [1, 4, 20])
def test_taped_schedule(tape):
    """The schedule with taped innermost segments: the count the model above
    gives, never more than the plain treeverse, T steps once the tape covers
    the run, and 834 forward steps for the 96^3 bubble's 400 steps with 20
    held states and 20 records."""
    for T in list(range(1, 60)) + [100, 400]:
        for snaps in (1, 2, 3, 5, 20):
            fwd, _ = adjoint_plan(T, snaps, tape)
            if snaps > T:
                assert fwd == T
                continue
            assert fwd == taped_forward_steps(T + 1, min(snaps - 1, T), min(tape, T)), (T, snaps, tape)
            assert fwd <= adjoint_plan(T, snaps)[0]
            if tape >= T:
                assert fwd == T
    if tape == 20:
        assert adjoint_plan(400, 20, 20)[0] == 834
