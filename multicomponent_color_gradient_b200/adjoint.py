"""Gradients of a bubble-shape objective through the time loop.

The periodic-box step (the reference's lbm.cuh:82-293 collision and
forces.cuh colour gradient, with the x/z wrap of bounds.cuh applied in y as
well) is differentiated as a discrete adjoint on the GPU
(``Solver.adjoint_run``, C entry point ``mcg_adjoint_run``): one reverse sweep
gives J = sum (psi_T - psi*)^2 and its derivatives with respect to the surface
tension sigma, the relaxation time tau and the initial velocity field u0.

Here u0 is a sum of Fourier modes of the periodic interior,

    u0(x) = sum_m a_m e_m cos(k_m . (x - 1) + phi_m),   k_m = 2 pi n_m / L,

n_m the integer wave vectors with max |n_i| <= max_mode (one of each +-n
pair), e_m two unit polarisations perpendicular to k_m (divergence-free
modes), phi_m seeded phases; dJ/da_m is the projection of dJ/du0 on mode m.
``BubbleObjective`` wraps the sweep as a ``torch.autograd.Function``.
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

from .cases import derive, get_case
from .solver import Solver


class FourierModes:
    """Divergence-free cosine modes of the periodic interior (ghost nodes 0)."""

    def __init__(self, case: Dict, max_mode: int = 1, seed: int = 0):
        c = derive(case)
        self.NX, self.NY, self.NZ = int(c["NX"]), int(c["NY"]), int(c["NZ"])
        self.N = self.NX * self.NY * self.NZ
        L = np.array([self.NX - 2, self.NY - 2, self.NZ - 2], np.float64)
        if not 2 * max_mode < L.min():
            raise ValueError("max_mode must be below half the interior extent")
        waves = []
        rng = range(-max_mode, max_mode + 1)
        for nz in rng:
            for ny in rng:
                for nx in rng:
                    n = (nx, ny, nz)
                    if n == (0, 0, 0):
                        continue
                    # one of each +-n pair: first non-zero component positive
                    first = next(v for v in n if v != 0)
                    if first > 0:
                        waves.append(n)
        gen = np.random.default_rng(seed)
        ks, pols, phases = [], [], []
        for n in waves:
            k = 2.0 * np.pi * np.asarray(n, np.float64) / L
            helper = np.array([1.0, 0.0, 0.0]) if abs(k[0]) < 0.9 * np.linalg.norm(k) else np.array([0.0, 1.0, 0.0])
            e1 = np.cross(k, helper)
            e1 /= np.linalg.norm(e1)
            e2 = np.cross(k, e1)
            e2 /= np.linalg.norm(e2)
            for e in (e1, e2):
                ks.append(k)
                pols.append(e)
                phases.append(gen.uniform(0.0, 2.0 * np.pi))
        self.k = np.array(ks)          # (M, 3)
        self.e = np.array(pols)        # (M, 3)
        self.phase = np.array(phases)  # (M,)
        self.count = len(phases)
        self.n = np.array([w for w in waves for _ in (0, 1)], np.int64)  # (M, 3) integer wave vectors
        self.L = L.astype(np.int64)

    # Synthesis and projection run through FFTs of the interior: mode m puts
    # a_m e_m exp(i phi_m) at wave vector n_m of the spectrum A, and
    # u = Re sum_n A_n exp(i k_n . xi) is L^3 times the real part of the
    # inverse FFT.  The projection is the transpose: Re(exp(i phi_m) e_m .
    # conj(V(n_m))) with V the forward FFT of the field.

    def _spectral_index(self):
        Lx, Ly, Lz = self.L
        return self.n[:, 2] % Lz, self.n[:, 1] % Ly, self.n[:, 0] % Lx

    def velocity(self, a: np.ndarray) -> np.ndarray:
        """u0 as (3, Ncells) float64 from amplitudes a (M,); ghost nodes 0."""
        a = np.asarray(a, np.float64).reshape(self.count)
        Lx, Ly, Lz = self.L
        iz, iy, ix = self._spectral_index()
        coef = a * np.exp(1j * self.phase)
        u = np.zeros((3, self.NZ, self.NY, self.NX))
        for c in range(3):
            A = np.zeros((Lz, Ly, Lx), np.complex128)
            np.add.at(A, (iz, iy, ix), coef * self.e[:, c])
            u[c, 1:-1, 1:-1, 1:-1] = np.fft.ifftn(A).real * (Lx * Ly * Lz)
        return u.reshape(3, self.N)

    def project(self, v: np.ndarray) -> np.ndarray:
        """The transpose of ``velocity``: sum_x v(x) . e_m cos(k_m.x + phi_m)."""
        v = np.asarray(v, np.float64).reshape(3, self.NZ, self.NY, self.NX)[:, 1:-1, 1:-1, 1:-1]
        iz, iy, ix = self._spectral_index()
        out = np.zeros(self.count)
        for c in range(3):
            V = np.fft.fftn(v[c])
            out += self.e[:, c] * np.real(np.exp(1j * self.phase) * np.conj(V[iz, iy, ix]))
        return out


class BubbleProblem:
    """J(a, sigma, tau) = sum over interior nodes of (psi_T - psi*)^2 for the
    periodic bubble started from feq(rho_c, u0(a)) and run `nsteps` steps.

    rho_c are the densities of the bubble after `relax_steps` steps from the
    reference's bubble initial state (bubble/bubbleIn.cuh) at u = 0, so the
    interface starts resolved; psi* defaults to their colour field."""

    def __init__(self, case="adjoint_bubble_96", nsteps: int = 100, snapshots: Optional[int] = None,
                 max_mode: int = 1, seed: int = 0, relax_steps: int = 50, target: Optional[np.ndarray] = None,
                 **overrides):
        self.case = get_case(case, **overrides) if isinstance(case, str) else derive(dict(case, **overrides))
        if self.case["boundary"] != "periodic":
            raise ValueError("the adjoint covers the periodic box")
        self.nsteps = int(nsteps)
        self.snapshots = int(snapshots) if snapshots else self.nsteps + 1
        self.tape = None  # records of the taped innermost segments (None: the handle's default)
        self.modes = FourierModes(self.case, max_mode, seed)
        with Solver(self.case) as S:
            S.init_bubble()
            if relax_steps:
                S.step(relax_steps)
                fr, fb = S.get_populations()
                Q = fr.size // S.N
                self.rhor = fr.reshape(Q, S.N).sum(0, dtype=np.float64).astype(np.float32)
                self.rhob = fb.reshape(Q, S.N).sum(0, dtype=np.float64).astype(np.float32)
                self._fill_ghosts(self.rhor)
                self._fill_ghosts(self.rhob)
            else:
                F = S.get_fields()
                self.rhor, self.rhob = F["rhor"], F["rhob"]
        if target is None:
            target = (self.rhor - self.rhob) / (self.rhor + self.rhob)
        self.target = np.ascontiguousarray(target, np.float32).reshape(-1)
        self._solver = None
        self._solver_key = None

    def _fill_ghosts(self, a: np.ndarray) -> None:
        """Ghost nodes mirror the opposite interior node (periodic box)."""
        NX, NY, NZ = self.modes.NX, self.modes.NY, self.modes.NZ
        v = a.reshape(NZ, NY, NX)
        v[:, :, 0], v[:, :, -1] = v[:, :, -2], v[:, :, 1]
        v[:, 0, :], v[:, -1, :] = v[:, -2, :], v[:, 1, :]
        v[0, :, :], v[-1, :, :] = v[-2, :, :], v[1, :, :]

    def solver(self, sigma: float, tau: float) -> Solver:
        key = (float(np.float32(sigma)), float(np.float32(tau)))
        if self._solver_key != key:
            if self._solver is not None:
                self._solver.close()
            self._solver = Solver(dict(self.case, sigma=key[0], tau=key[1]))
            self._solver_key = key
        return self._solver

    def initial_velocity(self, a) -> np.ndarray:
        return self.modes.velocity(a).astype(np.float32)

    def evaluate(self, a, sigma: Optional[float] = None, tau: Optional[float] = None) -> Dict:
        """J and dJ/da, dJ/dsigma, dJ/dtau from one forward + reverse sweep."""
        sigma = self.case["sigma"] if sigma is None else sigma
        tau = self.case["taub"] if tau is None else tau
        S = self.solver(sigma, tau)
        u = self.initial_velocity(a)
        S.init_equilibrium(self.rhor, self.rhob, u[0], u[1], u[2])
        r = S.adjoint_run(self.target, self.nsteps, self.snapshots, self.tape)
        r["dJ_da"] = self.modes.project(r["dJ_du0"])
        return r

    def close(self) -> None:
        if self._solver is not None:
            self._solver.close()
            self._solver = None


try:
    import torch

    class BubbleObjective(torch.autograd.Function):
        """J(a, sigma, tau) of a ``BubbleProblem`` as an autograd node: the
        forward pass runs the forward and the reverse sweep together (the
        reverse sweep needs the forward states anyway) and keeps the
        gradients for backward."""

        @staticmethod
        def forward(ctx, a, sigma, tau, problem: BubbleProblem):
            r = problem.evaluate(a.detach().cpu().double().numpy(), float(sigma), float(tau))
            ctx.grads = (torch.as_tensor(r["dJ_da"], dtype=a.dtype, device=a.device),
                         torch.as_tensor(r["dJ_dsigma"], dtype=sigma.dtype, device=sigma.device),
                         torch.as_tensor(r["dJ_dtau"], dtype=tau.dtype, device=tau.device))
            return torch.as_tensor(r["J"], dtype=torch.float64, device=a.device)

        @staticmethod
        def backward(ctx, gJ):
            da, ds, dt = ctx.grads
            return gJ.to(da.dtype) * da, gJ.to(ds.dtype) * ds, gJ.to(dt.dtype) * dt, None

except ImportError:  # pragma: no cover - torch is an optional dependency of this module
    BubbleObjective = None
