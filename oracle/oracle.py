"""ctypes wrapper of the CPU oracle (oracle/mcg_oracle.cpp) - TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as
the checker; the solver never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmcg_oracle.so")

_lib = None


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", HERE, "libmcg_oracle.so"], check=True, capture_output=True)
    lib = C.CDLL(LIB)
    P, D = C.c_void_p, C.POINTER(C.c_double)
    sig = {
        "orc_create": ([C.c_void_p, C.c_int], P),
        "orc_destroy": ([P], None),
        "orc_num_threads": ([], C.c_int),
        "orc_set_num_threads": ([C.c_int], None),
        "orc_init_jet": ([P], None),
        "orc_init_bubble": ([P], None),
        "orc_set_pops": ([P, D, D], None),
        "orc_get_pops": ([P, D, D], None),
        "orc_set_fields": ([P, D, D, D, D, D], None),
        "orc_get_fields": ([P, D, D, D, D, D], None),
        "orc_set_inlet_profile": ([P, D], None),
        "orc_adjoint_periodic": ([P, D, C.c_int, D, D], C.c_int),
        "orc_get_stress": ([P, D], None),
        "orc_macros": ([P], None),
        "orc_collistream": ([P], None),
        "orc_inlet": ([P], None),
        "orc_neumann": ([P], None),
        "orc_accumulate_radial": ([P], None),
        "orc_set_stats_mode": ([P, C.c_int], None),
        "orc_step": ([P, C.c_int], None),
        "orc_get_step": ([P], C.c_longlong),
        "orc_get_radial": ([P, D, C.POINTER(C.c_uint64)], None),
        "orc_get_radial_state": ([P, C.POINTER(C.c_int), C.POINTER(C.c_uint), C.POINTER(C.c_uint)], None),
        "orc_total_tke": ([P], C.c_double),
        "orc_update_uy_average": ([P], None),
        "orc_get_uy_average": ([P, D], None),
        "orc_conservation_sums": ([P, D], None),
        "orc_hash_uniform": ([C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64], C.c_float),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def num_threads() -> int:
    return int(_load().orc_num_threads())


def set_num_threads(n: int) -> None:
    _load().orc_set_num_threads(int(n))


def hash_uniform(seed: int, a: int, b: int, c: int) -> float:
    return float(_load().orc_hash_uniform(seed, a, b, c))


class Oracle:
    """The reference step on the CPU, in float32 (precision=32) or float64 (64)."""

    def __init__(self, case: dict, precision: int = 64):
        from multicomponent_color_gradient_b200.solver import params_struct  # plain struct, no compute

        self.lib = _load()
        self.params = params_struct(case)
        self.NX, self.NY, self.NZ = int(self.params.NX), int(self.params.NY), int(self.params.NZ)
        self.N = self.NX * self.NY * self.NZ
        self.NR_BINS = self.NX // 2
        self._h = self.lib.orc_create(C.byref(self.params), int(precision))
        if not self._h:
            raise ValueError("oracle rejected the parameters")

    def __del__(self):
        if getattr(self, "_h", None):
            self.lib.orc_destroy(self._h)
            self._h = None

    def init_jet(self):
        self.lib.orc_init_jet(self._h)

    def init_bubble(self):
        self.lib.orc_init_bubble(self._h)

    def set_populations(self, fr, fb):
        fr = np.ascontiguousarray(fr, np.float64).reshape(-1)
        fb = np.ascontiguousarray(fb, np.float64).reshape(-1)
        self.lib.orc_set_pops(self._h, _dp(fr), _dp(fb))

    def get_populations(self):
        fr = np.empty(27 * self.N)
        fb = np.empty(27 * self.N)
        self.lib.orc_get_pops(self._h, _dp(fr), _dp(fb))
        return fr, fb

    def set_fields(self, rhor, rhob, ux, uy, uz):
        arrs = [np.ascontiguousarray(a, np.float64).reshape(-1) for a in (rhor, rhob, ux, uy, uz)]
        self.lib.orc_set_fields(self._h, *[_dp(a) for a in arrs])

    def adjoint_periodic(self, target, nsteps: int):
        """Discrete adjoint of the periodic box from the current state: J =
        sum (psi_T - target)^2 and dJ/dsigma, dJ/dtau, dJ/du0 ((3, Ncells))."""
        tgt = np.ascontiguousarray(target, np.float64).reshape(-1)
        out = np.zeros(3)
        du0 = np.zeros(3 * self.N)
        rc = self.lib.orc_adjoint_periodic(self._h, _dp(tgt), int(nsteps), _dp(out), _dp(du0))
        if rc != 0:
            raise ValueError("the oracle's adjoint covers the periodic box")
        return {"J": out[0], "dJ_dsigma": out[1], "dJ_dtau": out[2], "dJ_du0": du0.reshape(3, self.N)}

    def set_inlet_profile(self, prof):
        """Per-column inlet velocity multipliers ((NZ, NX) or NX*NZ); None restores the top-hat."""
        if prof is None:
            self.lib.orc_set_inlet_profile(self._h, None)
            return
        a = np.ascontiguousarray(prof, np.float64).reshape(-1)
        assert a.size == self.NX * self.NZ
        self.lib.orc_set_inlet_profile(self._h, _dp(a))

    def get_fields(self):
        out = {k: np.empty(self.N) for k in ("rhor", "rhob", "ux", "uy", "uz")}
        self.lib.orc_get_fields(self._h, *[_dp(out[k]) for k in ("rhor", "rhob", "ux", "uy", "uz")])
        return out

    def get_stress(self):
        pi = np.empty(6 * self.N)
        self.lib.orc_get_stress(self._h, _dp(pi))
        return pi

    def macros(self):
        self.lib.orc_macros(self._h)

    def collistream(self):
        self.lib.orc_collistream(self._h)

    def inlet(self):
        self.lib.orc_inlet(self._h)

    def neumann(self):
        self.lib.orc_neumann(self._h)

    def accumulate_radial(self):
        self.lib.orc_accumulate_radial(self._h)

    def set_stats_mode(self, mode: int):
        self.lib.orc_set_stats_mode(self._h, int(mode))

    def step(self, n: int = 1):
        self.lib.orc_step(self._h, int(n))

    @property
    def current_step(self) -> int:
        return int(self.lib.orc_get_step(self._h))

    def get_radial(self):
        M = self.NY * self.NR_BINS
        sums = np.empty(5 * M)
        count = np.empty(M, np.uint64)
        self.lib.orc_get_radial(self._h, _dp(sums), count.ctypes.data_as(C.POINTER(C.c_uint64)))
        keys = ("sum_uy", "sum_uy2", "sum_ur", "sum_ur2", "sum_uruy")
        out = {k: sums[i * M:(i + 1) * M].copy() for i, k in enumerate(keys)}
        out["count"] = count
        return out

    def radial_state(self):
        st, s0, n = C.c_int(), C.c_uint(), C.c_uint()
        self.lib.orc_get_radial_state(self._h, C.byref(st), C.byref(s0), C.byref(n))
        return bool(st.value), int(s0.value), int(n.value)

    def total_tke(self) -> float:
        return float(self.lib.orc_total_tke(self._h))

    def update_uy_average(self):
        self.lib.orc_update_uy_average(self._h)

    def get_uy_average(self):
        a = np.empty(self.N)
        self.lib.orc_get_uy_average(self._h, _dp(a))
        return a

    def conservation_sums(self):
        out = np.zeros(5)
        self.lib.orc_conservation_sums(self._h, _dp(out))
        return out


def interior_mask(NX: int, NY: int, NZ: int) -> np.ndarray:
    """Boolean mask over id = x + NX*(y + NY*z) of interior nodes."""
    m = np.zeros((NZ, NY, NX), bool)
    m[1:-1, 1:-1, 1:-1] = True
    return m.reshape(-1)
