"""Python mirror of the reference's launch interface over the C ABI.

The reference drives its step from main.cu through the launchers of
launch.cuh:13-118 (launch_jetDensity, launch_Injet, launch_bubble,
launch_Macros, launch_accumulate_radial_moments, launch_collistream,
launch_inlet_bc, launch_neumann_bc, launch_compute_total_tke,
launch_update_tke_average, launch_update_uy_average) on an LbmDevice
(memory.cuh:11-25).  ``Solver`` exposes the same names with the same meaning
on a device-resident state owned by libmcg.so; ``step(n)`` runs the fused B200
path for n steps of main.cu:52-82.  Errors raise ``McgError`` (the reference
calls exit(1), utilities/cudaUtilities.cuh:9-19).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np

from . import _lib
from .cases import BOUNDARY, STORAGE, derive

Q = 27
# Direction order of stencil_ct.cuh:9-16.
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1])

_PARAM_KEYS = ["NX", "NY", "NZ", "NSTEP", "NOUTPUT", "NSTATS_START_STEP", "write_vti_output", "sponge_cells",
               "jet_radius", "jet_x0", "jet_z0", "jet_velocity", "bubble_radius", "bubble_x0", "bubble_y0",
               "bubble_z0", "rhor0", "rhob0", "Re", "We", "nu", "taur", "taub", "sigma", "beta_recolor", "sponge_K",
               "seed", "init_noise", "inlet_noise", "bubble_red_inside"]


def params_struct(case: Dict) -> _lib.McgParams:
    """mcg_params from a case dict (see cases.py); derived values taken as given."""
    c = dict(case)
    if "nu" not in c:
        c = derive(c)
    p = _lib.McgParams()
    for k in _PARAM_KEYS:
        setattr(p, k, float(c[k]) if isinstance(getattr(p, k), float) else int(c[k]))
    p.boundary = BOUNDARY[c["boundary"]] if isinstance(c["boundary"], str) else int(c["boundary"])
    p.storage = STORAGE[c["storage"]] if isinstance(c["storage"], str) else int(c["storage"])
    return p


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Solver:
    """One device-resident lattice (the reference's LbmDevice + MeanFieldsDevice)."""

    def __init__(self, case: Dict):
        self.lib = _lib.load()
        self.case = dict(case) if "nu" in case else derive(case)
        self.params = params_struct(self.case)
        self.NX, self.NY, self.NZ = int(self.params.NX), int(self.params.NY), int(self.params.NZ)
        self.N = self.NX * self.NY * self.NZ
        self.NR_BINS = self.NX // 2
        h = C.c_void_p()
        _lib.check(self.lib.mcg_create(C.byref(self.params), C.byref(h)), "mcg_create")
        self._h = h

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.mcg_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, name: str, *args) -> None:
        _lib.check(getattr(self.lib, name)(self._h, *args), name)

    def set_stream(self, stream_ptr: int) -> None:
        self._c("mcg_set_stream", C.c_void_p(stream_ptr))

    def synchronize(self) -> None:
        self._c("mcg_synchronize")

    # -- initial conditions (launch.cuh:13-29) ------------------------------
    def launch_jetDensity_and_Injet(self) -> None:
        self._c("mcg_init_jet")

    init_jet = launch_jetDensity_and_Injet

    def launch_bubble(self) -> None:
        self._c("mcg_init_bubble")

    init_bubble = launch_bubble

    def init_equilibrium(self, rhor, rhob, ux, uy, uz) -> None:
        """Per-colour equilibrium feq(rho_c, u) at every interior node (the
        bubble and jet initial states are the u = 0 case)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float32).reshape(-1) for a in (rhor, rhob, ux, uy, uz)]
        assert all(a.size == self.N for a in arrs)
        self._c("mcg_init_equilibrium", *[_fptr(a) for a in arrs])

    def set_jet_adjoint_tapes(self, tapes: int) -> None:
        """Segment tapes of the jet adjoints (mcg_set_jet_adjoint_tapes; 0: as
        many as device memory allows)."""
        self._c("mcg_set_jet_adjoint_tapes", int(tapes))

    def adjoint_jet_run(self, nsteps: int, t_begin: int, t_end: int, y_obs: int, segment: int = 0) -> Dict:
        """J = sum over steps t_begin..t_end of (1/2) sum_{y >= y_obs} uy^2 and
        dJ/dc of the inlet-profile coefficients (8 values), from one forward +
        reverse sweep of the jet (snapshots every `segment` steps when 0 <
        segment < nsteps); the state is unchanged."""
        J = C.c_double()
        dc = (C.c_double * 8)()
        fwd, ms = C.c_int64(), C.c_float()
        self._c("mcg_adjoint_jet_run", int(nsteps), int(t_begin), int(t_end), int(y_obs), int(segment), C.byref(J),
                dc, C.byref(fwd), C.byref(ms))
        return {"J": J.value, "dJ_dc": np.array(dc[:], np.float64), "forward_steps": int(fwd.value),
                "ms": float(ms.value)}

    def adjoint_jet_profile_run(self, nsteps: int, t_begin: int, t_end: int, y_lo: int, y_hi: int, uc_target,
                                rhalf_target, segment: int = 0) -> Dict:
        """J = 1/2 sum_{y_lo <= y <= y_hi} ((uc - uc*)/U)^2 + ((r_half - r_half*)/D)^2
        of the time-averaged centreline velocity and half-width over steps
        t_begin..t_end, and dJ/dc of the inlet-profile coefficients, from one
        forward + reverse sweep of the jet; the state is unchanged."""
        uct = np.ascontiguousarray(uc_target, dtype=np.float32).reshape(-1)
        rht = np.ascontiguousarray(rhalf_target, dtype=np.float32).reshape(-1)
        assert uct.size == self.NY and rht.size == self.NY
        J = C.c_double()
        dc = (C.c_double * 8)()
        fwd, ms = C.c_int64(), C.c_float()
        self._c("mcg_adjoint_jet_profile_run", int(nsteps), int(t_begin), int(t_end), int(y_lo), int(y_hi),
                _fptr(uct), _fptr(rht), int(segment), C.byref(J), dc, C.byref(fwd), C.byref(ms))
        return {"J": J.value, "dJ_dc": np.array(dc[:], np.float64), "forward_steps": int(fwd.value),
                "ms": float(ms.value)}

    def jet_profile_metrics(self):
        """(uc[NY], r_half[NY]) of the radial statistics accumulated so far:
        the centreline velocity and the half-width (NaN where undefined)."""
        uc = np.empty(self.NY, np.float32)
        rh = np.empty(self.NY, np.float32)
        self._c("mcg_jet_profile_metrics", _fptr(uc), _fptr(rh))
        return uc, rh

    # -- inlet profile ---------------------------------------------------------
    def set_inlet_bessel(self, coeffs) -> None:
        """Inlet velocity U (1 + sum_k c_k J0(alpha_k r / R)) in jet columns
        (alpha_k the zeros of J0); an empty sequence restores the top-hat."""
        c = np.ascontiguousarray(coeffs, dtype=np.float32).reshape(-1)
        self._c("mcg_set_inlet_bessel", _fptr(c) if c.size else None, int(c.size))

    def inlet_profile(self) -> np.ndarray:
        """Per-column inlet velocity multipliers, (NZ, NX)."""
        out = np.empty(self.case["NX"] * self.case["NZ"], np.float32)
        self._c("mcg_get_inlet_profile", _fptr(out))
        return out.reshape(self.case["NZ"], self.case["NX"])

    # -- discrete adjoint (periodic box, float32 storage) ----------------------
    def adjoint_run(self, psi_target, nsteps: int, snapshots: int, tape: Optional[int] = None) -> Dict:
        """J = sum (psi_T - psi_target)^2 over interior nodes after `nsteps`
        steps from the current state, with dJ/dsigma, dJ/dtau and dJ/du0
        ((3, Ncells) float32) from one reverse sweep; the state is unchanged.
        `tape`: moment records of the innermost taped segments
        (mcg_set_adjoint_tape; None keeps the handle's setting, 20 by default)."""
        tgt = np.ascontiguousarray(psi_target, dtype=np.float32).reshape(-1)
        assert tgt.size == self.N
        if tape is not None:
            self._c("mcg_set_adjoint_tape", int(tape))
        J, ds, dt = C.c_double(), C.c_double(), C.c_double()
        du0 = np.empty(3 * self.N, np.float32)
        fwd, ms = C.c_int64(), C.c_float()
        self._c("mcg_adjoint_run", _fptr(tgt), int(nsteps), int(snapshots), C.byref(J), C.byref(ds), C.byref(dt),
                _fptr(du0), C.byref(fwd), C.byref(ms))
        return {"J": J.value, "dJ_dsigma": ds.value, "dJ_dtau": dt.value, "dJ_du0": du0.reshape(3, self.N),
                "forward_steps": int(fwd.value), "ms": float(ms.value)}

    # -- the per-step sequence (main.cu:52-82) -------------------------------
    def launch_Macros(self) -> None:
        self._c("mcg_macros")

    def launch_accumulate_radial_moments(self) -> None:
        self._c("mcg_accumulate_radial_moments")

    def launch_collistream(self) -> None:
        self._c("mcg_collistream")

    def launch_inlet_bc(self) -> None:
        self._c("mcg_inlet_bc")

    def launch_neumann_bc(self) -> None:
        self._c("mcg_neumann_bc")

    def step(self, nsteps: int = 1) -> None:
        self._c("mcg_step", int(nsteps))

    def step_timed(self, nsteps: int) -> float:
        ms = C.c_float()
        self._c("mcg_step_timed", int(nsteps), C.byref(ms))
        return float(ms.value)

    def step_profiled(self, nsteps: int):
        """(total ms, {fused, boundary} ms) with an event between launches."""
        tot = C.c_float()
        ks = (C.c_float * 3)()
        self._c("mcg_step_profiled", int(nsteps), C.byref(tot), ks)
        return float(tot.value), {"fused": ks[0], "boundary": ks[1]}

    @property
    def current_step(self) -> int:
        s = C.c_int64()
        self._c("mcg_get_step", C.byref(s))
        return int(s.value)

    @property
    def launches(self) -> int:
        n = C.c_uint64()
        self._c("mcg_launch_count", C.byref(n))
        return int(n.value)

    # -- state transfer (reference layout f[i*Ncells + id]) -------------------
    def set_populations(self, fr: np.ndarray, fb: np.ndarray) -> None:
        fr = np.ascontiguousarray(fr, dtype=np.float32).reshape(-1)
        fb = np.ascontiguousarray(fb, dtype=np.float32).reshape(-1)
        assert fr.size == Q * self.N and fb.size == Q * self.N
        self._c("mcg_set_populations", _fptr(fr), _fptr(fb))

    def get_populations(self):
        fr = np.empty(Q * self.N, np.float32)
        fb = np.empty(Q * self.N, np.float32)
        self._c("mcg_get_populations", _fptr(fr), _fptr(fb))
        return fr, fb

    def set_fields(self, rhor=None, rhob=None, ux=None, uy=None, uz=None) -> None:
        arrs = []
        for a in (rhor, rhob, ux, uy, uz):
            if a is None:
                arrs.append(None)
            else:
                a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
                assert a.size == self.N
                arrs.append(a)
        self._c("mcg_set_fields", *[(_fptr(a) if a is not None else None) for a in arrs])

    def get_fields(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        """rhor, rhob, ux, uy, uz of the current state; `out` may give the
        destination arrays (float32, Ncells each, e.g. views of pinned memory)."""
        keys = ("rhor", "rhob", "ux", "uy", "uz")
        if out is None:
            out = {k: np.empty(self.N, np.float32) for k in keys}
        for k in keys:
            assert out[k].dtype == np.float32 and out[k].size == self.N and out[k].flags.c_contiguous
        self._c("mcg_get_fields", *[_fptr(out[k]) for k in keys])
        return out

    def get_stress(self) -> np.ndarray:
        pi = np.empty(6 * self.N, np.float32)
        self._c("mcg_get_stress", _fptr(pi))
        return pi

    # -- mean fields (meanF/) --------------------------------------------------
    def set_radial_statistics(self, mode: int) -> None:
        self._c("mcg_set_radial_statistics", int(mode))

    def get_radial(self) -> Dict[str, np.ndarray]:
        M = self.NY * self.NR_BINS
        sums = {k: np.empty(M, np.float64) for k in ("sum_uy", "sum_uy2", "sum_ur", "sum_ur2", "sum_uruy")}
        count = np.empty(M, np.uint64)
        self._c("mcg_get_radial", *[_dptr(sums[k]) for k in ("sum_uy", "sum_uy2", "sum_ur", "sum_ur2", "sum_uruy")],
                count.ctypes.data_as(C.POINTER(C.c_uint64)))
        sums["count"] = count
        return sums

    def radial_state(self):
        st, s0, n = C.c_int32(), C.c_uint32(), C.c_uint32()
        self._c("mcg_get_radial_state", C.byref(st), C.byref(s0), C.byref(n))
        return bool(st.value), int(s0.value), int(n.value)

    def launch_compute_total_tke(self, step: int):
        tot, avg = C.c_float(), C.c_float()
        self._c("mcg_compute_tke", int(step), C.byref(tot), C.byref(avg))
        return float(tot.value), float(avg.value)

    def launch_update_uy_average(self) -> None:
        self._c("mcg_update_uy_average")

    def get_uy_average(self):
        a = np.empty(self.N, np.float32)
        n = C.c_uint32()
        self._c("mcg_get_uy_average", _fptr(a), C.byref(n))
        return a, int(n.value)

    # -- diagnostics -------------------------------------------------------------
    def conservation_sums(self) -> np.ndarray:
        out = np.zeros(5, np.float64)
        self._c("mcg_conservation_sums", _dptr(out))
        return out

    def check_finite(self) -> bool:
        st = self.lib.mcg_check_finite(self._h)
        if st == 4:
            return False
        _lib.check(st, "mcg_check_finite")
        return True

    # -- output files --------------------------------------------------------------
    def output_open(self, root_dir: str) -> None:
        self._c("mcg_output_open", str(root_dir).encode())

    def output_step(self, step: int) -> None:
        self._c("mcg_output_step", int(step))

    def output_step_async(self, step: int) -> None:
        """mcg_output_step without stopping the GPU; files appear after output_flush."""
        self._c("mcg_output_step_async", int(step))

    def tiling(self) -> dict:
        """Launch shape of the fused step (mcg_get_tiling)."""
        out = np.zeros(8, np.int32)
        self._c("mcg_get_tiling", out.ctypes.data_as(C.POINTER(C.c_int32)))
        keys = ("rows_per_tile", "planes_per_chunk", "threads_per_row", "y_tiles", "z_chunks", "smem_bytes",
                "pipelined", "fixed_row_length")
        return {k: int(v) for k, v in zip(keys, out)}

    def set_stage_wait_limit(self, tries: int) -> None:
        """Tries of a staged-row wait of the bulk-staged march
        (mcg_set_stage_wait_limit; 0 makes every wait run out)."""
        self._c("mcg_set_stage_wait_limit", int(tries))

    def output_flush(self) -> None:
        self._c("mcg_output_flush")

    def write_radial_outputs(self) -> None:
        self._c("mcg_write_radial_outputs")

    def write_vti(self, path: str) -> None:
        self._c("mcg_write_vti", str(path).encode())

    def write_uy_average(self) -> None:
        self._c("mcg_write_uy_average")

    def output_dirs(self):
        bufs = [C.create_string_buffer(4096) for _ in range(3)]
        self._c("mcg_output_dirs", bufs[0], bufs[1], bufs[2], C.c_size_t(4096))
        return tuple(b.value.decode() for b in bufs)

    def output_close(self) -> None:
        self._c("mcg_output_close")


def adjoint_plan(nsteps: int, snapshots: int, tape: int = 0):
    """(forward steps, recomputation depth r) of the checkpointing schedule;
    tape > 0: with taped innermost segments of up to tape + 1 ops (what
    adjoint_run runs with that tape setting)."""
    lib = _lib.load()
    f, r = C.c_int64(), C.c_int32()
    _lib.check(lib.mcg_adjoint_plan_taped(int(nsteps), int(snapshots), int(tape), C.byref(f), C.byref(r)),
               "mcg_adjoint_plan_taped")
    return int(f.value), int(r.value)


def device_count() -> int:
    return int(_lib.load().mcg_device_count())


def write_constants_header(case: Dict, path: str) -> None:
    lib = _lib.load()
    p = params_struct(case)
    _lib.check(lib.mcg_write_constants_header(C.byref(p), str(path).encode()), "mcg_write_constants_header")
