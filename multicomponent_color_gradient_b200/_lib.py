"""ctypes binding of the C ABI in include/mcg.h (libmcg.so, built in-tree).

Loading fails loudly: there is no CPU fallback for the solver.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmcg.so")


class McgParams(C.Structure):
    """struct mcg_params (include/mcg.h), field for field."""

    _fields_ = [
        ("NX", C.c_int32), ("NY", C.c_int32), ("NZ", C.c_int32),
        ("NSTEP", C.c_int32), ("NOUTPUT", C.c_int32), ("NSTATS_START_STEP", C.c_int32),
        ("write_vti_output", C.c_int32), ("sponge_cells", C.c_int32),
        ("jet_radius", C.c_float), ("jet_x0", C.c_float), ("jet_z0", C.c_float), ("jet_velocity", C.c_float),
        ("bubble_radius", C.c_float), ("bubble_x0", C.c_float), ("bubble_y0", C.c_float), ("bubble_z0", C.c_float),
        ("rhor0", C.c_float), ("rhob0", C.c_float),
        ("Re", C.c_float), ("We", C.c_float),
        ("nu", C.c_float), ("taur", C.c_float), ("taub", C.c_float), ("sigma", C.c_float),
        ("beta_recolor", C.c_float), ("sponge_K", C.c_float),
        ("boundary", C.c_int32), ("storage", C.c_int32),
        ("seed", C.c_uint64),
        ("init_noise", C.c_float), ("inlet_noise", C.c_float),
        ("bubble_red_inside", C.c_int32),
        ("reserved", C.c_int32 * 9),
    ]


STATUS = {0: "MCG_OK", 1: "MCG_ERR_INVALID_ARG", 2: "MCG_ERR_OOM", 3: "MCG_ERR_CUDA", 4: "MCG_ERR_NONFINITE",
          5: "MCG_ERR_IO", 6: "MCG_ERR_TIMEOUT", 7: "MCG_ERR_STATE", 8: "MCG_ERR_UNSUPPORTED",
          9: "MCG_ERR_NO_DEVICE"}


class McgError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str):
        super().__init__(f"{what}: {STATUS.get(status, status)}: {detail}")
        self.status = status


_P = C.c_void_p
_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_U64 = C.POINTER(C.c_uint64)
_U32 = C.POINTER(C.c_uint32)
_I32 = C.POINTER(C.c_int32)
_PP = C.POINTER(McgParams)

# name: argtypes (restype is mcg_status = int unless listed in _RESTYPE)
SIGNATURES = {
    "mcg_params_default": [_PP],
    "mcg_params_derive": [_PP],
    "mcg_params_set_tau": [_PP, C.c_float],
    "mcg_write_constants_header": [_PP, C.c_char_p],
    "mcg_create": [_PP, C.POINTER(_P)],
    "mcg_destroy": [_P],
    "mcg_set_stream": [_P, _P],
    "mcg_synchronize": [_P],
    "mcg_get_params": [_P, _PP],
    "mcg_device_bytes": [_P, _U64],
    "mcg_init_jet": [_P],
    "mcg_init_bubble": [_P],
    "mcg_set_populations": [_P, _F, _F],
    "mcg_get_populations": [_P, _F, _F],
    "mcg_set_fields": [_P, _F, _F, _F, _F, _F],
    "mcg_get_fields": [_P, _F, _F, _F, _F, _F],
    "mcg_get_stress": [_P, _F],
    "mcg_macros": [_P],
    "mcg_accumulate_radial_moments": [_P],
    "mcg_collistream": [_P],
    "mcg_inlet_bc": [_P],
    "mcg_neumann_bc": [_P],
    "mcg_step": [_P, C.c_int32],
    "mcg_step_timed": [_P, C.c_int32, _F],
    "mcg_step_profiled": [_P, C.c_int32, _F, _F],
    "mcg_get_step": [_P, C.POINTER(C.c_int64)],
    "mcg_launch_count": [_P, _U64],
    "mcg_set_radial_statistics": [_P, C.c_int32],
    "mcg_get_radial": [_P, _D, _D, _D, _D, _D, _U64],
    "mcg_get_radial_state": [_P, _I32, _U32, _U32],
    "mcg_compute_tke": [_P, C.c_int32, _F, _F],
    "mcg_update_uy_average": [_P],
    "mcg_get_uy_average": [_P, _F, _U32],
    "mcg_conservation_sums": [_P, _D],
    "mcg_check_finite": [_P],
    "mcg_conservation_sums_static": [_P, _P, C.c_int32, C.c_int32, C.c_int32, _P, _P],
    "mcg_init_equilibrium": [_P, _F, _F, _F, _F, _F],
    "mcg_set_inlet_bessel": [_P, _F, C.c_int32],
    "mcg_get_inlet_profile": [_P, _F],
    "mcg_adjoint_run": [_P, _F, C.c_int32, C.c_int32, _D, _D, _D, _F, C.POINTER(C.c_int64), _F],
    "mcg_adjoint_plan": [C.c_int32, C.c_int32, C.POINTER(C.c_int64), _I32],
    "mcg_adjoint_plan_taped": [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int64), _I32],
    "mcg_set_adjoint_tape": [_P, C.c_int32],
    "mcg_set_jet_adjoint_tapes": [_P, C.c_int32],
    "mcg_adjoint_jet_run": [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _D, _D, C.POINTER(C.c_int64),
                            _F],
    "mcg_adjoint_jet_profile_run": [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _F, _F, C.c_int32, _D,
                                    _D, C.POINTER(C.c_int64), _F],
    "mcg_jet_profile_metrics": [_P, _F, _F],
    "mcg_output_open": [_P, C.c_char_p],
    "mcg_output_step": [_P, C.c_int32],
    "mcg_output_step_async": [_P, C.c_int32],
    "mcg_output_flush": [_P],
    "mcg_get_tiling": [_P, _I32],
    "mcg_set_stage_wait_limit": [_P, C.c_int32],
    "mcg_write_radial_outputs": [_P],
    "mcg_write_vti": [_P, C.c_char_p],
    "mcg_write_uy_average": [_P],
    "mcg_output_dirs": [_P, C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t],
    "mcg_output_close": [_P],
    "mcg_last_error_string": [],
    "mcg_status_string": [C.c_int],
    "mcg_abi_version": [],
    "mcg_device_count": [],
}
_RESTYPE = {
    "mcg_last_error_string": C.c_char_p,
    "mcg_status_string": C.c_char_p,
    "mcg_abi_version": C.c_int32,
    "mcg_device_count": C.c_int32,
}

_lib = None


def load() -> C.CDLL:
    """Load libmcg.so from the package directory (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libmcg.so not found at {LIB_PATH}; build it with "
                          "`make -C multicomponent_color_gradient_b200/csrc` (or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, C.c_int)
    _lib = lib
    return lib


def check(status: int, what: str) -> None:
    if status != 0:
        lib = load()
        raise McgError(status, what, lib.mcg_last_error_string().decode(errors="replace"))
