"""ctypes binding of libtlw.so (the CUDA library; entry points declared in include/tlw.h).

The shared library is built in-tree by ``__graft_entry__.build()`` (or ``python -m trixilw.build``) into
this directory. There is no CPU fallback: if the library is missing or no CUDA device is usable, every
call raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtlw.so")

TLW_OK = 0
TLW_E_ARG = 1
TLW_E_CUDA = 2
TLW_E_NONADMISSIBLE = 3
TLW_E_STATE = 4
TLW_E_UNSUPPORTED = 5

TLW_LW, TLW_MDRK = 0, 1
TLW_FLUX_RUSANOV, TLW_FLUX_HLL = 0, 1
TLW_SPEED_NAIVE, TLW_SPEED_DAVIS = 0, 1
TLW_WHERE_HOST, TLW_WHERE_DEVICE = 0, 1
TLW_STAGE_LW, TLW_STAGE_MDRK1, TLW_STAGE_MDRK2 = 0, 1, 2
TLW_CACHE_U_TRACES, TLW_CACHE_F_TRACES, TLW_CACHE_U2, TLW_CACHE_F2, TLW_CACHE_ALPHA, TLW_CACHE_FN_LOW = 0, 1, 2, 3, 4, 5
TLW_VOLUME_FR, TLW_VOLUME_FR_SHOCK_CAPTURING = 0, 1
TLW_LIMIT_DENSITY, TLW_LIMIT_PRESSURE, TLW_LIMIT_DENSITY_PRESSURE = 0, 1, 2
TLW_BC_DIRICHLET, TLW_BC_SLIP_WALL_VERTICAL, TLW_BC_SLIP_WALL_HORIZONTAL = 0, 1, 2
TLW_WALL_NOSLIP_ADIABATIC, TLW_WALL_NOSLIP_ISOTHERMAL = 1, 2
TLW_RECONSTRUCTION_FIRST_ORDER, TLW_RECONSTRUCTION_MUSCL, TLW_RECONSTRUCTION_MUSCL_HANCOCK = 0, 1, 2

# every symbol include/tlw.h declares
EXPORTED = (
    "tlw_abi_version", "tlw_create", "tlw_destroy", "tlw_set_tree_mesh", "tlw_set_boundary_data", "tlw_rhs",
    "tlw_max_dt", "tlw_set_state", "tlw_get_state", "tlw_step", "tlw_get_time", "tlw_get_cache",
    "tlw_cache_size", "tlw_synchronize", "tlw_get_stream", "tlw_state_pointer", "tlw_last_error",
    "tlw_step_timed", "tlw_step_host", "tlw_set_unstructured_mesh", "tlw_dd_stages", "tlw_dd_halo_values", "tlw_dd_alpha_buffers", "tlw_dd_comm_stream", "tlw_set_source_terms",
    "tlw_probe_fp64_tflops", "tlw_probe_reciprocal", "tlw_rhs_lw_noalloc",
    "tlw_batch_create", "tlw_batch_destroy", "tlw_batch_add_tree_mesh", "tlw_batch_finalize",
    "tlw_batch_set_state", "tlw_batch_get_state", "tlw_batch_step", "tlw_batch_synchronize",
    "tlw_batch_get_stream", "tlw_batch_autotune", "tlw_batch_num_groups", "tlw_batch_last_error",
    "tlw_adjoint_step", "tlw_forward_record", "tlw_adjoint_sweep", "tlw_adjoint_solve", "tlw_adjoint_dt_sequence",
    "tlw_solve_dts", "tlw_set_curved_mesh", "tlw_curved_colors", "tlw_set_tree_mortars",
    "tlw_set_parabolic", "tlw_adaptive_trial", "tlw_adaptive_accept", "tlw_adaptive_begin", "tlw_adaptive_run",
    "tlw_set_positivity_limiter", "tlw_apply_positivity_limiter", "tlw_set_boundary_kinds", "tlw_set_parabolic_walls",
    "tlw_set_curved_boundaries", "tlw_set_reconstruction", "tlw_set_curved_mortars", "tlw_set_curved_mortar_jacobian",
    "tlw_set_halo", "tlw_dd_buffers", "tlw_dd_begin", "tlw_dd_volume", "tlw_dd_finish",
)


class TlwOpts(ctypes.Structure):
    _fields_ = [
        ("polydeg", ctypes.c_int32),
        ("time_discretization", ctypes.c_int32),
        ("surface_flux", ctypes.c_int32),
        ("max_speed", ctypes.c_int32),
        ("gamma", ctypes.c_double),
        ("device", ctypes.c_int32),
        ("volume_integral", ctypes.c_int32),
        ("alpha_max", ctypes.c_double),
        ("alpha_min", ctypes.c_double),
        ("alpha_smooth", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 3),
    ]


class DomainError(ArithmeticError):
    """Raised where the reference raises Julia's DomainError (square root of a negative pressure or
    density), so that adaptive callers can catch it exactly like the reference's ``test_rhs!``."""


class TlwError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libtlw error {code}: {msg}")
        self.code = code


_lib = None


def lib() -> ctypes.CDLL:
    """Load libtlw.so once; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libtlw.so not built at {LIB_PATH}; run __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    dp = ctypes.POINTER(ctypes.c_double)
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.tlw_abi_version.restype = i32
    L.tlw_create.argtypes = [ctypes.POINTER(TlwOpts), ctypes.POINTER(P)]
    L.tlw_destroy.argtypes = [P]
    L.tlw_set_tree_mesh.argtypes = [P, i64, dp, i64, i64p, i64p, i64, i64p, i64p, i64p, i64p]
    L.tlw_set_boundary_data.argtypes = [P, P, P, i32]
    L.tlw_rhs.argtypes = [P, i32, P, P, P, dbl, dbl, i32]
    L.tlw_max_dt.argtypes = [P, P, i32, dbl, dp]
    L.tlw_set_state.argtypes = [P, P, i32, dbl]
    L.tlw_get_state.argtypes = [P, P, i32, dp]
    L.tlw_step.argtypes = [P, i32, dbl, dbl, dbl, i32]
    L.tlw_get_time.argtypes = [P, dp, dp, i64p]
    L.tlw_step_timed.argtypes = [P, i32, dbl, dbl, dbl, dp]
    L.tlw_step_host.argtypes = [P, P, P, dbl, i32, dbl, dbl, dbl]
    L.tlw_set_unstructured_mesh.argtypes = [P, i64, P, P, P, i64, P, P, P, P]
    L.tlw_dd_stages.argtypes = [P]
    L.tlw_dd_stages.restype = i32
    L.tlw_dd_halo_values.argtypes = [P]
    L.tlw_dd_halo_values.restype = i32
    L.tlw_dd_alpha_buffers.argtypes = [P, P, P]
    L.tlw_dd_comm_stream.argtypes = [P, P]
    L.tlw_set_source_terms.argtypes = [P, i32, P]
    L.tlw_probe_fp64_tflops.argtypes = [i32, dp]
    L.tlw_probe_reciprocal.argtypes = [i32, P, P, i64]
    L.tlw_rhs_lw_noalloc.argtypes = [i32, dbl, i32, i32, i64, P, i32, P, P, i32, P, P, P, P, dbl, P]
    L.tlw_get_cache.argtypes = [P, i32, P, i32]
    L.tlw_cache_size.argtypes = [P, i32]
    L.tlw_cache_size.restype = i64
    L.tlw_synchronize.argtypes = [P]
    L.tlw_get_stream.argtypes = [P, ctypes.POINTER(P)]
    L.tlw_state_pointer.argtypes = [P, ctypes.POINTER(P)]
    L.tlw_last_error.argtypes = [P]
    L.tlw_last_error.restype = ctypes.c_char_p
    i32p = ctypes.POINTER(ctypes.c_int32)
    L.tlw_set_curved_mesh.argtypes = [P, i64, dp, dp, i64, i64p, i32p, i64p, i32p, i32p]
    L.tlw_set_tree_mortars.argtypes = [P, i64, i64p, i64p, i64p]
    L.tlw_set_parabolic.argtypes = [P, dbl, dbl]
    L.tlw_set_positivity_limiter.argtypes = [P, i32, P, P]
    L.tlw_apply_positivity_limiter.argtypes = [P]
    L.tlw_set_boundary_kinds.argtypes = [P, P]
    L.tlw_set_parabolic_walls.argtypes = [P, P, P]
    L.tlw_set_curved_boundaries.argtypes = [P, i64, P, P, P]
    L.tlw_set_reconstruction.argtypes = [P, i32]
    L.tlw_set_curved_mortars.argtypes = [P, i64, P, P, P, P, P, P]
    L.tlw_set_curved_mortar_jacobian.argtypes = [P, P]
    L.tlw_set_halo.argtypes = [P, i64, P, P]
    L.tlw_dd_buffers.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P)]
    L.tlw_dd_begin.argtypes = [P, dbl, dbl, dbl]
    L.tlw_dd_volume.argtypes = [P]
    L.tlw_dd_finish.argtypes = [P]
    L.tlw_adaptive_trial.argtypes = [P, dbl, dbl, dbl, dp, ctypes.POINTER(ctypes.c_int32)]
    L.tlw_adaptive_accept.argtypes = [P, dbl]
    L.tlw_adaptive_begin.argtypes = [P, dbl, dbl, P]
    L.tlw_adaptive_run.argtypes = [P, i32, dbl, dbl, P, P, P]
    L.tlw_curved_colors.argtypes = [P]
    L.tlw_curved_colors.restype = i32
    L.tlw_adjoint_step.argtypes = [P, P, P, P, dbl, i32]
    L.tlw_forward_record.argtypes = [P, P, i32, dbl, i32, P, i32]
    L.tlw_adjoint_sweep.argtypes = [P, P, P, i32, dp]
    L.tlw_adjoint_solve.argtypes = [P, P, i32, dbl, i32, P, P, dp, P, i32, dp]
    L.tlw_adjoint_dt_sequence.argtypes = [P, dp, i32]
    L.tlw_solve_dts.argtypes = [P, P, i32, dp, P, i32]
    L.tlw_batch_create.argtypes = [ctypes.POINTER(TlwOpts), ctypes.POINTER(P)]
    L.tlw_batch_destroy.argtypes = [P]
    L.tlw_batch_add_tree_mesh.argtypes = [P, i32, i64, dp, i64, i64p, i64p, i32p]
    L.tlw_batch_finalize.argtypes = [P]
    L.tlw_batch_set_state.argtypes = [P, i32, P, i32, dbl, dbl, dbl]
    L.tlw_batch_get_state.argtypes = [P, i32, P, i32, dp, i64p]
    L.tlw_batch_step.argtypes = [P, i32, i32]
    L.tlw_batch_synchronize.argtypes = [P]
    L.tlw_batch_get_stream.argtypes = [P, ctypes.POINTER(P)]
    L.tlw_batch_autotune.argtypes = [P, i32, i32p]
    L.tlw_batch_num_groups.argtypes = [P]
    L.tlw_batch_num_groups.restype = i32
    L.tlw_batch_last_error.argtypes = [P]
    L.tlw_batch_last_error.restype = ctypes.c_char_p
    for name in EXPORTED:
        keep = ("tlw_abi_version", "tlw_cache_size", "tlw_last_error", "tlw_batch_num_groups", "tlw_batch_last_error",
                "tlw_curved_colors", "tlw_dd_stages", "tlw_dd_halo_values")
        L[name].restype = L[name].restype if name in keep else ctypes.c_int
    _lib = L
    return L


def check(handle, rc: int, batch: bool = False) -> None:
    if rc == TLW_OK:
        return
    err = lib().tlw_batch_last_error if batch else lib().tlw_last_error
    msg = err(handle).decode() if handle else ""
    if rc == TLW_E_NONADMISSIBLE:
        raise DomainError(msg or "non-admissible state")
    raise TlwError(rc, msg)
