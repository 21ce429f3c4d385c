"""ctypes binding of ``libfj_uvlm.so`` (declarations in ``include/fj_uvlm.h``).

The library is loaded from ``flapjax_b200/_lib/`` (built in-tree by
``flapjax_b200.build``).  There is no fallback: if the library is missing or the
machine has no CUDA device, the calls that need it raise.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libfj_uvlm.so"

FJ_OK = 0
FJ_ERR_SHAPE = -1
FJ_ERR_NONFINITE = -2
FJ_ERR_SINGULAR = -3
FJ_ERR_TIMEOUT = -4
FJ_ERR_NOMEM = -5
FJ_ERR_CUDA = -6
FJ_ERR_UNSUPPORTED = -7
FJ_ERR_NOT_CONVERGED = -8

FJ_KERNEL_EPSILON = 0
FJ_KERNEL_CUTOFF = 1
FJ_KERNEL_PLAIN = 2

FJ_PREC_FP64 = 0
FJ_PREC_MIXED = 1

FJ_FLOW_CONSTANT = 0
FJ_FLOW_ONE_MINUS_COSINE = 1

FJ_MAX_SURF = 8

_D3 = C.c_double * 3
_I8 = C.c_int * FJ_MAX_SURF


class FjFlowfield(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("relative_motion", C.c_int),
        ("u_inf", _D3),
        ("rho", C.c_double),
        ("gust_length", C.c_double),
        ("gust_amplitude", C.c_double),
        ("gust_travel_dir", _D3),
        ("gust_amplitude_dir", _D3),
        ("gust_x0", _D3),
    ]


class FjCaseConfig(C.Structure):
    _fields_ = [
        ("n_surf", C.c_int),
        ("m", _I8),
        ("n", _I8),
        ("m_star", _I8),
        ("n_nodes", C.c_int),
        ("n_tstep", C.c_int),
        ("kernel", C.c_int),
        ("r_cut", C.c_double),
        ("free_wake", C.c_int),
        ("mirror", C.c_int),
        ("mirror_point", _D3),
        ("mirror_normal", _D3),
        ("dt", C.c_double),
        ("gamma_dot_relaxation", C.c_double),
        ("flow", FjFlowfield),
        ("precision", C.c_int),
        ("variable_wake", _I8),
        ("polar_points", _I8),
        ("polar_circulation_scale", C.c_double),
    ]


_P = C.c_void_p


class FjCaseBuffers(C.Structure):
    _fields_ = [
        ("d_zeta_b0", _P),
        ("d_dof_mapping", _P),
        ("d_hg_t", _P),
        ("d_hg_dot_t", _P),
        ("d_delta_w", _P),
        ("d_t", _P),
        ("d_zeta_b", _P),
        ("d_zeta_b_dot", _P),
        ("d_zeta_w", _P),
        ("d_c", _P),
        ("d_nc", _P),
        ("d_gamma_b", _P),
        ("d_gamma_b_dot", _P),
        ("d_gamma_w", _P),
        ("d_f_steady", _P),
        ("d_f_unsteady", _P),
        ("d_alpha", _P),
        ("d_force_total", _P),
        ("d_polars", _P),
    ]


class FjProfile(C.Structure):
    _fields_ = [
        ("launches", C.c_int64),
        ("vind_launches", C.c_int64),
        ("vind_ms", C.c_double),
        ("vind_ms_max", C.c_double),
        ("vind_pairs", C.c_double),
        ("vind64_launches", C.c_int64),
        ("vind64_ms", C.c_double),
        ("vind64_pairs", C.c_double),
    ]


FJ_REUSE_FACTORS = 1
FJ_NO_GRAPH = 2
FJ_REUSE_CONVECTION = 4


class FjBatchItem(C.Structure):
    _fields_ = [
        ("cfg", C.POINTER(FjCaseConfig)),
        ("bufs", C.POINTER(FjCaseBuffers)),
        ("d_ws", C.c_void_p),
        ("ws_bytes", C.c_size_t),
        ("i_ts", C.c_int),
        ("flags", C.c_int),
    ]

# name -> (restype, argtypes)
_SIGS = {
    "fj_last_error_string": (C.c_char_p, []),
    "fj_version": (C.c_int, []),
    "fj_case_workspace_size": (C.c_int, [C.POINTER(FjCaseConfig), C.POINTER(C.c_size_t)]),
    "fj_solve_static": (C.c_int, [C.POINTER(FjCaseConfig), C.POINTER(FjCaseBuffers), C.c_int, C.c_double, _P,
                                  C.c_size_t, _P]),
    "fj_solve_prescribed_dynamic": (C.c_int, [C.POINTER(FjCaseConfig), C.POINTER(FjCaseBuffers), C.c_int, C.c_int,
                                              C.c_int, _P, C.c_size_t, _P]),
    "fj_case_step": (C.c_int, [C.POINTER(FjCaseConfig), C.POINTER(FjCaseBuffers), C.c_int, C.c_int, _P, C.c_size_t,
                               _P]),
    "fj_peak_fp32": (C.c_int, [C.POINTER(C.c_double), _P]),
    "fj_batch_workspace_size": (C.c_int, [C.c_int, C.POINTER(C.c_size_t)]),
    "fj_step_batched": (C.c_int, [C.POINTER(FjBatchItem), C.c_int, _P, C.c_size_t, _P]),
    "fj_batch_release": (C.c_int, [_P]),
    "fj_lti_march": (C.c_int, [_P, C.c_int, _P, C.c_int64, _P, C.c_int64, C.c_int, _P]),
    "fj_batch_graph_stats": (C.c_int, [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "fj_case_residual": (C.c_int, [C.POINTER(FjCaseConfig), _P, C.c_size_t, C.c_int, C.POINTER(C.c_double), _P]),
    "fj_case_factors_copy": (C.c_int, [C.POINTER(FjCaseConfig), _P, C.c_size_t, _P, _P, _P]),
    "fj_rhs_workspace_size": (C.c_int, [C.c_int64, _P, _P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_size_t)]),
    "fj_rhs": (C.c_int, [_P, _P, _P, C.c_int64, C.POINTER(FjFlowfield), C.c_double, _P, _P, _P, _P, C.c_int,
                         _P, _P, C.c_int, C.c_double, C.c_int, _P, _P, C.c_size_t, _P]),
    "fj_wake_shed_convect": (C.c_int, [_P, _P, _P, _P, _P, C.c_int, C.c_int, C.POINTER(FjFlowfield), C.c_double,
                                       C.c_double, _P, _P, _P]),
    "fj_forces_workspace_size": (C.c_int, [C.c_int, C.c_int, _P, _P, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.c_size_t)]),
    "fj_forces": (C.c_int, [_P, _P, _P, _P, _P, C.c_int, C.c_int, C.POINTER(FjFlowfield), C.c_double, _P, _P, _P,
                            _P, C.c_int, _P, _P, C.c_int, C.c_double, C.c_int, _P, _P, _P, C.c_size_t, _P]),
    "fj_aic_vjp_workspace_size": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_size_t)]),
    "fj_aic_vjp": (C.c_int, [_P, C.c_int, C.c_int, _P, _P, C.c_int, _P, _P, C.c_size_t, _P]),
    "fj_wake_vjp": (C.c_int, [_P, _P, C.c_int, C.c_int, _P, _P, _P, _P, _P]),
    "fj_launch_count": (C.c_int64, []),
    "fj_profile_begin": (C.c_int, []),
    "fj_profile_end": (C.c_int, [C.c_void_p]),
    "fj_biot_savart": (C.c_int, [_P, _P, C.c_int64, C.c_int, C.c_double, _P, _P]),
    "fj_vind_workspace_size": (C.c_int, [C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_size_t)]),
    "fj_vind": (C.c_int, [_P, C.c_int64, C.POINTER(_P), C.POINTER(_P), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int,
                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_double, C.c_int, _P, _P,
                          C.c_size_t, _P]),
    "fj_vind_noalloc": (C.c_int, [_P, C.c_int64, C.POINTER(_P), C.POINTER(_P), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int,
                                  C.c_double, C.c_int, _P, _P]),
    "fj_vind_vjp_workspace_size": (C.c_int, [C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_int,
                                             C.POINTER(C.c_size_t)]),
    "fj_vind_vjp": (C.c_int, [_P, C.c_int64, C.POINTER(_P), C.POINTER(_P), C.POINTER(C.c_int), C.POINTER(C.c_int),
                              C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_double, _P, _P,
                              C.POINTER(_P), C.POINTER(_P), _P, C.c_size_t, _P]),
    "fj_lu_solve_t": (C.c_int, [_P, C.c_int, _P, _P, _P, C.c_size_t, _P]),
    "fj_ring_influence": (C.c_int, [_P, C.c_int64, _P, _P, C.c_int, C.c_int, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.c_int, C.c_double, _P, C.c_int64, _P]),
    "fj_vertex_jacobian": (C.c_int, [_P, C.c_int64, _P, _P, _P, C.c_int, C.c_int, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.c_int, C.c_double, _P, C.c_int64, _P]),
    "fj_lu_solve_many_workspace_size": (C.c_int, [C.c_int, C.c_int64, C.POINTER(C.c_size_t)]),
    "fj_lu_solve_many": (C.c_int, [_P, C.c_int, _P, _P, C.c_int64, C.c_int64, _P, C.c_size_t, _P]),
    "fj_aic_workspace_size": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_size_t)]),
    "fj_aic_assemble": (C.c_int, [C.POINTER(_P), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.POINTER(_P),
                                  C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int,
                                  C.c_double, _P, _P, C.c_size_t, _P]),
    "fj_lu_workspace_size": (C.c_int, [C.c_int, C.POINTER(C.c_size_t)]),
    "fj_lu_factor": (C.c_int, [_P, C.c_int, _P, _P, C.c_size_t, _P]),
    "fj_lu_solve": (C.c_int, [_P, C.c_int, _P, _P, _P, C.c_size_t, _P]),
    "fj_solve_mixed_workspace_size": (C.c_int, [C.c_int, C.POINTER(C.c_size_t)]),
    "fj_solve_mixed": (C.c_int, [_P, C.c_int, _P, _P, C.c_int, _P, _P, C.c_size_t, _P]),
    "fj_gemm_tf32": (C.c_int, [_P, C.c_int, _P, C.c_int, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                               C.c_float, C.c_int, _P, _P]),
    "fj_gemm_tf32_scratch_floats": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_size_t)]),
    "fj_gemm_tf32_tma": (C.c_int, [_P, C.c_int, _P, C.c_int, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                   C.c_float, C.c_int, _P, C.c_size_t, _P, _P]),
    "fj_autotune_vind_workspace_size": (C.c_int, [C.c_int, _P, _P, C.c_int, C.POINTER(C.c_size_t)]),
    "fj_autotune_vind": (C.c_int, [C.c_int, C.c_int, C.c_double, _P, _P, C.c_int, _P, _P, _P, _P, _P, C.c_size_t,
                                   _P]),
    "fj_autotune_table_size": (C.c_int, [C.POINTER(C.c_int)]),
    "fj_autotune_get": (C.c_int, [_P, C.c_int]),
    "fj_autotune_set": (C.c_int, [_P, C.c_int]),
    "fj_tc_wait_selftest": (C.c_int, [_P, _P, _P]),
}

EXPORTED = tuple(_SIGS)

_lock = threading.Lock()
_lib = None


class FjError(RuntimeError):
    """A non-zero status from libfj_uvlm; ``.code`` is the FJ_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[fj {code}] {msg}")
        self.code = code


def load(path: Path | None = None) -> C.CDLL:
    """Load (once) and return the library with its prototypes set."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = Path(path) if path is not None else LIB_PATH
        if not p.exists():
            raise FileNotFoundError(
                f"{p} is missing: build it with `python -m flapjax_b200.build` (there is no CPU fallback)"
            )
        lib = C.CDLL(str(p))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = lib
        return lib


def check(status: int) -> None:
    if status != FJ_OK:
        msg = load().fj_last_error_string()
        raise FjError(status, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
