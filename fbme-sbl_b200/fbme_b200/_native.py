"""ctypes binding of the C ABI in ``include/fbme_b200.h``.

The shared library ``libfbme_b200.so`` is built in-tree by
``fbme_b200.build``.  There is no fallback: if the library is missing or
fails to load, every entry point raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_float, c_int, c_int32, c_int64, c_size_t, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfbme_b200.so"

FBME_OK = 0
FBME_ERR_INVALID = 1
FBME_ERR_UNSUPPORTED = 2
FBME_ERR_CUDA = 3
FBME_ERR_WORKSPACE = 4

STATUS_NONFINITE = 1
STATUS_CHOLESKY = 2
STATUS_TIMEOUT = 4
STATUS_PCG_BREAKDOWN = 8
STATUS_ITER_CAP = 16

NUM_GROUPS = 14


class FbmeShape(ctypes.Structure):
    _fields_ = [("n1", c_int32), ("n2", c_int32), ("m1", c_int32), ("m2", c_int32)]


class FbmeShapeParams(ctypes.Structure):
    """Per-shape settings of a plan (uneven batches, tuned tile width)."""
    _fields_ = [("shape", FbmeShape), ("uamp_iterations", c_int32), ("uamp_damping", c_float),
                ("exchange_size", c_int32), ("dft_n_tile", c_int32)]


class FbmeConfig(ctypes.Structure):
    _fields_ = [
        ("uamp_iterations", c_int32),
        ("uamp_damping", c_float),
        ("damping", c_float),
        ("initialization_blend", c_float),
        ("initial_noise_fraction", c_float),
        ("fixed_noise_variance", c_float),
        ("min_variance", c_float),
        ("max_precision", c_float),
        ("hyper_shape", c_float),
        ("hyper_rate", c_float),
        ("noise_shape", c_float),
        ("noise_rate", c_float),
        ("noise_update", c_int32),
        ("polish_size", c_int32),
        ("polish_iterations", c_int32),
        ("polish_prune_tail", c_int32),
        ("polish_reinitialize", c_int32),
        ("polish_evidence_gate", c_int32),
        ("polish_damping", c_float),
        ("evidence_margin_factor", c_float),
        ("exchange_size", c_int32),
        ("fixed_budget_diagnostics", c_int32),
        ("cholesky_jitter_multiplier", c_float),
        ("support_false_alarm_budget", c_float),
        ("dft_terms", c_int32),
    ]


class FbmeOutputs(ctypes.Structure):
    _fields_ = [
        ("x", c_void_p),
        ("posterior_variance", c_void_p),
        ("precision", c_void_p),
        ("support_mask", c_void_p),
        ("noise_variance", c_void_p),
        ("effective_dof", c_void_p),
        ("negative_log_evidence", c_void_p),
        ("evidence_trace", c_void_p),
        ("support_exchanges_accepted", c_void_p),
        ("fixed_budget_gamma_residual", c_void_p),
        ("fixed_budget_noise_residual", c_void_p),
        ("fixed_budget_objective_decrease", c_void_p),
        ("fixed_budget_monotone", c_void_p),
        ("support_score_threshold", c_void_p),
        ("active_indices", c_void_p),
        ("active_values", c_void_p),
        ("status", c_void_p),
    ]


class FbmeCertificate(ctypes.Structure):
    _fields_ = [
        ("support_repairs", c_int32),
        ("coordinate_tolerance", c_float),
        ("familywise_ratio_threshold", c_float),
        ("inactive_max_evidence_ratio", c_void_p),
        ("inactive_best_index", c_void_p),
        ("inactive_evidence_gain", c_void_p),
        ("inactive_optimal_variance", c_void_p),
        ("support_repairs_accepted", c_void_p),
        ("active_max_evidence_gain", c_void_p),
        ("active_best_index", c_void_p),
        ("active_optimal_variance", c_void_p),
        ("active_max_deletion_gain", c_void_p),
        ("active_penalized_evidence_gain", c_void_p),
        ("coordinate_stationary", c_void_p),
        ("type2_map_coordinate_stationary", c_void_p),
        ("familywise_no_discovery", c_void_p),
        ("workspace", c_void_p),
        ("workspace_bytes", c_size_t),
    ]


class FbmeState(ctypes.Structure):
    _fields_ = [
        ("mean", c_void_p),
        ("variance", c_void_p),
        ("prior_variance", c_void_p),
        ("message", c_void_p),
        ("prediction", c_void_p),
        ("backprojection", c_void_p),
        ("noise_variance", c_void_p),
        ("data_variance", c_void_p),
    ]


class FbmeCgConfig(ctypes.Structure):
    _fields_ = [
        ("max_iter", c_int32),
        ("min_iter", c_int32),
        ("cg_min_iter", c_int32),
        ("tol", c_float),
        ("convergence_patience", c_int32),
        ("convergence_check_interval", c_int32),
        ("hyper_shape", c_float),
        ("hyper_rate", c_float),
        ("noise_shape", c_float),
        ("noise_rate", c_float),
        ("initial_noise_fraction", c_float),
        ("initialization_blend", c_float),
        ("fixed_noise_variance", c_float),
        ("noise_update", c_int32),
        ("damping", c_float),
        ("cg_damping", c_float),
        ("min_variance", c_float),
        ("max_precision", c_float),
        ("cg_tolerance", c_float),
        ("cg_initial_tolerance", c_float),
        ("cg_max_iter", c_int32),
        ("cg_check_interval", c_int32),
        ("cg_fixed_iterations", c_int32),
        ("preconditioner_rank", c_int32),
        ("probes", c_int32),
        ("initial_probes", c_int32),
        ("adaptive_cg", c_int32),
        ("adaptive_probes", c_int32),
        ("warm_start", c_int32),
        ("jitter_multiplier", c_float),
        ("dft_terms", c_int32),
        ("active_set_start", c_int32),
        ("active_set_check_interval", c_int32),
        ("active_set_min_size", c_int32),
        ("active_set_max_size", c_int32),
        ("active_set_tail_fraction", c_float),
        ("dense", c_int32),
    ]


class FbmeCgOutputs(ctypes.Structure):
    _fields_ = [
        ("x", c_void_p),
        ("posterior_variance", c_void_p),
        ("precision", c_void_p),
        ("noise_variance", c_void_p),
        ("effective_dof", c_void_p),
        ("support_mask", c_void_p),
        ("support_threshold", c_float),
        ("status", c_void_p),
    ]


class FbmeCgInfo(ctypes.Structure):
    _fields_ = [
        ("iterations", c_int32),
        ("converged", c_int32),
        ("relative_change", c_float),
        ("last_cg_iterations", c_int32),
        ("history", POINTER(c_float)),
        ("active_set_size", c_int32),
        ("active_set_iteration", c_int32),
    ]


CG_HISTORY_COLUMNS = ("relative_change", "noise_variance", "effective_dof", "cg_iterations",
                      "hutchinson_probes", "cg_tolerance")

# Every symbol include/fbme_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "fbme_plan_workspace_bytes": (c_size_t, [POINTER(FbmeShape), c_int32, POINTER(FbmeConfig)]),
    "fbme_plan_create": (c_int, [POINTER(FbmeShape), c_int32, POINTER(FbmeConfig), c_void_p,
                                 c_size_t, c_void_p, POINTER(c_void_p)]),
    "fbme_plan_workspace_bytes_ex": (c_size_t, [POINTER(FbmeShape), c_int32, POINTER(FbmeConfig),
                                                POINTER(FbmeShapeParams), c_int32]),
    "fbme_plan_create_ex": (c_int, [POINTER(FbmeShape), c_int32, POINTER(FbmeConfig),
                                    POINTER(FbmeShapeParams), c_int32, c_void_p, c_size_t, c_void_p,
                                    POINTER(c_void_p)]),
    "fbme_plan_bucket_count": (c_int32, [c_void_p]),
    "fbme_plan_bucket": (c_int, [c_void_p, c_int32, POINTER(FbmeShapeParams), POINTER(c_int32)]),
    "fbme_plan_replay": (c_int, [c_void_p, c_void_p, POINTER(FbmeOutputs), c_void_p]),
    "fbme_plan_destroy": (c_int, [c_void_p]),
    "fbme_dft_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "fbme_dft_adjoint": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "fbme_uamp_run": (c_int, [c_void_p, c_void_p, c_void_p]),
    "fbme_polish_run": (c_int, [c_void_p, c_void_p, POINTER(FbmeOutputs), c_void_p]),
    "fbme_plan_state": (c_int, [c_void_p, POINTER(FbmeState)]),
    "fbme_plan_set_observation_mask": (c_int, [c_void_p, c_void_p, c_void_p]),
    "fbme_plan_set_certificate": (c_int, [c_void_p, POINTER(FbmeCertificate)]),
    "fbme_plan_certificate_workspace_bytes": (c_size_t, [c_void_p]),
    "fbme_plan_set_warm_prior_map": (c_int, [c_void_p, c_void_p]),
    "fbme_selftest_workspace_bytes": (c_size_t, []),
    "fbme_selftest_stage_timeout": (c_int, [c_void_p, c_size_t, c_void_p, c_int64, c_void_p]),
    "fbme_uamp_prior_update": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int64, c_float,
                                       c_float, c_float, c_float, c_void_p, c_void_p]),
    "fbme_plan_profile": (c_int, [c_void_p, c_void_p, POINTER(FbmeOutputs), c_void_p,
                                  POINTER(c_float), POINTER(c_int32), c_int32]),
    "fbme_profile_group_name": (c_char_p, [c_int32]),
    "fbme_topk_workspace_bytes": (c_size_t, [c_int64, c_int32, c_int32]),
    "fbme_topk": (c_int, [c_void_p, c_int64, c_int32, c_int32, c_void_p, c_size_t, c_void_p,
                          c_void_p, c_void_p]),
    "fbme_topk_static": (c_int, [c_void_p, c_int64, c_int32, c_int32, c_void_p, c_void_p,
                                 c_void_p]),
    "fbme_topk_static_error": (c_char_p, []),
    "fbme_cg_workspace_bytes": (c_size_t, [POINTER(FbmeShape), c_int32, POINTER(FbmeCgConfig)]),
    "fbme_cg_create": (c_int, [POINTER(FbmeShape), c_int32, POINTER(FbmeCgConfig), c_void_p,
                               c_size_t, c_void_p, POINTER(c_void_p)]),
    "fbme_cg_solve": (c_int, [c_void_p, c_void_p, c_void_p, POINTER(FbmeCgOutputs),
                              POINTER(FbmeCgInfo), c_void_p]),
    "fbme_cg_destroy": (c_int, [c_void_p]),
    "fbme_cg_matvec": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                               c_void_p]),
    "fbme_pcg_solve": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                               c_float, c_void_p, POINTER(c_int32), c_void_p]),
    "fbme_cnn_param_count": (c_int32, []),
    "fbme_cnn_workspace_bytes": (c_size_t, [c_int32, c_int32, c_int32]),
    "fbme_cnn_features": (c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p]),
    "fbme_cnn_forward": (c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_void_p]),
    "fbme_cnn_backward": (c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_void_p,
                                  c_void_p]),
    "fbme_cnn_adam": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_float, c_void_p]),
    "fbme_plan_warm_workspace_bytes": (c_size_t, [POINTER(FbmeShape), c_int32]),
    "fbme_plan_set_warm_start": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "fbme_last_error": (c_char_p, []),
    "fbme_version": (c_char_p, []),
}

_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """Load the native library once; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"FBME native library not built ({LIB_PATH}); run `python -m fbme_b200.build`."
        )
    try:
        handle = ctypes.CDLL(str(LIB_PATH))
    except OSError as exc:  # pragma: no cover - depends on the machine
        raise RuntimeError(f"cannot load {LIB_PATH}: {exc}") from exc
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    _lib = handle
    return handle


def last_error() -> str:
    return lib().fbme_last_error().decode()


def check(rc: int, what: str) -> None:
    """Map an FBME_* return code to the reference's exception types."""
    if rc == FBME_OK:
        return
    msg = f"{what}: {last_error()}"
    if rc in (FBME_ERR_INVALID, FBME_ERR_WORKSPACE):
        raise ValueError(msg)
    if rc == FBME_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)
