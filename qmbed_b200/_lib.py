"""ctypes binding of libqmbed_b200.so (the C ABI declared in include/qmbed_b200.h).

The library must exist: there is no CPU fallback. Importing this module on a
machine without the built library raises ``QmbedError`` with build
instructions; calling a GPU entry point without a GPU returns the CUDA error
through the usual status/last-error path.
"""

from __future__ import annotations

import ctypes
import json
import os
from functools import lru_cache
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
LIBRARY = PACKAGE / "libqmbed_b200.so"


class QmbedError(RuntimeError):
    """Error raised by the engine; ``code`` is the C-ABI status value."""

    def __init__(self, message: str, code: int = 0):
        super().__init__(message)
        self.code = code


STATUS = {
    "ok": 0,
    "invalid_operator": 1,
    "invalid_coupling": 2,
    "invalid_site": 3,
    "state_not_in_basis": 4,
    "invalid_sector": 5,
    "incompatible_symmetry": 6,
    "non_hermitian": 7,
    "invalid_options": 8,
    "dimension_mismatch": 9,
    "rank_deficient": 10,
    "unsupported_backend": 11,
    "internal_state": 13,
    "non_convergence": 14,
    "cuda_error": 20,
}


class EigshOptionsC(ctypes.Structure):
    _fields_ = [
        ("eigenpairs", ctypes.c_uint64),
        ("target", ctypes.c_int),
        ("shift", ctypes.c_double),
        ("krylov_dimension", ctypes.c_uint64),
        ("tolerance", ctypes.c_double),
        ("max_iterations", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("mode", ctypes.c_int),
    ]


class EigshInfoC(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_uint64),
        ("reorthogonalization_passes", ctypes.c_uint64),
        ("conditional_second_passes", ctypes.c_uint64),
        ("fp32_iterations", ctypes.c_uint64),
        ("fp64_iterations", ctypes.c_uint64),
        ("operator_applications", ctypes.c_uint64),
        ("converged", ctypes.c_int),
        ("complex_vectors", ctypes.c_int),
    ]


class EigshHintC(ctypes.Structure):
    _fields_ = [
        ("lower", ctypes.c_double),
        ("upper", ctypes.c_double),
        ("gap", ctypes.c_double),
        ("restart_keep", ctypes.c_uint64),
        ("check_steps", ctypes.c_int),
        ("used", ctypes.c_int),
        ("bound_applications", ctypes.c_uint64),
    ]


def library_path() -> Path:
    configured = os.environ.get("QMBED_B200_LIBRARY")
    return Path(configured) if configured else LIBRARY


@lru_cache(maxsize=None)
def lib() -> ctypes.CDLL:
    path = library_path()
    if not path.exists():
        raise QmbedError(
            f"libqmbed_b200.so not found at {path}; build it with `python -m qmbed_b200.build` "
            "(nvcc for sm_100a)", STATUS["unsupported_backend"])
    L = ctypes.CDLL(str(path))
    vp, i, u64, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_double
    P = ctypes.POINTER
    L.qmbed_gpu_last_error.restype = ctypes.c_char_p
    L.qmbed_gpu_device_count.argtypes = [P(i)]
    L.qmbed_gpu_flip_wait_selftest.argtypes = [i, P(i)]
    L.qmbed_gpu_launch_count.argtypes = [P(u64)]
    L.qmbed_gpu_spin_basis_create.argtypes = [i, i, i, i, i, i, i, P(vp)]
    L.qmbed_gpu_basis_destroy.argtypes = [vp]
    L.qmbed_gpu_basis_dimension.argtypes = [vp, P(u64)]
    L.qmbed_gpu_basis_states.argtypes = [vp, u64, u64, vp, vp, vp]
    L.qmbed_gpu_basis_images.argtypes = [vp, vp, vp, u64, vp, vp, vp]
    L.qmbed_gpu_basis_build_seconds.argtypes = [vp, P(d)]
    L.qmbed_gpu_basis_table_images.argtypes = [vp, vp, u64, vp, vp, vp]
    L.qmbed_gpu_operator_set_lookup.argtypes = [vp, i]
    L.qmbed_gpu_operator_apply_rows_device.argtypes = [vp, i, ctypes.c_uint64, ctypes.c_uint64, vp, vp, vp]
    L.qmbed_gpu_operator_lookup_info.argtypes = [vp, P(i), P(i), P(u64), P(d)]
    L.qmbed_gpu_operator_create.argtypes = [vp, i, vp, ctypes.c_char_p, vp, vp, vp, i, i, i, P(vp)]
    L.qmbed_gpu_operator_destroy.argtypes = [vp]
    L.qmbed_gpu_operator_info.argtypes = [vp, P(u64), P(i), P(i), P(u64), P(i), P(d)]
    L.qmbed_gpu_operator_apply_device.argtypes = [vp, i, i, vp, vp, vp, i]
    L.qmbed_gpu_operator_apply_host.argtypes = [vp, i, vp, vp, i]
    L.qmbed_gpu_operator_apply_device_noalloc.argtypes = [vp, i, i, vp, vp, vp]
    L.qmbed_gpu_operator_apply_block_device.argtypes = [vp, i, i, vp, vp, vp, d, d, d, vp]
    L.qmbed_gpu_operator_export_csr.argtypes = [vp, P(u64), vp, vp, vp]
    L.qmbed_gpu_operator_operand_bytes.argtypes = [vp, i, i, P(d)]
    L.qmbed_gpu_eigsh.argtypes = [vp, P(EigshOptionsC), vp, i, vp, vp, vp, P(EigshInfoC)]
    L.qmbed_gpu_eigsh_hinted.argtypes = [vp, P(EigshOptionsC), P(EigshHintC), vp, i, vp, vp, vp, P(EigshInfoC)]
    L.qmbed_gpu_expm_plan.argtypes = [vp, d, d, u64, d, u64, P(u64), P(u64), vp, P(d)]
    L.qmbed_gpu_expm_apply_host.argtypes = [vp, d, d, u64, d, u64, i, vp, vp, u64]
    L.qmbed_gpu_deterministic_start.argtypes = [i, u64, u64, vp]
    L.qmbed_gpu_evolve.argtypes = [vp, vp, i, vp, u64, d, u64, vp, vp]
    L.qmbed_gpu_expm_lanczos.argtypes = [vp, vp, d, u64, vp]
    L.qmbed_gpu_chebyshev_evolve.argtypes = [vp, vp, i, vp, d, d, d, i, i, vp, vp]
    L.qmbed_gpu_chebyshev_evolve_device.argtypes = [vp, vp, i, vp, d, d, d, i, vp]
    L.qmbed_gpu_lanczos_extremes.argtypes = [vp, i, u64, vp]
    L.qmbed_gpu_scan_lowest.argtypes = [i, i, vp, i, vp, i, d, i, u64, vp, vp, vp]
    L.qmbed_gpu_scan_solve.argtypes = [i, i, vp, i, vp, i, d, i, u64, vp, vp, vp, vp, vp]
    L.qmbed_gpu_scan_barrier_selftest.argtypes = [i, P(i)]
    L.qmbed_gpu_lanczos_create.argtypes = [vp, vp, u64, d, P(vp)]
    L.qmbed_gpu_lanczos_destroy.argtypes = [vp]
    L.qmbed_gpu_lanczos_info.argtypes = [vp, P(u64), P(u64), P(d), P(i), P(u64)]
    L.qmbed_gpu_lanczos_ritz.argtypes = [vp, vp, vp, vp, vp]
    L.qmbed_gpu_lanczos_basis.argtypes = [vp, vp]
    L.qmbed_gpu_lanczos_combine.argtypes = [vp, vp, vp]
    L.qmbed_gpu_lanczos_exponential.argtypes = [vp, d, d, vp]
    L.qmbed_gpu_lanczos_thermal.argtypes = [vp, i, i, vp, i, vp, vp, vp]
    L.qmbed_gpu_lanczos_project.argtypes = [vp, i, vp, vp]
    L.qmbed_gpu_thermal_contraction.argtypes = [i, i, vp, vp, i, vp, i, vp, vp, vp]
    L.qmbed_gpu_thermal_iteration.argtypes = [vp, vp, i, vp, u64, d, vp, vp, P(u64)]
    L.qmbed_gpu_shift_create.argtypes = [vp, vp, i, vp, ctypes.c_char_p, vp, vp, vp, P(vp)]
    L.qmbed_gpu_shift_destroy.argtypes = [vp]
    L.qmbed_gpu_shift_apply_host.argtypes = [vp, u64, vp, u64, vp]
    L.qmbed_gpu_shift_apply_device.argtypes = [vp, vp, vp, vp]
    L.qmbed_gpu_spectral_function.argtypes = [vp, vp, u64, vp, i, vp, d, d, u64, d, vp]
    L.qmbed_gpu_ftlm_start.argtypes = [vp, u64, i, vp]
    L.qmbed_gpu_ftlm_sample.argtypes = [vp, i, u64, i, vp, u64, d, vp, vp, vp]
    L.qmbed_gpu_mlp_create.argtypes = [i, i, i, i, i, u64, P(vp)]
    L.qmbed_gpu_mlp_destroy.argtypes = [vp]
    L.qmbed_gpu_mlp_parameter_count.argtypes = [vp, P(u64)]
    L.qmbed_gpu_mlp_get_parameters.argtypes = [vp, vp]
    L.qmbed_gpu_mlp_set_parameters.argtypes = [vp, vp]
    L.qmbed_gpu_mlp_set_scaling.argtypes = [vp, vp, vp, vp, vp]
    L.qmbed_gpu_mlp_get_scaling.argtypes = [vp, vp, vp, vp, vp]
    L.qmbed_gpu_mlp_gradients.argtypes = [vp, vp, vp, i, vp, P(ctypes.c_float)]
    L.qmbed_gpu_mlp_train.argtypes = [vp, vp, vp, i, i, i, ctypes.c_float, u64, P(ctypes.c_float)]
    L.qmbed_gpu_mlp_predict.argtypes = [vp, vp, i, vp]
    for name in ("qmbed_run_json", "qmbed_command_json"):
        getattr(L, name).argtypes = [ctypes.c_char_p]
        getattr(L, name).restype = ctypes.c_void_p
    L.qmbed_string_free.argtypes = [ctypes.c_void_p]
    L.qmbed_string_free.restype = None
    return L


def check(status: int) -> None:
    if status != 0:
        raise QmbedError(lib().qmbed_gpu_last_error().decode(), status)


def call_json(symbol: str, request: dict) -> dict:
    """Send one request through the JSON boundary and decode the response."""
    function = getattr(lib(), symbol)
    pointer = function(json.dumps(request, separators=(",", ":")).encode())
    if not pointer:
        raise QmbedError("QMBED returned a null response")
    try:
        response = json.loads(ctypes.string_at(pointer))
    finally:
        lib().qmbed_string_free(pointer)
    if response.get("status") != "ok":
        raise QmbedError(response.get("error", "unknown QMBED error"))
    return response["result"]


def run(request: dict) -> dict:
    return call_json("qmbed_run_json", request)


def command(request: dict) -> dict:
    return call_json("qmbed_command_json", request)
