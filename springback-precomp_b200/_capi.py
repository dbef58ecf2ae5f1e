"""ctypes bindings of libsbk.so (the C ABI of include/sbk.h).

The library is loaded from this package's directory only; importing this
module on a machine without the built library, or calling a compute entry
point without a CUDA device, raises - there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbk.so")

SBK_OK = 0
STATUS = {0: "OK", 1: "ARGUMENT", 2: "CONFIG", 3: "MESH", 4: "SOLVER", 5: "CUDA", 6: "UNSUPPORTED",
          7: "NO_EXTENSION"}
ELEMENT_CODES = {0: "OK", 1: "INVERTED_POINT", 2: "RETURN_NO_CONVERGE", 3: "LOCAL_NO_CONVERGE",
                 4: "LOCAL_SINGULAR", 5: "LOCAL_NO_DESCENT", 6: "MESH_INVERTED", 7: "NONFINITE",
                 8: "DEGENERATE", 9: "BAD_NODE"}
KINEMATICS = {"small": 0, "finite": 1, "logarithmic": 2}
MAX_POINTS = 32


class SbkError(RuntimeError):
    """A non-zero status of the C ABI (the reference's exceptions)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class SolverError(SbkError):
    """An element's SolverError: the reference cuts the increment."""

    def __init__(self, status, message, element=-1, code=0):
        super().__init__(status, message)
        self.element = element
        self.code = code
        self.reason = ELEMENT_CODES.get(code, str(code))


class sbk_material(ctypes.Structure):
    _fields_ = [("youngs_modulus", ctypes.c_double), ("poisson_ratio", ctypes.c_double),
                ("yield_stress", ctypes.c_double), ("hardening_modulus", ctypes.c_double),
                ("kinematic_hardening_modulus", ctypes.c_double), ("saturation_stress", ctypes.c_double),
                ("saturation_rate", ctypes.c_double), ("criterion", ctypes.c_int),
                ("num_backstresses", ctypes.c_int), ("kinematic_integration", ctypes.c_int),
                ("reserved", ctypes.c_int), ("backstress_modulus", ctypes.c_double * 4),
                ("backstress_recovery", ctypes.c_double * 4), ("r0", ctypes.c_double), ("r45", ctypes.c_double),
                ("r90", ctypes.c_double), ("shear_l", ctypes.c_double), ("shear_m", ctypes.c_double),
                ("rolling_direction", ctypes.c_double * 3), ("sheet_normal", ctypes.c_double * 3)]


class sbk_rule(ctypes.Structure):
    _fields_ = [("stiffness_points", ctypes.c_int), ("thickness_points", ctypes.c_int),
                ("thickness_axis", ctypes.c_int), ("reserved", ctypes.c_int)]


class sbk_mesh(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int32), ("num_elements", ctypes.c_int32),
                ("coords", ctypes.POINTER(ctypes.c_double)), ("connectivity", ctypes.POINTER(ctypes.c_int32))]


class sbk_pattern(ctypes.Structure):
    _fields_ = [("num_dofs", ctypes.c_int64), ("nnz", ctypes.c_int64), ("outer_dev", ctypes.c_void_p),
                ("inner_dev", ctypes.c_void_p)]


class sbk_evaluation(ctypes.Structure):
    _fields_ = [("internal_dev", ctypes.c_void_p), ("residual_dev", ctypes.c_void_p), ("values_dev", ctypes.c_void_p),
                ("energy", ctypes.c_double), ("gross", ctypes.c_double), ("yielding_points", ctypes.c_int32),
                ("failed_element", ctypes.c_int32), ("failure_code", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class sbk_tool(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int32), ("num_knots", ctypes.c_int32), ("num_slaves", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("radius", ctypes.c_double), ("friction", ctypes.c_double),
                ("tangential_ratio", ctypes.c_double), ("normal", ctypes.c_double * 3),
                ("axis", ctypes.c_double * 3), ("times", ctypes.POINTER(ctypes.c_double)),
                ("points", ctypes.POINTER(ctypes.c_double)), ("nodes", ctypes.POINTER(ctypes.c_int32)),
                ("area", ctypes.POINTER(ctypes.c_double)), ("kappa", ctypes.POINTER(ctypes.c_double))]


class sbk_contact_result(ctypes.Structure):
    _fields_ = [("residual_dev", ctypes.c_void_p), ("block_nodes_dev", ctypes.c_void_p),
                ("blocks_dev", ctypes.c_void_p), ("num_blocks", ctypes.c_int32), ("symmetric", ctypes.c_int32),
                ("gross", ctypes.c_double), ("round_off", ctypes.c_double), ("force_norm", ctypes.c_double),
                ("failed", ctypes.c_int32), ("reserved", ctypes.c_int32)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

# Every symbol the header declares, with its argument types.
SIGNATURES = {
    "sbk_rule_size": (_I, [ctypes.POINTER(sbk_rule)]),
    "sbk_state_fields": (_I, [ctypes.POINTER(sbk_material)]),
    "sbk_yield_matrix": (_I, [ctypes.POINTER(sbk_material), ctypes.POINTER(_D)]),
    "sbk_element_batch": (_I, [ctypes.POINTER(sbk_material), ctypes.POINTER(sbk_rule), _I, _I64] + [_P] * 12 + [_P]),
    "sbk_system_create": (_I, [ctypes.POINTER(sbk_mesh), ctypes.POINTER(sbk_material), ctypes.POINTER(sbk_rule), _I,
                               ctypes.POINTER(_P)]),
    "sbk_system_destroy": (_I, [_P]),
    "sbk_system_set_stream": (_I, [_P, _P]),
    "sbk_system_set_elements_per_block": (_I, [_P, _I]),
    "sbk_set_local_iteration": (_I, [_I]),
    "sbk_system_set_values_buffer": (_I, [_P, _P]),
    "sbk_system_set_local_iteration": (_I, [_P, _I]),
    "sbk_system_set_element": (_I, [_P, _I, _I]),
    "sbk_system_element": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "sbk_system_set_schedule": (_I, [_P, _I]),
    "sbk_system_pattern": (_I, [_P, ctypes.POINTER(sbk_pattern)]),
    "sbk_system_evaluate": (_I, [_P, _P, _D, _I, ctypes.POINTER(sbk_evaluation)]),
    "sbk_system_commit": (_I, [_P]),
    "sbk_system_enqueue": (_I, [_P, _P, _I, _P]),
    "sbk_system_set_stable_buffers": (_I, [_P, _I]),
    "sbk_system_set_timing": (_I, [_P, _I]),
    "sbk_system_last_timings": (_I, [_P, ctypes.POINTER(_D)]),
    "sbk_system_get_committed": (_I, [_P, _P, _P]),
    "sbk_system_set_committed": (_I, [_P, _P, _P]),
    "sbk_system_get_trial": (_I, [_P, _P, _P, _P]),
    "sbk_system_buffers": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    "sbk_system_symmetric": (_I, [_P]),
    "sbk_system_plastic": (_I, [_P]),
    "sbk_system_add_node_blocks": (_I, [_P, _I32, _P, _P]),
    "sbk_system_stiffness_gross": (_I, [_P, _P, _I32, _P, ctypes.POINTER(_D)]),
    "sbk_system_stress": (_I, [_P, _P, _P]),
    "sbk_system_vjp_x": (_I, [_P, _P, _P, _I, _P]),
    "sbk_system_set_frozen": (_I, [_P, _I]),
    "sbk_system_set_coordinates": (_I, [_P, _P]),
    "sbk_contact_create": (_I, [ctypes.POINTER(sbk_mesh), _I32, ctypes.POINTER(sbk_tool), _I, ctypes.POINTER(_P)]),
    "sbk_contact_destroy": (_I, [_P]),
    "sbk_contact_set_stream": (_I, [_P, _P]),
    "sbk_contact_begin": (_I, [_P, _P, _D, _D, _P, _D]),
    "sbk_contact_resultants": (_I, [_P, ctypes.POINTER(_D)]),
    "sbk_contact_evaluate": (_I, [_P, _P, _D, _I, ctypes.POINTER(sbk_contact_result)]),
    "sbk_contact_anticipate": (_I, [_P, _P, _P, _D, _P, ctypes.POINTER(_I32), ctypes.POINTER(sbk_contact_result)]),
    "sbk_contact_commit": (_I, [_P]),
    "sbk_contact_history": (_I, [_P, _I32, _I32, ctypes.POINTER(_D), ctypes.POINTER(_I32)]),
    "sbk_contact_set_search": (_I, [_P, _I]),
    "sbk_contact_candidates": (_I, [_P, _I32, ctypes.POINTER(_I32)]),
    "sbk_evaluate_noalloc": (_I, [ctypes.POINTER(sbk_material), ctypes.POINTER(sbk_rule), _I, _I32, _I32]
                             + [_P] * 7 + [_I64] + [_P] * 7),
    "sbk_partition_create": (_I, [_I64, _P, _P, _I64, _I32, _P, ctypes.POINTER(_P)]),
    "sbk_partition_destroy": (_I, [_P]),
    "sbk_partition_set_stream": (_I, [_P, _P]),
    "sbk_partition_info": (_I, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I64)]),
    "sbk_partition_pattern": (_I, [_P, _P, _P]),
    "sbk_partition_assemble": (_I, [_P, _P, _P]),
    "sbk_partition_restrict": (_I, [_P, _P, _P]),
    "sbk_partition_add_to": (_I, [_P, _P, _P, _D]),
    "sbk_partition_factorize": (_I, [_P, _P, _I, ctypes.POINTER(_I)]),
    "sbk_partition_solve": (_I, [_P, _P, _P]),
    "sbk_partition_solve_transpose": (_I, [_P, _P, _P]),
    "sbk_partition_counts": (_I, [_P, ctypes.POINTER(_I64 * 9)]),
    "sbk_partition_set_dense_limit": (_I, [_P, _I32]),
    "sbk_last_error": (ctypes.c_char_p, []),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                              "(the element loop has no CPU fallback)")
        # torch first: the library's cuSOLVER and cuSPARSE then resolve to
        # the copies torch has loaded, one set of CUDA math libraries per
        # process.
        import torch  # noqa: F401
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().sbk_last_error().decode(errors="replace")


def check(status: int):
    if status != SBK_OK:
        raise SbkError(status, last_error())
