"""ctypes binding of libfemd_cuda.so (the C ABI declared in include/femd_cuda.h).

The library is built in place by `python femd_b200/build.py`.  There is no fallback: if the
shared library is missing or does not load, importing this module raises, and every GPU entry
point of femd_b200 fails loudly instead of computing anything on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfemd_cuda.so")

FEMD_OK, FEMD_EINVAL, FEMD_ENOMEM, FEMD_ECUDA, FEMD_EOUTSIDE, FEMD_EZERODIAG, FEMD_ETIMEOUT, FEMD_EABORT, FEMD_EPIVOT = \
    range(9)
PC_ILU0, PC_SSOR = 1, 2
COEF_CONST, COEF_POINTS, COEF_SINSIN, COEF_SINSIN_HELM, COEF_FIELD = range(5)
ASM_FAST, ASM_EXACT = 0, 1


class femd_coef(C.Structure):
    _fields_ = [("kind", C.c_int), ("value", C.c_double), ("points_dev", C.c_void_p), ("field_dev", C.c_void_p),
                ("p", C.c_double * 4)]


class femd_mesh2d(C.Structure):
    _fields_ = [("nverts", C.c_int), ("ncells", C.c_int), ("points_dev", C.c_void_p), ("tris_dev", C.c_void_p)]


class femd_rule(C.Structure):
    _fields_ = [("k", C.c_int), ("nloc", C.c_int), ("nq", C.c_int), ("ref_host", C.c_void_p), ("xi_host", C.c_void_p),
                ("eta_host", C.c_void_p), ("w_host", C.c_void_p)]


class femd_integrand(C.Structure):
    _fields_ = [("code_host", C.c_void_p), ("ncode", C.c_int), ("nreg", C.c_int), ("nconst", C.c_int),
                ("ninput", C.c_int)]


class femd_facet_rule(C.Structure):
    _fields_ = [("k", C.c_int), ("nloc", C.c_int), ("nq", C.c_int), ("xi_host", C.c_void_p), ("eta_host", C.c_void_p),
                ("gw_host", C.c_void_p), ("ref_host", C.c_void_p)]


class femd_cg_result(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("residual", C.c_double), ("breakdown", C.c_int),
                ("status", C.c_int), ("outer", C.c_int), ("seconds", C.c_double)]


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_PI = C.POINTER(C.c_int)

# name: (restype, argtypes)
SIGNATURES = {
    "femd_cuda_last_error": (C.c_char_p, []),
    "femd_cuda_version": (C.c_char_p, []),
    "femd_cuda_kernel_launches": (C.c_longlong, []),
    "femd_cuda_ctx_create": (_I, [_I, C.POINTER(_P)]),
    "femd_cuda_ctx_destroy": (_I, [_P]),
    "femd_cuda_ctx_stream": (_P, [_P]),
    "femd_cuda_ctx_sync": (_I, [_P]),
    "femd_cuda_release": (None, [_P]),
    "femd_cuda_pattern_from_cells": (_I, [_P, _I, _I, _I, _P, C.POINTER(_P)]),
    "femd_cuda_pattern_info": (_I, [_P, _PI, _PI, C.POINTER(C.c_longlong)]),
    "femd_cuda_pattern_arrays": (_I, [_P, C.POINTER(_P), C.POINTER(_P)]),
    "femd_cuda_pattern_to_host": (_I, [_P, _P, _P]),
    "femd_cuda_pattern_from_csr_host": (_I, [_P, _I, _I, _P, _P, C.POINTER(_P)]),
    "femd_cuda_scatter_map": (_I, [_P, _P, _P]),
    "femd_cuda_pattern_map": (_I, [_P, C.POINTER(_P)]),
    "femd_cuda_matrix_create": (_I, [_P, _P, C.POINTER(_P)]),
    "femd_cuda_matrix_arrays": (_I, [_P, C.POINTER(_P), C.POINTER(_P)]),
    "femd_cuda_matrix_set_host": (_I, [_P, _P]),
    "femd_cuda_matrix_to_host": (_I, [_P, _P]),
    "femd_cuda_matrix_jacobi": (_I, [_P, _P]),
    "femd_cuda_matrix_set_inv_diag": (_I, [_P, _P, _P]),
    "femd_cuda_matrix_inv_diag_to_host": (_I, [_P, _P]),
    "femd_cuda_assemble_matrix": (_I, [_P, C.POINTER(femd_mesh2d), C.POINTER(femd_rule), _P, _I, _P, _P,
                                       C.POINTER(femd_coef), _I, _P, _I]),
    "femd_cuda_assemble_vector": (_I, [_P, C.POINTER(femd_mesh2d), C.POINTER(femd_rule), _P, _I, _P,
                                       C.POINTER(femd_coef), _I, _P]),
    "femd_cuda_integrand_eval": (_I, [_P, C.POINTER(femd_integrand), _P, _P, C.c_longlong, _P, _P, _P, _P, _P]),
    "femd_cuda_integrand_eval_cells": (_I, [_P, C.POINTER(femd_integrand), _P, _P, C.POINTER(femd_mesh2d),
                                            C.POINTER(femd_rule), _P]),
    "femd_cuda_eval_field": (_I, [_P, C.POINTER(femd_mesh2d), C.POINTER(femd_rule), _P, _P, _I, _P, _P]),
    "femd_cuda_facets_create": (_I, [_P, _P, _I, _P, _P, C.POINTER(_P)]),
    "femd_cuda_facet_points": (_I, [_P, _P, C.POINTER(femd_mesh2d), C.POINTER(femd_facet_rule), _P, _P, _P, _P, _P]),
    "femd_cuda_assemble_facet_matrix": (_I, [_P, _P, C.POINTER(femd_mesh2d), C.POINTER(femd_facet_rule), _I, _P, _P,
                                             C.POINTER(femd_coef), _P]),
    "femd_cuda_assemble_facet_vector": (_I, [_P, _P, C.POINTER(femd_mesh2d), C.POINTER(femd_facet_rule), _I, _P,
                                             C.POINTER(femd_coef), _P]),
    "femd_cuda_prolongate": (_I, [_P, _I, _P, _P, _P]),
    "femd_cuda_spmv": (_I, [_P, _P, _P, _P]),
    "femd_cuda_spmv_autotune": (_I, [_P, _P, _I, _PI, C.POINTER(C.c_double)]),
    "femd_cuda_spmv_set_tpr": (_I, [_P, _I]),
    "femd_cuda_asymmetry": (_I, [_P, _P, C.POINTER(C.c_double)]),
    "femd_cuda_combine": (_I, [_P, _D, _P, _D, _P, _P]),
    "femd_cuda_cg_jacobi": (_I, [_P, _P, _I, _P, _P, _I, _D, C.POINTER(femd_cg_result)]),
    "femd_cuda_cg_solve_host": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _P, _I, _D, C.POINTER(femd_cg_result)]),
    "femd_cuda_kernel_time": (_I, [_P, _P, _I, _I, C.POINTER(C.c_double)]),
    "femd_cuda_precond_create": (_I, [_P, _P, _I, _D, C.POINTER(_P)]),
    "femd_cuda_precond_info": (_I, [_P, _PI, _PI, _PI, C.POINTER(C.c_double)]),
    "femd_cuda_precond_apply": (_I, [_P, _P, _P, _P]),
    "femd_cuda_cg_precond": (_I, [_P, _P, _P, _P, _P, _I, _D, C.POINTER(femd_cg_result)]),
    "femd_cuda_pcg_mixed": (_I, [_P, _P, _P, _P, _I, _D, C.POINTER(femd_cg_result)]),
    "femd_cuda_cg_jacobi_noalloc": (_I, [_P, _P, _I, _P, _P, _I, _D, C.POINTER(femd_cg_result)]),
    "femd_cuda_batch_create": (_I, [_P, _I, _P, _I, C.POINTER(_P)]),
    "femd_cuda_batch_solve": (_I, [_P, _P, _P, _P, _I, _D, _I, C.POINTER(femd_cg_result)]),
    "femd_cuda_batch_solve_lockstep": (_I, [_P, _P, _P, _P, _I, _D, _I, C.POINTER(femd_cg_result)]),
    "femd_cuda_batch_lockstep_configure": (_I, [_P, _I, _I, _I, _I]),
    "femd_cuda_batch_step_lockstep": (_I, [_P, _P, _I, _PI, _PI, C.POINTER(femd_cg_result)]),
    "femd_cuda_batch_advance_lockstep": (_I, [_P, _P, _I, _I, _PI, _PI, C.POINTER(femd_cg_result)]),
    "femd_cuda_batch_abort": (_I, [_P]),
    "femd_cuda_batch_lockstep_stats": (_I, [_P, C.POINTER(C.c_longlong)]),
    "femd_cuda_pattern_batch_layout": (_I, [_P, _P, C.POINTER(C.c_int)]),
    "femd_cuda_batch_info": (_I, [_P, _PI, _PI, _PI, _PI]),
    "femd_cuda_batch_debug": (_I, [_P, _I, C.c_longlong]),
    "femd_cuda_batch_profile": (_I, [_P, C.POINTER(C.c_longlong)]),
    "femd_cuda_batch_configure": (_I, [_P, _I, _I, _I]),
    "femd_cuda_batch_params": (_I, [_P, _PI, _PI, _PI, _PI]),
    "femd_cuda_batch_tune": (_I, [_P, _P, _P, _P, _I, _D, _I, _PI, C.POINTER(C.c_double)]),
    "femd_cuda_batch_add": (_I, [_P, _P, _PI]),
    "femd_cuda_batch_remove": (_I, [_P, _I]),
    "femd_cuda_batch_arm": (_I, [_P, _I, _P, _P, _I, _D]),
    "femd_cuda_batch_step": (_I, [_P, _P, _I, _I, _PI, _PI, C.POINTER(femd_cg_result)]),
    "femd_cuda_lagrange_numbering": (_I, [_P, _I, _I, _P, _I, _I, _P, _PI, _PI]),
    "femd_host_rectangle_mesh": (_I, [_D, _D, _D, _D, _I, _I, _P, _P]),
    "femd_host_lagrange_numbering": (_I, [_I, _I, _P, _I, _I, _P, _PI, _PI]),
    "femd_host_triangle_quadrature": (_I, [_I, _P, _P, _P]),
    "femd_host_tabulate": (_I, [_I, _I, _P, _P, _P]),
    "femd_host_rcm_order": (_I, [_I, _P, _P, _P]),
    "femd_host_compact_layout": (_I, [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "femd_host_lagrange_raw": (_I, [_I, _I, _P, _I, _P, _PI]),
    "femd_host_lagrange_nodes": (_I, [_I, _P, _P]),
    "femd_host_exterior_facets": (_I, [_I, _I, _P, _P, _D, _D, _D, _D, _P, _P, _P, _P]),
    "femd_host_facet_rule": (_I, [_I, _I, _P, _P, _P, _P]),
}


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python femd_b200/build.py` (nvcc, sm_100a)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = load()


class FemdError(RuntimeError):
    """A failing libfemd_cuda call; .status is the FEMD_E* code."""

    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


def check(status: int, what: str = ""):
    """Raise the exception the reference raises for the same failure (nanobind's mapping:
    std::invalid_argument -> ValueError, std::logic_error / runtime_error -> RuntimeError)."""
    if status == FEMD_OK:
        return
    msg = lib.femd_cuda_last_error().decode() or what
    if status in (FEMD_EINVAL, FEMD_EZERODIAG):
        e = ValueError(msg)
    elif status == FEMD_ENOMEM:
        e = MemoryError(msg)
    elif status in (FEMD_EOUTSIDE, FEMD_EPIVOT):
        e = RuntimeError(msg)
    else:
        e = FemdError(status, msg)
    e.status = status
    raise e
