"""ctypes declarations of the C ABI in include/tptfem.h.

Loads ``tpt-fem_b200/lib/libtptfem.so``.  There is no fallback: if the
library is missing or the GPU is unusable, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libtptfem.so")

OK = 0
STATUS_NAMES = {
    0: "OK", 1: "CREATION", 2: "SYMBOLIC", 3: "NUMERIC", 4: "MODEL_DIM_MISMATCH", 5: "NOT_CONVERGED",
    6: "BREAKDOWN", 7: "DEVICE", 8: "TIMEOUT", 9: "INVALID_ARG", 10: "OUT_OF_MEMORY",
}
CELL_TRI3, CELL_QUAD4, CELL_TET4 = 2, 3, 4
MODEL_BAR_AXIAL, MODEL_PLANE_STRESS, MODEL_PLANE_STRAIN, MODEL_CONTINUUM_3D = 0, 1, 2, 3
SOLVER_JACOBI_PCG, SOLVER_MP_PCG, SOLVER_FSAI_MP_PCG, SOLVER_LEARNED_FSAI_PCG = 0, 1, 2, 3
SOLVE_FRESH_SETUP = 1
SOLVE_CSR_ONLY = 2
SOLVE_FULL_OPERATOR = 4
SOLVE_COARSE = 8


class SolverOpts(C.Structure):
    _fields_ = [("solver", C.c_int32), ("max_outer", C.c_int32), ("rel_tol", C.c_double),
                ("inner_rel_tol", C.c_double), ("max_iter", C.c_int64), ("batch", C.c_int32),
                ("flags", C.c_int32), ("coarse_aggregates", C.c_int32), ("reserved", C.c_int32)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("outer_steps", C.c_int32), ("solver_used", C.c_int32),
                ("rel_residual", C.c_double), ("setup_ms", C.c_double), ("solve_ms", C.c_double),
                ("fell_back", C.c_int32), ("coarse_size", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TopoptInstance(C.Structure):
    _fields_ = [("nelx", C.c_int32), ("nely", C.c_int32), ("max_iter", C.c_int32), ("density_filter", C.c_int32),
                ("h", C.c_double), ("e0", C.c_double), ("nu", C.c_double), ("vol_frac", C.c_double),
                ("penal", C.c_double), ("filter_radius", C.c_double), ("move_limit", C.c_double),
                ("emin", C.c_double), ("f", C.c_void_p), ("load_dof", C.c_int64), ("load_value", C.c_double),
                ("bc_dof", C.c_void_p), ("bc_val", C.c_void_p), ("nbc", C.c_int64)]


class TopoptOpts(C.Structure):
    _fields_ = [("rel_tol", C.c_double), ("max_pcg_iter", C.c_int32), ("block_threads", C.c_int32),
                ("use_graph", C.c_int32), ("plain_jacobi", C.c_int32), ("pcg_only", C.c_int32)]


class TopoptStats(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("tune_ms", C.c_double), ("pcg_iterations", C.c_int64),
                ("block_threads", C.c_int32), ("not_converged", C.c_int32), ("refinement_steps", C.c_int64),
                ("direct_instances", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = C.c_void_p
_pp = C.POINTER(C.c_void_p)
_i64 = C.c_int64
_pi64 = C.POINTER(C.c_int64)
_pd = C.POINTER(C.c_double)
_pint = C.POINTER(C.c_int)

SOURCE_FN = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_int, C.c_void_p)
FLUX_FN = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_void_p)
BODY_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_void_p)

SIGNATURES = {
    "tptfem_mesh_quadrature_points": (C.c_int, [_vp, _vp, C.c_int, C.POINTER(C.c_int32), _vp]),
    "tptfem_mesh_boundary_points": (C.c_int, [_vp, _vp, _pi64, _vp, _vp]),
    "tptfem_load_poisson_source_points": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp]),
    "tptfem_load_body_points": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp]),
    "tptfem_apply_neumann_points": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_uint32, _vp]),
    "tptfem_assemble_poisson_robin_points": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, _vp, _pp]),
    "tptfem_solve_poisson_fn": (C.c_int, [_vp, _vp, C.c_double, C.c_int, SOURCE_FN, _vp, _vp, _vp, _i64, FLUX_FN,
                                          _vp, FLUX_FN, _vp, _vp, _vp, _vp]),
    "tptfem_solve_elasticity_fn": (C.c_int, [_vp, _vp, C.c_int, C.c_double, C.c_double, C.c_int, BODY_FN, _vp,
                                             _vp, _vp, _i64, _vp, _vp, _vp]),
    "tptfem_system_refresh": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "tptfem_system_coarse": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                       C.c_void_p, C.c_void_p]),
    "tptfem_topopt_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    "tptfem_topopt_element_stiffness": (C.c_int, [C.c_double, C.c_double, C.c_void_p]),
    "tptfem_grf_eval": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_double,
                                  C.c_void_p]),
    "tptfem_version": (C.c_char_p, []),
    "tptfem_create": (C.c_int, [C.c_int, _pp]),
    "tptfem_destroy": (None, [_vp]),
    "tptfem_last_error": (C.c_size_t, [_vp, C.c_char_p, C.c_size_t]),
    "tptfem_synchronize": (C.c_int, [_vp]),
    "tptfem_mesh_upload": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _i64, _vp, _i64, _pp]),
    "tptfem_mesh_box": (C.c_int, [_vp, _vp, _vp, _vp, _pp]),
    "tptfem_mesh_sizes": (C.c_int, [_vp, _pi64, _pi64, _pint, _pint]),
    "tptfem_mesh_download": (C.c_int, [_vp, _vp, _vp, _vp]),
    "tptfem_mesh_free": (None, [_vp]),
    "tptfem_assemble_poisson": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, _pp]),
    "tptfem_mesh_write_vtk": (C.c_int, [_vp, _vp, C.c_char_p, C.c_char_p, C.c_int, _vp, _vp]),
    "tptfem_mesh_write_exodus": (C.c_int, [_vp, _vp, C.c_char_p]),
    "tptfem_lanczos_eigs": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp]),
    "tptfem_dist_create": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _vp, _pp]),
    "tptfem_dist_counts": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "tptfem_dist_buffers": (C.c_int, [_vp, _pp, _pp]),
    "tptfem_dist_start": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_dist_pack": (C.c_int, [_vp, _vp]),
    "tptfem_dist_spmv_dot": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_dist_update": (C.c_int, [_vp, _vp, C.c_double, _vp]),
    "tptfem_dist_direction": (C.c_int, [_vp, _vp, C.c_double]),
    "tptfem_dist_solution": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_dist_free": (None, [_vp]),
    "tptfem_dist_set_precond": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, _vp]),
    "tptfem_dist_coarse_buffers": (C.c_int, [_vp, _pp, _pp]),
    "tptfem_dist_coarse_factor": (C.c_int, [_vp, _vp]),
    "tptfem_dist_precondition": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_dist_residual_begin": (C.c_int, [_vp, _vp]),
    "tptfem_dist_residual_end": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_dist_solve_local": (C.c_int, [_vp, _vp, C.c_int, C.c_double, C.c_int64, _vp, _vp, _vp]),
    "tptfem_dist_solve_local_precond": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int64, _vp,
                                                  _vp, _vp]),
    "tptfem_power_iteration": (C.c_int, [_vp, _vp, C.c_int, C.c_double, _vp, _vp, _vp]),
    "tptfem_assemble_poisson_robin": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                                _pp]),
    "tptfem_assemble_elasticity": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_int, C.c_double, C.c_int, _pp]),
    "tptfem_reassemble": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "tptfem_matrix_sizes": (C.c_int, [_vp, _pi64, _pi64, _pi64]),
    "tptfem_matrix_download": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "tptfem_matrix_free": (None, [_vp]),
    "tptfem_csr_matvec": (C.c_int, [_vp, _vp, _vp, _i64, _vp]),
    "tptfem_load_poisson_source": (C.c_int, [_vp, _vp, C.c_double, C.c_int, _vp]),
    "tptfem_load_body": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp]),
    "tptfem_apply_traction": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_double, _vp, _vp]),
    "tptfem_reduce_system": (C.c_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i64, _pp]),
    "tptfem_system_sizes": (C.c_int, [_vp, _pi64, _pi64]),
    "tptfem_system_download": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "tptfem_system_solve": (C.c_int, [_vp, _vp, C.POINTER(SolverOpts), C.POINTER(SolveStats)]),
    "tptfem_system_solution": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_system_free": (None, [_vp]),
    "tptfem_system_profile_spmv": (C.c_int, [_vp, _vp, C.c_int, _pd, _pd, _pd, _pd, _pd, _pd]),
    "tptfem_matrix_profile_assembly": (C.c_int, [_vp, _vp, C.c_int, _pd]),
    "tptfem_system_fsai": (C.c_int, [_vp, _vp, _pi64]),
    "tptfem_lfsai_param_count": (C.c_int64, []),
    "tptfem_lfsai_create": (C.c_int, [_vp, C.c_uint64, _pp]),
    "tptfem_lfsai_free": (None, [_vp]),
    "tptfem_lfsai_get_params": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_lfsai_set_params": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_lfsai_loss": (C.c_int, [_vp, _vp, _vp, C.c_int32, _pd, _vp]),
    "tptfem_lfsai_adam": (C.c_int, [_vp, _vp, C.c_double, C.c_double]),
    "tptfem_system_attach_lfsai": (C.c_int, [_vp, _vp, _vp]),
    "tptfem_rel_residual_noalloc": (C.c_int, [C.c_int, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _pd, C.c_char_p,
                                              C.c_size_t]),
    "tptfem_system_fsai_download": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "tptfem_solve_with_dirichlet": (C.c_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i64, C.POINTER(SolverOpts), _vp,
                                              C.POINTER(SolveStats)]),
    "tptfem_solve_poisson": (C.c_int, [_vp, _vp, C.c_double, C.c_int, C.c_double, _vp, _vp, _i64,
                                       C.POINTER(SolverOpts), _vp, C.POINTER(SolveStats)]),
    "tptfem_solve_elasticity": (C.c_int, [_vp, _vp, C.c_int, C.c_double, C.c_double, C.c_int, _vp, _vp, _vp, _i64,
                                          C.POINTER(SolverOpts), _vp, C.POINTER(SolveStats)]),
}

_lib = None


def load():
    """Load libtptfem.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libtptfem.so not found at {LIB_PATH}: run __graft_entry__.build() first")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def declared_symbols(header=None):
    """Function names declared in include/tptfem.h (for the export check)."""
    import re
    header = header or os.path.join(os.path.dirname(PKG_ROOT), "include", "tptfem.h")
    text = open(header).read()
    return sorted(set(re.findall(r"\b(tptfem_[a-z0-9_]+)\s*\(", text)))


def ptr(a):
    """Raw data pointer of a contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)
