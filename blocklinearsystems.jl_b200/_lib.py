"""ctypes bindings of libblsgpu.so and libblsscene.so (the C ABI declared in include/blsgpu.h).

The libraries are loaded from this directory. A missing library is an error: there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent

BLS_OK, BLS_NOT_PD, BLS_EINVAL, BLS_EDIM, BLS_EPATTERN, BLS_ECUDA, BLS_EUNSUPPORTED, BLS_ENOMEM = 0, 1, -1, -2, -3, -4, -5, -6
BLS_NOT_CONVERGED = 2
BLS_F64, BLS_F32 = 0, 1

i64 = C.c_int64
p64 = C.POINTER(C.c_int64)
pdbl = C.POINTER(C.c_double)
vp = C.c_void_p


class ArgumentError(ValueError):
    """The reference's ArgumentError."""


class DimensionMismatch(ValueError):
    """The reference's DimensionMismatch."""


class BlsError(RuntimeError):
    """A CUDA or resource error of the device library."""


class bls_schur_plan_desc(C.Structure):
    _fields_ = [
        ("nrblocks", i64), ("neblocks", i64),
        ("r_dims", p64), ("e_dims", p64), ("eliminated_ptr", p64), ("entry_retained", p64), ("coffsets", p64),
        ("eoffsets", p64),
        ("block_colptr", p64), ("block_rowval", p64), ("block_row_offsets", p64), ("col_heights", p64),
        ("S_colptr", p64), ("S_rowval", p64), ("diag_inds", p64), ("r_to_s_map", p64), ("R_length", i64),
    ]


class bls_qr_plan_desc(C.Structure):
    _fields_ = [
        ("nrblocks", i64), ("neblocks", i64), ("ntables", i64),
        ("r_dims", p64), ("e_dims", p64), ("table_nrows", p64), ("table_ncols", p64), ("table_top", p64), ("table_ptr", p64),
        ("entry_retained", p64), ("entry_col", p64), ("raw_offsets", p64), ("residual_offsets", p64),
        ("block_colptr", p64), ("block_rowval", p64), ("block_row_offsets", p64), ("col_heights", p64), ("S_colptr", p64),
    ]


_gpu = None
_scene = None


def _load(name: str) -> C.CDLL:
    path = HERE / name
    if not path.exists():
        raise RuntimeError(f"{path} is missing: build it with `python {HERE / 'build.py'}` (no CPU fallback exists)")
    return C.CDLL(str(path))


def gpu() -> C.CDLL:
    global _gpu
    if _gpu is None:
        L = _load("libblsgpu.so")
        sig = {
            "bls_version": (C.c_int, []),
            "bls_last_error": (C.c_char_p, []),
            "bls_ctx_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
            "bls_ctx_destroy": (C.c_int, [vp]),
            "bls_ctx_set_stream": (C.c_int, [vp, vp]),
            "bls_ctx_synchronize": (C.c_int, [vp]),
            "bls_structure_from_description": (C.c_int, [i64, p64, i64, p64, p64, C.POINTER(C.c_uint8), i64, i64, C.POINTER(vp)]),
            "bls_structure_positional": (C.c_int, [i64, p64, i64, p64, p64, p64, i64, i64, C.POINTER(vp)]),
            "bls_structure_field": (i64, [vp, C.c_char_p, p64]),
            "bls_structure_destroy": (C.c_int, [vp]),
            "bls_schur_pattern_build": (C.c_int, [vp, i64, p64, C.POINTER(vp)]),
            "bls_pattern_field": (i64, [vp, C.c_char_p, p64]),
            "bls_pattern_destroy": (C.c_int, [vp]),
            "bls_build_r_to_s_map": (C.c_int, [vp, vp, p64]),
            "bls_sparse_indices": (i64, [vp, vp, C.c_int, p64, p64, p64]),
            "bls_r_to_s_map_csc": (C.c_int, [i64, p64, p64, p64, p64, p64]),
            "bls_r_to_s_map_blocks_csc": (C.c_int, [i64, p64, p64, p64, p64, i64, p64, p64, p64, p64]),
            "bls_schur_plan_create": (C.c_int, [vp, C.POINTER(bls_schur_plan_desc), C.POINTER(vp)]),
            "bls_schur_plan_destroy": (C.c_int, [vp]),
            "bls_schur_plan_device_bytes": (i64, [vp]),
            "bls_reset_schur_sparse": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_double, vp]),
            "bls_reset_schur_dense": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_double, vp]),
            "bls_reduce_schur_sparse": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, C.c_double, vp, vp, vp, vp, p64]),
            "bls_reset_reduce_schur_sparse_host": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, C.c_double, vp, vp, vp, vp, vp, p64]),
            "bls_reduce_schur_dense": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, C.c_double, vp, vp, vp, vp, p64]),
            "bls_schur_query_status": (C.c_int, [vp, p64]),
            "bls_schur_plan_instrument": (C.c_int, [vp, C.c_int]),
            "bls_schur_plan_set_kernel": (C.c_int, [vp, C.c_int]),
            "bls_schur_plan_set_stage_unit": (C.c_int, [vp, C.c_int]),
            "bls_schur_plan_phase2_kernel": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_char_p, i64]),
            "bls_schur_plan_set_problems": (C.c_int, [vp, i64, p64, p64, p64, p64]),
            "bls_schur_plan_problem_status": (C.c_int, [vp, p64]),
            "bls_schur_plan_counters": (C.c_int, [vp, p64, pdbl, p64]),
            "bls_backsubstitute": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp]),
            "bls_scatter_copy": (C.c_int, [vp, C.c_int, vp, vp, vp, i64]),
            "bls_symmetrify_full": (C.c_int, [vp, C.c_int, i64, p64, p64, p64, p64, vp, p64, i64, vp, i64]),
            "bls_reduce_schur_dense_noalloc": (C.c_int, [vp, C.c_int, i64, i64, i64, vp, vp, vp, vp, vp, vp, vp, C.c_double, vp, vp, p64]),
            "bls_reduce_schur_dense_noalloc_status": (C.c_int, [vp, p64]),
            "bls_qr_structure_from_description": (C.c_int, [i64, p64, i64, p64, p64, p64, C.POINTER(C.c_uint8), i64, i64, C.POINTER(vp)]),
            "bls_qr_structure_positional": (C.c_int, [vp, p64, i64, p64, p64, p64, i64, C.POINTER(vp)]),
            "bls_qr_structure_field": (i64, [vp, C.c_char_p, p64]),
            "bls_qr_structure_schur": (C.c_int, [vp, C.POINTER(vp)]),
            "bls_qr_structure_destroy": (C.c_int, [vp]),
            "bls_qr_plan_create": (C.c_int, [vp, C.POINTER(bls_qr_plan_desc), C.POINTER(vp)]),
            "bls_qr_plan_destroy": (C.c_int, [vp]),
            "bls_qr_plan_set_staging": (C.c_int, [vp, C.c_int]),
            "bls_qr_normal_residual": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_double, vp, vp, vp]),
            "bls_qr_reduce_rhs": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
            "bls_qr_backsubstitute_rhs": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
            "bls_reduce_qr": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, C.c_double, vp, p64]),
            "bls_qr_backsubstitute": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
            "bls_qr_query_status": (C.c_int, [vp, p64]),
            "bls_qr_plan_counters": (i64, [vp]),
            "bls_reduced_normal_sparse": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
            "bls_reduced_normal_dense": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
            "bls_reduced_residual": (C.c_int, [vp, vp, vp, i64]),
            "bls_reduced_mul": (C.c_int, [vp, C.c_int, vp, vp, i64, vp, i64]),
            "bls_reduced_tmul": (C.c_int, [vp, C.c_int, vp, vp, i64, vp, i64]),
            "bls_lsmr_reduced": (C.c_int, [vp, C.c_int, vp, vp, C.c_double, vp, vp, i64, C.c_double, C.c_double, C.c_double, i64,
                                           p64, C.POINTER(C.c_int), pdbl]),
            "bls_reduced_jacobian_dense": (C.c_int, [vp, C.c_int, vp, vp, vp, i64, i64, vp, i64]),
            "bls_reduced_jacobian_sparse": (C.c_int, [vp, C.c_int, vp, vp, i64, i64, p64, p64, vp, vp, i64]),
            "bls_reduced_jacobian_pattern": (i64, [vp, p64, p64]),
            "bls_reduced_diagonal_blocks": (C.c_int, [vp, C.c_int, vp, vp]),
            "bls_assemble_hessian": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, C.c_int, vp]),
            "bls_jtr": (C.c_int, [vp, C.c_int, vp, vp, vp]),
            "bls_jtj_diag": (C.c_int, [vp, C.c_int, vp, vp]),
            "bls_jtj_quadform": (C.c_int, [vp, C.c_int, vp, vp, pdbl]),
            "bls_prepare_scale": (C.c_int, [vp, C.c_int, i64, vp, C.c_double, vp, vp, C.c_int, C.POINTER(C.c_int)]),
            "bls_dense_solver_create": (C.c_int, [vp, i64, C.POINTER(vp)]),
            "bls_dense_solver_destroy": (C.c_int, [vp]),
            "bls_dense_cholesky": (C.c_int, [vp, C.c_int, vp, p64]),
            "bls_dense_cholesky_shifted": (C.c_int, [vp, C.c_int, vp, C.c_double, vp, p64]),
            "bls_dense_cholesky_solve": (C.c_int, [vp, vp, vp]),
            "bls_block_jacobi_create": (C.c_int, [vp, i64, p64, C.POINTER(vp)]),
            "bls_block_jacobi_destroy": (C.c_int, [vp]),
            "bls_factor_diagonal_blocks": (C.c_int, [vp, C.c_int, vp, p64]),
            "bls_solve_diagonal_blocks": (C.c_int, [vp, C.c_int, vp, vp, vp]),
            "bls_pcg_plan_create": (C.c_int, [vp, i64, p64, p64, p64, p64, p64, p64, C.POINTER(vp)]),
            "bls_pcg_plan_destroy": (C.c_int, [vp]),
            "bls_spmv_sym": (C.c_int, [vp, C.c_int, vp, vp, vp]),
            "bls_extract_diagonal_blocks": (C.c_int, [vp, C.c_int, vp, vp]),
            "bls_pcg_solve": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_double, i64, C.c_int, p64, pdbl, p64]),
            "bls_pcg_solve_refined": (C.c_int, [vp, vp, C.c_int, vp, vp, vp, C.c_double, vp, vp, vp, C.c_double, C.c_double, i64, i64,
                                                p64, p64, pdbl, p64]),
            "bls_schur_apply_elimination": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
            "bls_hessian_bilinear": (C.c_int, [vp, C.c_int, vp, C.c_int, vp, vp, vp, vp, pdbl]),
            "bls_hessian_diagonal": (C.c_int, [vp, C.c_int, vp, C.c_int, vp, vp]),
            "bls_pcg_plan_counters": (i64, [vp]),
            "bls_pcg_set_preconditioner": (C.c_int, [vp, vp]),
            "bls_gnn_param_count": (i64, []),
            "bls_gnn_create": (C.c_int, [vp, p64, p64, p64, p64, p64, C.POINTER(vp)]),
            "bls_gnn_destroy": (C.c_int, [vp]),
            "bls_gnn_prepare": (C.c_int, [vp, C.c_int, vp, p64]),
            "bls_gnn_forward": (C.c_int, [vp, vp, C.c_int, vp]),
            "bls_gnn_outputs": (C.c_int, [vp, vp, vp, vp]),
            "bls_gnn_edge_count": (i64, [vp]),
            "bls_gnn_loss_grad": (C.c_int, [vp, C.c_int, vp, vp, vp, i64, pdbl, vp]),
            "bls_adam_step": (C.c_int, [vp, vp, vp, vp, vp, i64, C.c_float, C.c_float, C.c_float, C.c_float, i64]),
        }
        for fn, (res, args) in sig.items():
            f = getattr(L, fn)
            f.restype = res
            f.argtypes = args
        _gpu = L
    return _gpu


def scene_lib() -> C.CDLL:
    global _scene
    if _scene is None:
        L = _load("libblsscene.so")
        L.bls_scene_generate.restype = C.c_int
        L.bls_scene_generate.argtypes = [i64, i64, C.c_int, i64, i64, C.c_double, i64, i64, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_uint64, C.POINTER(vp)]
        L.bls_scene_destroy.argtypes = [vp]
        L.bls_scene_size.restype = i64
        L.bls_scene_size.argtypes = [vp, C.c_int]
        L.bls_scene_arrays.argtypes = [vp, p64, p64, pdbl, pdbl, pdbl]
        L.bls_scene_description.argtypes = [vp, p64, C.POINTER(C.c_uint8), p64, p64]
        L.bls_scene_assemble.argtypes = [vp, p64, p64, p64, p64, p64, p64, p64, i64, p64, pdbl, i64, pdbl, i64, pdbl, i64,
                                         pdbl, i64, pdbl, i64]
        L.bls_scene_assemble_qr.restype = C.c_int
        L.bls_scene_assemble_qr.argtypes = [vp, p64, p64, p64, p64, p64, p64, p64, p64, p64, p64, pdbl, i64, pdbl, i64]
        _scene = L
    return _scene


def check(rc: int, what: str = "") -> int:
    """Raise the reference's exception for a negative status; return BLS_OK / BLS_NOT_PD unchanged."""
    if rc >= 0:
        return rc
    msg = gpu().bls_last_error().decode(errors="replace")
    if what:
        msg = f"{what}: {msg}"
    if rc == BLS_EINVAL or rc == BLS_EPATTERN:
        raise ArgumentError(msg)
    if rc == BLS_EDIM:
        raise DimensionMismatch(msg)
    raise BlsError(f"status {rc}: {msg}")


def ptr64(a):
    """int64 numpy array -> POINTER(c_int64) (None passes through)."""
    if a is None:
        return None
    return a.ctypes.data_as(p64)


def dptr(t):
    """A device tensor's address (None passes through)."""
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())
