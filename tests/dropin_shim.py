"""A ctypes mirror of the Julia extension in INTEGRATION.md (`ext/BLSGPUExt.jl`): GPU methods of the reference's
reset_schur_sparse!, reduce_schur_sparse! and backsubstitute! with the reference's exact positional signatures
(src/schur_reduction.jl:416-436, :489-507, :519-538), dispatching on a GPU workspace that takes the place of the
reference's SchurReductionWorkspace in the linear system. The system's arrays stay host arrays, as in the reference;
the workspace holds the plan and device mirrors, uploads what a call reads and writes back what it outputs, so the
caller (the reference's schur_solve!, src/schur_linear_systems.jl:362-406) runs unchanged: reset, reduce, its own
sparse factorisation of S on the host, back-substitution.

Test infrastructure: device memory comes from torch (plumbing only); every computation is a call of the C ABI.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

DEV = "cuda:0"


class ArgumentError(ValueError):
    pass


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _p64(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


class GPUSchurWorkspace:
    """GPUSchurWorkspace{T}: the plan of a SchurStructure + pattern (0-based copies of the reference's arrays) and
    the device mirrors of the system's buffers; `failed_block` is the reference's ws.failed_block[] (1-based)."""

    def __init__(self, bls, structure, pattern, r_to_s_map, dtype):
        self.lib = bls._lib.gpu()
        self.bls = bls
        self.dtype = dtype
        self.code = bls._lib.BLS_F32 if dtype == torch.float32 else bls._lib.BLS_F64
        ctx = bls.context(0)
        st = structure
        keep = [np.ascontiguousarray(a, np.int64) for a in (
            st.r_dims, st.e_dims, st.eliminated_ptr, st.entry_retained, st.coffsets, st.eoffsets, pattern.block_colptr,
            pattern.block_rowval, pattern.block_row_offsets, pattern.col_heights, pattern.S_colptr, pattern.S_rowval,
            pattern.diag_inds, r_to_s_map)]
        d = bls._lib.bls_schur_plan_desc()
        d.nrblocks, d.neblocks = st.nrblocks, st.neblocks
        (d.r_dims, d.e_dims, d.eliminated_ptr, d.entry_retained, d.coffsets, d.eoffsets, d.block_colptr, d.block_rowval,
         d.block_row_offsets, d.col_heights, d.S_colptr, d.S_rowval, d.diag_inds, d.r_to_s_map) = [_p64(a) for a in keep]
        d.R_length = len(r_to_s_map)
        h = C.c_void_p()
        rc = self.lib.bls_schur_plan_create(ctx, C.byref(d), C.byref(h))
        if rc != 0:
            raise RuntimeError(self.lib.bls_last_error())
        self.plan = h
        self.failed_block = 0
        self.nnz, self.nr, self.ne = pattern.nnz, st.nr, st.ne
        f = lambda n, dt=dtype: torch.zeros(max(n, 1), dtype=dt, device=DEV)
        self.S = f(self.nnz)
        self.g = f(self.nr, torch.float64)
        self.R = f(len(r_to_s_map))
        self.E = f(int(st.E_length))
        self.Cd = f(int(st.C_length))
        self.b_r, self.sc_r, self.s_r = f(self.nr, torch.float64), f(self.nr, torch.float64), f(self.nr, torch.float64)
        self.b_e, self.sc_e, self.s_e = f(self.ne, torch.float64), f(self.ne, torch.float64), f(self.ne, torch.float64)
        self.x_r, self.x_e = f(self.nr, torch.float64), f(self.ne, torch.float64)
        self.pending_reset = False

    def __del__(self):
        if getattr(self, "plan", None) is not None:
            self.lib.bls_schur_plan_destroy(self.plan)
            self.plan = None

    def up(self, dev, host, dtype=None):
        dev[: len(host)].copy_(torch.from_numpy(np.ascontiguousarray(host)).to(dtype or dev.dtype))
        return dev


def _check_damping(lam, scaling, name):
    """check_damping (src/utils.jl:100-107): thrown before anything is written."""
    if not (np.isfinite(lam) and lam >= 0):
        raise ArgumentError(f"lambda must be finite and non-negative, got {lam}")
    bad = ~(np.isfinite(scaling) & (scaling >= 0))
    if bad.any():
        raise ArgumentError(f"{name} must be finite and non-negative, but entry {int(np.argmax(bad)) + 1} is not")


def _scale(ws, dev, s):
    return None if s is None else ws.up(dev, s)


def reset_schur_sparse(nzval, R_nzval, r_to_s_map, diag_inds, scaling_r, lam, ws: GPUSchurWorkspace, s_r=None, S=None):
    """reset_schur_sparse!(nzval, R_nzval, r_to_s_map, diag_inds, scaling_r, lambda, ws, s_r, S): S = R + lambda
    diag(scaling_r) on the device. r_to_s_map, diag_inds and the pattern are the plan's (structure constants passed
    again by the caller); `nzval` on the host is written by the reduce_schur_sparse! that follows, which returns S."""
    _check_damping(lam, scaling_r, "scaling_r")
    ws.up(ws.R, R_nzval)
    ws.up(ws.sc_r, scaling_r)
    rc = ws.lib.bls_reset_schur_sparse(ws.plan, ws.code, _ptr(ws.S), _ptr(ws.R), _ptr(ws.sc_r), C.c_double(lam),
                                       _ptr(_scale(ws, ws.s_r, s_r)))
    if rc < 0:
        raise ArgumentError(ws.lib.bls_last_error())
    ws.failed_block = 0
    ws.pending_reset = True


def reduce_schur_sparse(S_nzval, g_S, b_r, b_e, scaling_e, lam, structure, E_data, C_data, block_colptr, block_rowval,
                        block_row_offsets, col_heights, ws: GPUSchurWorkspace, s_r=None, s_e=None) -> bool:
    """reduce_schur_sparse!(S, g_S, b_r, b_e, scaling_e, lambda, structure, E_data, C_data, block_colptr,
    block_rowval, block_row_offsets, col_heights, ws, s_r, s_e) -> Bool. On false, S and g_S are untouched and
    ws.failed_block is the lowest failing eliminated block (1-based)."""
    _check_damping(lam, scaling_e, "scaling_e")
    if not ws.pending_reset:            # S.nzval already holds the reset system (the caller reset it itself)
        ws.up(ws.S, S_nzval)
    ws.pending_reset = False
    for dev, host in ((ws.b_r, b_r), (ws.b_e, b_e), (ws.sc_e, scaling_e), (ws.E, E_data), (ws.Cd, C_data)):
        ws.up(dev, host)
    fb = C.c_int64(0)
    rc = ws.lib.bls_reduce_schur_sparse(ws.plan, ws.code, _ptr(ws.S), _ptr(ws.g), _ptr(ws.b_r), _ptr(ws.b_e), _ptr(ws.sc_e),
                                        C.c_double(lam), _ptr(ws.E), _ptr(ws.Cd), _ptr(_scale(ws, ws.s_r, s_r)),
                                        _ptr(_scale(ws, ws.s_e, s_e)), C.byref(fb))
    if rc < 0:
        raise ArgumentError(ws.lib.bls_last_error())
    ws.failed_block = int(fb.value)
    if rc != 0:
        return False
    S_nzval[:] = ws.S[: len(S_nzval)].cpu().numpy()
    g_S[:] = ws.g[: len(g_S)].cpu().numpy()
    return True


def backsubstitute(x_e, x_r, structure, C_data, ws: GPUSchurWorkspace, s_r=None, s_e=None):
    """backsubstitute!(x_e, x_r, structure, C_data, ws, s_r, s_e): x_e = z - E^-1 sum C x_r from the last successful
    reduction's caches (C_data's device mirror is the one that reduction read)."""
    ws.up(ws.x_r, x_r)
    rc = ws.lib.bls_backsubstitute(ws.plan, ws.code, _ptr(ws.x_e), _ptr(ws.x_r), _ptr(ws.Cd), _ptr(_scale(ws, ws.s_r, s_r)),
                                   _ptr(_scale(ws, ws.s_e, s_e)))
    if rc < 0:
        raise ArgumentError(ws.lib.bls_last_error())
    x_e[:] = ws.x_e[: len(x_e)].cpu().numpy()
