"""Device Schur reduction, mirroring the reference's kernel API on device (torch CUDA) tensors.

SchurReductionWorkspace   src/schur_reduction.jl:16-92 (here: the device plan of libblsgpu)
reset_schur_sparse        src/schur_reduction.jl:416-436
reset_schur_dense         src/schur_reduction.jl:389-407
reduce_schur_sparse       src/schur_reduction.jl:489-507 -> bool
reduce_schur_dense        src/schur_reduction.jl:465-479 -> bool
backsubstitute            src/schur_reduction.jl:519-538
scatter_copy              src/SparseBlockLinearSystem.jl:356-362 (copyto!(csc, bsm, scatter_map))
symmetrifyfull(_)         src/SparseBlockLinearSystem.jl:288-341 (symmetrifyfull / symmetrifyfull!)

Element type T of the block storage is the dtype of the tensors: torch.float64 (FP64 throughout) or torch.float32 (the
mixed form: FP32 storage, pair products and accumulation; FP64 damped inverse, z and gradient). Gradients, right-hand
sides, solutions, scalings and scales are float64 tensors, as in the reference. Every call runs the compiled library on
the tensors' device; there is no other implementation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import BLS_F32, BLS_F64, BLS_NOT_PD, ArgumentError, DimensionMismatch, check, dptr, ptr64
from .layout import BlockSystem, SchurPattern, SchurStructure, build_r_to_s_map, build_schur_pattern

_contexts: dict[int, C.c_void_p] = {}


def context(device: int = 0) -> C.c_void_p:
    """The library context of a CUDA device, bound to torch's current stream at each call."""
    if not torch.cuda.is_available():
        raise RuntimeError("libblsgpu needs a CUDA device (none is visible); there is no CPU fallback")
    if device not in _contexts:
        h = C.c_void_p()
        check(_lib.gpu().bls_ctx_create(device, C.byref(h)))
        _contexts[device] = h
    h = _contexts[device]
    _lib.gpu().bls_ctx_set_stream(h, C.c_void_p(torch.cuda.current_stream(device).cuda_stream))
    return h


def _dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float64:
        return BLS_F64
    if t.dtype == torch.float32:
        return BLS_F32
    raise ArgumentError(f"block storage must be float64 or float32, got {t.dtype}")


def _dev(t: torch.Tensor, name: str, n: int | None = None, dtype=None) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ArgumentError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ArgumentError(f"{name} must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise ArgumentError(f"{name} must be {dtype}, got {t.dtype}")
    if n is not None and t.numel() != n:
        raise DimensionMismatch(f"{name} has length {t.numel()}, expected {n}")
    return t


class SchurReductionWorkspace:
    """The device plan of an elimination: the structure and pattern uploaded once, the coupling-pair work lists, and
    the E^-1 / z caches and failure word of the reference's workspace. `failed_block` is the lowest failing
    eliminated block of the last reduction, 1-based, 0 for none (src/schur_reduction.jl:26, :233-257)."""

    def __init__(self, structure: SchurStructure, pattern: SchurPattern | None = None, r_to_s_map: np.ndarray | None = None,
                 *, device: int = 0):
        self.structure = structure
        self.pattern = pattern
        self.device = device
        ctx = context(device)
        st = structure
        self._keep = []

        def arr(a):
            a = np.ascontiguousarray(a, np.int64)
            self._keep.append(a)
            return ptr64(a)

        d = _lib.bls_schur_plan_desc()
        d.nrblocks, d.neblocks = st.nrblocks, st.neblocks
        d.r_dims, d.e_dims = arr(st.r_dims), arr(st.e_dims)
        d.eliminated_ptr, d.entry_retained = arr(st.eliminated_ptr), arr(st.entry_retained)
        d.coffsets, d.eoffsets = arr(st.coffsets), arr(st.eoffsets)
        if pattern is not None:
            if r_to_s_map is None:
                r_to_s_map = build_r_to_s_map(structure, pattern)
            self.r_to_s_map = r_to_s_map
            d.block_colptr, d.block_rowval = arr(pattern.block_colptr), arr(pattern.block_rowval)
            d.block_row_offsets, d.col_heights = arr(pattern.block_row_offsets), arr(pattern.col_heights)
            d.S_colptr, d.S_rowval, d.diag_inds = arr(pattern.S_colptr), arr(pattern.S_rowval), arr(pattern.diag_inds)
            d.r_to_s_map, d.R_length = arr(r_to_s_map), len(r_to_s_map)
        h = C.c_void_p()
        check(_lib.gpu().bls_schur_plan_create(ctx, C.byref(d), C.byref(h)))
        self._h = h
        self._keep = []
        self.failed_block = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_schur_plan_destroy(h)
            self._h = None

    @property
    def handle(self):
        context(self.device)   # bind the current stream
        return self._h

    def device_bytes(self) -> int:
        return int(_lib.gpu().bls_schur_plan_device_bytes(self._h))

    def set_kernel(self, which: str) -> None:
        """Phase-2 kernel of the 6/3 fast path: "stage" (block-column owned: the column's point-side operands staged in
        shared memory, a thread per 6 x 6 block accumulating in registers; the default for a sparse S), "pairs" (block
        owned, six lanes per pair list; the default for a dense S), "lanes" (block owned, a lane per pair, a warp per
        pair list), "columns" (block-column owned, a warp per visit), "tiles" (block-column owned, visits staged in
        chunks; sparse S without conditioning scales, else "pairs") or "points" (point-major, six lanes per pair,
        vector reductions into S)."""
        check(_lib.gpu().bls_schur_plan_set_kernel(self._h, {"columns": 0, "pairs": 1, "lanes": 2, "tiles": 3, "points": 4,
                                                             "stage": 5}[which]))

    def set_stage_unit(self, unit: int) -> None:
        """Rebuild the "stage" schedule of both storage types with units of at most `unit` pairs (one thread's run of
        one S block's pairs between two writes to the column tile); 20 for FP32 storage and 16 for FP64 at plan
        creation."""
        check(_lib.gpu().bls_schur_plan_set_stage_unit(self._h, int(unit)))

    def phase2_kernel_name(self, dtype=torch.float32, *, dense: bool = False, scaled: bool = False) -> str:
        """The phase-2 kernel the next reduction with this storage type launches (as the profiler lists it)."""
        buf = C.create_string_buffer(64)
        check(_lib.gpu().bls_schur_plan_phase2_kernel(self._h, _lib.BLS_F32 if dtype == torch.float32 else _lib.BLS_F64,
                                                      int(dense), int(scaled), buf, 64))
        return buf.value.decode()

    def instrument(self, timing: bool = True) -> None:
        """Bracket the pair kernel of each reduction with CUDA events (read them with counters())."""
        check(_lib.gpu().bls_schur_plan_instrument(self._h, int(timing)))

    def counters(self) -> dict:
        """Device launches since the last read, and the summed pair-kernel time (ms) over its timed launches."""
        n, ms, k = C.c_int64(0), C.c_double(0.0), C.c_int64(0)
        check(_lib.gpu().bls_schur_plan_counters(self._h, C.byref(n), C.byref(ms), C.byref(k)))
        return {"launches": int(n.value), "pair_kernel_ms": float(ms.value), "pair_kernel_launches": int(k.value)}

    def apply_elimination(self, y: torch.Tensor, y0: torch.Tensor, x: torch.Tensor, C_data: torch.Tensor) -> torch.Tensor:
        """y = y0 - C' E^-1 C x in FP64, from the E^-1 of this plan's last successful reduction (y distinct from y0)."""
        st = self.structure
        for name, t in (("y", y), ("y0", y0), ("x", x)):
            _dev(t, name, st.nr, torch.float64)
        T = _dtype_code(_dev(C_data, "C_data", st.C_length))
        check(_lib.gpu().bls_schur_apply_elimination(self.handle, T, dptr(y), dptr(y0), dptr(x), dptr(C_data)))
        return y

    def hessian_bilinear(self, R: torch.Tensor, E_data: torch.Tensor, C_data: torch.Tensor, x: torch.Tensor, y: torch.Tensor,
                         *, dense: bool = False) -> float:
        """dot(x, H, y) (src/linalg.jl:133-262) of the Hessian (R on this plan's pattern, or dense nr x nr column-major;
        E_data, C_data) for x, y = [x_r; x_e], FP64."""
        st = self.structure
        n = st.nr + st.ne
        T = _dtype_code(_dev(R, "R", st.nr * st.nr if dense else self.pattern.nnz))
        _dev(E_data, "E_data", st.E_length, R.dtype)
        _dev(C_data, "C_data", st.C_length, R.dtype)
        _dev(x, "x", n, torch.float64)
        _dev(y, "y", n, torch.float64)
        out = C.c_double(0.0)
        check(_lib.gpu().bls_hessian_bilinear(self.handle, T, dptr(R), int(dense), dptr(E_data), dptr(C_data), dptr(x), dptr(y),
                                              C.byref(out)))
        return float(out.value)

    def hessian_diagonal(self, R: torch.Tensor, E_data: torch.Tensor, *, dense: bool = False) -> torch.Tensor:
        """[diag R; the diagonals of the E blocks], float64 (what prepare_scale! reads on the Hessian side)."""
        st = self.structure
        T = _dtype_code(_dev(R, "R", st.nr * st.nr if dense else self.pattern.nnz))
        _dev(E_data, "E_data", st.E_length, R.dtype)
        d = torch.empty(st.nr + st.ne, dtype=torch.float64, device=R.device)
        check(_lib.gpu().bls_hessian_diagonal(self.handle, T, dptr(R), int(dense), dptr(E_data), dptr(d)))
        return d

    def query_status(self) -> bool:
        fb = C.c_int64(0)
        rc = check(_lib.gpu().bls_schur_query_status(self.handle, C.byref(fb)))
        self.failed_block = int(fb.value)
        return rc == 0


def reset_schur_sparse(nzval: torch.Tensor, R_nzval: torch.Tensor, r_to_s_map, diag_inds, scaling_r: torch.Tensor, lam: float,
                       ws: SchurReductionWorkspace, s_r: torch.Tensor | None = None) -> None:
    """S = R + lam*diag(scaling_r) (scaled by s_r), and the failure word cleared (src/schur_reduction.jl:416-436).
    The r -> s map and diag_inds are the plan's (uploaded once); the ones passed are checked for length only.
    A bad scaling_r leaves nzval untouched and is reported by the next reduction."""
    st, pat = ws.structure, ws.pattern
    if pat is None:
        raise ArgumentError("the workspace was built without a sparse pattern")
    T = _dtype_code(_dev(nzval, "nzval", pat.nnz))
    _dev(R_nzval, "R_nzval", pat.R_length, nzval.dtype)
    if r_to_s_map is not None and len(r_to_s_map) != pat.R_length:
        raise DimensionMismatch("r_to_s_map does not match the retained storage")
    if diag_inds is not None and len(diag_inds) != st.nr:
        raise DimensionMismatch("diag_inds must have one entry per retained variable")
    _dev(scaling_r, "scaling_r", st.nr, torch.float64)
    if s_r is not None:
        _dev(s_r, "s_r", st.nr, torch.float64)
    check(_lib.gpu().bls_reset_schur_sparse(ws.handle, T, dptr(nzval), dptr(R_nzval), dptr(scaling_r), float(lam), dptr(s_r)))


def reset_schur_dense(S: torch.Tensor, R: torch.Tensor, scaling_r: torch.Tensor, lam: float, ws: SchurReductionWorkspace,
                      s_r: torch.Tensor | None = None) -> None:
    """S = R + lam*diag(scaling_r) for a dense column-major nr x nr S (src/schur_reduction.jl:389-407). A torch tensor
    of shape (nr, nr) is taken as the column-major matrix stored in its memory (pass S.T of a row-major matrix)."""
    nr = ws.structure.nr
    T = _dtype_code(_dev(S, "S", nr * nr))
    _dev(R, "R", nr * nr, S.dtype)
    _dev(scaling_r, "scaling_r", nr, torch.float64)
    check(_lib.gpu().bls_reset_schur_dense(ws.handle, T, dptr(S), dptr(R), dptr(scaling_r), float(lam), dptr(s_r)))


def _reduce(fn, S, g_S, b_r, b_e, scaling_e, lam, structure, E_data, C_data, ws, s_r, s_e, sync):
    st = ws.structure
    if structure is not st:
        raise ArgumentError("the structure and the workspace were built for different structures")
    T = _dtype_code(S)
    _dev(g_S, "g_S", st.nr, torch.float64)
    _dev(b_r, "b_r", st.nr, torch.float64)
    _dev(b_e, "b_e", st.ne, torch.float64)
    _dev(scaling_e, "scaling_e", st.ne, torch.float64)
    _dev(E_data, "E_data", st.E_length, S.dtype)
    _dev(C_data, "C_data", st.C_length, S.dtype)
    for name, s, n in (("s_r", s_r, st.nr), ("s_e", s_e, st.ne)):
        if s is not None:
            _dev(s, name, n, torch.float64)
    fb = C.c_int64(0)
    rc = check(fn(ws.handle, T, dptr(S), dptr(g_S), dptr(b_r), dptr(b_e), dptr(scaling_e), float(lam), dptr(E_data),
                  dptr(C_data), dptr(s_r), dptr(s_e), C.byref(fb) if sync else None))
    if not sync:
        return True
    ws.failed_block = int(fb.value)
    return rc != BLS_NOT_PD


def reduce_schur_sparse(S_nzval: torch.Tensor, g_S, b_r, b_e, scaling_e, lam, structure, E_data, C_data, block_colptr,
                        block_rowval, block_row_offsets, col_heights, ws: SchurReductionWorkspace, s_r=None, s_e=None,
                        *, sync: bool = True) -> bool:
    """Two-phase Schur reduction into S.nzval (already holding R plus damping) and g_S (src/schur_reduction.jl:489-507).
    Returns False if an eliminated block is singular or not positive definite (ws.failed_block names the lowest).
    The pattern arrays are the plan's; the ones passed are checked for length only. sync=False launches without
    waiting for the verdict (read it with ws.query_status())."""
    pat = ws.pattern
    if pat is None:
        raise ArgumentError("the workspace was built without a sparse pattern")
    _dev(S_nzval, "S.nzval", pat.nnz)
    if block_colptr is not None and len(block_colptr) != len(pat.block_colptr):
        raise DimensionMismatch("block_colptr does not match the plan's pattern")
    return _reduce(_lib.gpu().bls_reduce_schur_sparse, S_nzval, g_S, b_r, b_e, scaling_e, lam, structure, E_data, C_data, ws,
                   s_r, s_e, sync)


def _host(t, name: str, n: int, dtype) -> torch.Tensor:
    if isinstance(t, np.ndarray):
        t = torch.from_numpy(t)
    if not isinstance(t, torch.Tensor) or t.is_cuda:
        raise ArgumentError(f"{name} must be a host (CPU) tensor or array")
    if not t.is_contiguous():
        raise ArgumentError(f"{name} must be contiguous")
    if t.dtype != dtype:
        raise ArgumentError(f"{name} must be {dtype}, got {t.dtype}")
    if t.numel() != n:
        raise DimensionMismatch(f"{name} has length {t.numel()}, expected {n}")
    return t


def reset_reduce_schur_sparse_host(S_nzval, g_S, R_nzval, scaling_r, lam, b_r, b_e, scaling_e, structure, E_data, C_data,
                                   ws: SchurReductionWorkspace) -> bool:
    """reset_schur_sparse! then reduce_schur_sparse! (src/schur_reduction.jl:416-436, 489-507) on host arrays (CPU
    tensors or numpy arrays; page-locked tensors let the library overlap the copies with the reduction). S_nzval and
    g_S are written only when the reduction succeeds; returns False (ws.failed_block set) when a point block fails.
    Sparse plans on the 6/3 fast path without conditioning scales."""
    st, pat = ws.structure, ws.pattern
    if structure is not st:
        raise ArgumentError("the structure and the workspace were built for different structures")
    if pat is None:
        raise ArgumentError("the workspace was built without a sparse pattern")
    dt = S_nzval.dtype if isinstance(S_nzval, torch.Tensor) else torch.from_numpy(S_nzval[:0]).dtype
    S_nzval = _host(S_nzval, "S.nzval", pat.nnz, dt)
    T = _dtype_code(S_nzval)
    g_S = _host(g_S, "g_S", st.nr, torch.float64)
    R_nzval = _host(R_nzval, "R_nzval", pat.R_length, dt)
    scaling_r = _host(scaling_r, "scaling_r", st.nr, torch.float64)
    b_r = _host(b_r, "b_r", st.nr, torch.float64)
    b_e = _host(b_e, "b_e", st.ne, torch.float64)
    scaling_e = _host(scaling_e, "scaling_e", st.ne, torch.float64)
    E_data = _host(E_data, "E_data", st.E_length, dt)
    C_data = _host(C_data, "C_data", st.C_length, dt)
    fb = C.c_int64(0)
    p = lambda t: C.c_void_p(t.data_ptr())
    rc = check(_lib.gpu().bls_reset_reduce_schur_sparse_host(ws.handle, T, p(S_nzval), p(g_S), p(R_nzval), p(scaling_r), float(lam),
                                                             p(b_r), p(b_e), p(scaling_e), p(E_data), p(C_data), C.byref(fb)))
    ws.failed_block = int(fb.value)
    return rc != BLS_NOT_PD


def reduce_schur_dense(S: torch.Tensor, g_S, b_r, b_e, scaling_e, lam, structure, E_data, C_data, ws: SchurReductionWorkspace,
                       s_r=None, s_e=None, *, sync: bool = True) -> bool:
    """Two-phase Schur reduction into the upper triangle of a dense column-major S (src/schur_reduction.jl:465-479)."""
    _dev(S, "S", ws.structure.nr ** 2)
    return _reduce(_lib.gpu().bls_reduce_schur_dense, S, g_S, b_r, b_e, scaling_e, lam, structure, E_data, C_data, ws, s_r,
                   s_e, sync)


def backsubstitute(x_e: torch.Tensor, x_r: torch.Tensor, structure, C_data: torch.Tensor, ws: SchurReductionWorkspace,
                   s_r=None, s_e=None) -> None:
    """x_e = z - E^-1 sum_r C_er x_r per eliminated block (src/schur_reduction.jl:519-576), from the caches of the last
    successful reduction on `ws`."""
    st = ws.structure
    _dev(x_e, "x_e", st.ne, torch.float64)
    _dev(x_r, "x_r", st.nr, torch.float64)
    T = _dtype_code(_dev(C_data, "C_data", st.C_length))
    check(_lib.gpu().bls_backsubstitute(ws.handle, T, dptr(x_e), dptr(x_r), dptr(C_data), dptr(s_r), dptr(s_e)))


def prepare_scale(s: torch.Tensor, d: torch.Tensor, lam: float, sc: torch.Tensor, dtype=torch.float64, *, stale: bool) -> bool:
    """prepare_scale! (src/conditioning.jl:60-87): s = the conditioning scale of every variable from the diagonal d (as
    filled) and the damping lam * sc, for a system stored in `dtype`; recomputed when `stale` (the first solve of a
    fill) or when some variable has drifted out of [2^-16, 2^16] (|d + lam sc| s^2) and its scale would change. Returns
    whether s was rewritten. Bit-identical to the reference's scales."""
    n = s.numel()
    for name, t in (("s", s), ("d", d), ("sc", sc)):
        _dev(t, name, n, torch.float64)
    T = BLS_F64 if dtype == torch.float64 else BLS_F32 if dtype == torch.float32 else None
    if T is None:
        raise ArgumentError(f"dtype must be float64 or float32, got {dtype}")
    rec = C.c_int(0)
    check(_lib.gpu().bls_prepare_scale(context(s.device.index or 0), T, n, dptr(d), float(lam), dptr(sc), dptr(s), int(stale),
                                       C.byref(rec)))
    return bool(rec.value)


def scatter_copy(dest: torch.Tensor, src: torch.Tensor, scatter_map: torch.Tensor) -> torch.Tensor:
    """copyto!(csc, bsm, scatter_map): dest[i] = src[scatter_map[i]] (src/SparseBlockLinearSystem.jl:356-362)."""
    _dev(scatter_map, "scatter_map", dest.numel(), torch.int64)
    if dest.dtype != src.dtype:
        raise ArgumentError("dest and src must have the same dtype")
    T = _dtype_code(_dev(dest, "dest"))
    _dev(src, "src")
    check(_lib.gpu().bls_scatter_copy(context(dest.device.index or 0), T, dptr(dest), dptr(src), dptr(scatter_map), dest.numel()))
    return dest


def _block_list(bsys: BlockSystem, blocks):
    if blocks is None:
        return None, bsys.size
    b = np.asarray(blocks)
    if b.dtype == bool:   # a mask, as the reference's AbstractVector{Bool}
        if len(b) != len(bsys.blocksizes):
            raise ArgumentError("the block mask has the wrong length")
        b = np.flatnonzero(b)
    b = np.ascontiguousarray(b, np.int64).reshape(-1)
    ok = (b >= 0) & (b < len(bsys.blocksizes))
    return b, int(np.sum(bsys.blocksizes[b[ok]]))


def symmetrifyfull_(mat: torch.Tensor, bsys: BlockSystem, data: torch.Tensor, blocks=None) -> torch.Tensor:
    """symmetrifyfull!(mat, bsm, blocks) (src/SparseBlockLinearSystem.jl:299-341): mat (m x m, column-major, or a
    square tensor, the matrix being symmetric) = the dense symmetric matrix of the blocks of bsys (all, or the 0-based
    `blocks` in the order they take, or a boolean mask), zero elsewhere. Raises ArgumentError for a block out of range
    or listed twice and DimensionMismatch for a wrong size, before any write."""
    T = _dtype_code(_dev(data, "data"))
    _dev(mat, "mat")
    if mat.dtype != data.dtype:
        raise ArgumentError("mat and data must have the same dtype")
    b, _ = _block_list(bsys, blocks)
    n = mat.numel()
    m = int(round(n ** 0.5))
    if m * m != n:
        raise DimensionMismatch(f"target matrix has {n} entries, not a square")
    bs, cp, rv, st = (np.ascontiguousarray(a, np.int64) for a in (bsys.blocksizes, bsys.colptr, bsys.rowval, bsys.starts))
    check(_lib.gpu().bls_symmetrify_full(context(data.device.index or 0), T, len(bs), ptr64(bs), ptr64(cp), ptr64(rv), ptr64(st),
                                         dptr(data), None if b is None else ptr64(b), 0 if b is None else len(b),
                                         dptr(mat) if n else None, m))
    return mat


def symmetrifyfull(bsys: BlockSystem, data: torch.Tensor, blocks=None) -> torch.Tensor:
    """symmetrifyfull(bsm) (src/SparseBlockLinearSystem.jl:288-297), optionally of a block subset: a new m x m
    tensor."""
    _, m = _block_list(bsys, blocks)
    mat = torch.empty(m, m, dtype=data.dtype, device=data.device)
    return symmetrifyfull_(mat, bsys, data, blocks)
