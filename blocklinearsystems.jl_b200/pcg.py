"""Block-Jacobi and PCG on the reduced camera system, on the device.

BlockJacobi / factor_diagonal_blocks / solve_diagonal_blocks    src/diagonal_blocks.jl:6-61
PCGWorkspace.solve                                             no reference counterpart: the iterative solve of
                                                               S x = g that the sparse reduction feeds (the reference
                                                               solves it with CHOLMOD, src/schur_linear_systems.jl:362-406,
                                                               or LSMR with block-Jacobi, ext/KrylovExt.jl:97-132)

S is a reduction's output (the upper blocks on build_schur_pattern's pattern), float64 or float32; every vector,
scalar and product is float64. Convergence is judged on an explicit FP64 residual ||g - S x|| / ||g||.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import BLS_NOT_CONVERGED, BLS_NOT_PD, ArgumentError, check, dptr, ptr64
from .layout import SchurPattern, SchurStructure
from .reduction import _dev, _dtype_code, context


class BlockJacobi:
    """The block layout of a flat array of square diagonal blocks (dims[b] x dims[b], column-major, in order)."""

    def __init__(self, dims, *, device: int = 0):
        self.dims = np.ascontiguousarray(dims, np.int64)
        self.device = device
        self.length = int((self.dims ** 2).sum())
        self.n = int(self.dims.sum())
        h = C.c_void_p()
        check(_lib.gpu().bls_block_jacobi_create(context(device), len(self.dims), ptr64(self.dims), C.byref(h)))
        self._h = h
        self.failed_block = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_block_jacobi_destroy(h)
            self._h = None

    @property
    def handle(self):
        context(self.device)
        return self._h


def factor_diagonal_blocks(D: torch.Tensor, bj: BlockJacobi) -> bool:
    """Each block's Cholesky factor in place in its lower triangle (src/diagonal_blocks.jl:6-29). False if a block is
    not positive definite or not finite (bj.failed_block: the lowest, 1-based)."""
    T = _dtype_code(_dev(D, "D", bj.length))
    fb = C.c_int64(0)
    rc = check(_lib.gpu().bls_factor_diagonal_blocks(bj.handle, T, dptr(D), C.byref(fb)))
    bj.failed_block = int(fb.value)
    return rc != BLS_NOT_PD


def solve_diagonal_blocks(y: torch.Tensor, D: torch.Tensor, bj: BlockJacobi, x: torch.Tensor) -> torch.Tensor:
    """y = (L L')^-1 x block by block, with D factored (src/diagonal_blocks.jl:31-61); y may be x."""
    T = _dtype_code(_dev(D, "D", bj.length))
    _dev(x, "x", bj.n, torch.float64)
    _dev(y, "y", bj.n, torch.float64)
    check(_lib.gpu().bls_solve_diagonal_blocks(bj.handle, T, dptr(y), dptr(D), dptr(x)))
    return y


@dataclass
class PCGResult:
    converged: bool
    iterations: int
    rel_residual: float      # ||g - S x|| / ||g||, FP64, of the returned x
    failed_block: int = 0    # with converged False and iterations 0: a diagonal block of S that is not PD (1-based)


@dataclass
class RefinedResult:
    converged: bool
    corrections: int         # outer corrections (PCG solves on the stored S)
    iterations: int          # PCG iterations over all corrections
    rel_residual: float      # ||g - A x|| / ||g|| with A the FP64 reduced operator
    failed_block: int = 0


class PCGWorkspace:
    """The device plan of PCG on the reduced system of `structure` on `pattern`: per-row block lists for y = S x, the
    block-Jacobi factorisation and the solver's vectors."""

    def __init__(self, structure: SchurStructure, pattern: SchurPattern, *, device: int = 0):
        self.structure, self.pattern, self.device = structure, pattern, device
        st = structure
        keep = [np.ascontiguousarray(a, np.int64) for a in (st.r_dims, pattern.block_colptr, pattern.block_rowval,
                                                            pattern.block_row_offsets, pattern.col_heights, pattern.S_colptr)]
        h = C.c_void_p()
        check(_lib.gpu().bls_pcg_plan_create(context(device), st.nrblocks, *[ptr64(a) for a in keep], C.byref(h)))
        self._h = h
        self.ndiag = int((np.asarray(st.r_dims, np.int64) ** 2).sum())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_pcg_plan_destroy(h)
            self._h = None

    @property
    def handle(self):
        context(self.device)
        return self._h

    def _S(self, S):
        return _dtype_code(_dev(S, "S.nzval", self.pattern.nnz))

    def spmv(self, S: torch.Tensor, x: torch.Tensor, y: torch.Tensor | None = None) -> torch.Tensor:
        """y = S x, S symmetric from its upper blocks (FP64 products)."""
        T = self._S(S)
        nr = self.structure.nr
        _dev(x, "x", nr, torch.float64)
        if y is None:
            y = torch.empty(nr, dtype=torch.float64, device=x.device)
        _dev(y, "y", nr, torch.float64)
        check(_lib.gpu().bls_spmv_sym(self.handle, T, dptr(S), dptr(x), dptr(y)))
        return y

    def diagonal_blocks(self, S: torch.Tensor) -> torch.Tensor:
        """The full diagonal blocks of S (upper triangles mirrored), float64, block after block."""
        T = self._S(S)
        D = torch.empty(self.ndiag, dtype=torch.float64, device=S.device)
        check(_lib.gpu().bls_extract_diagonal_blocks(self.handle, T, dptr(S), dptr(D)))
        return D

    def launches(self) -> int:
        return int(_lib.gpu().bls_pcg_plan_counters(self._h))

    def solve(self, S: torch.Tensor, g: torch.Tensor, x: torch.Tensor | None = None, *, tol: float = 1e-8, maxit: int | None = None,
              graph: bool = True, preconditioner: torch.Tensor | None = None) -> tuple[torch.Tensor, PCGResult]:
        """PCG from x (zero when None) to ||g - S x|| <= tol ||g|| on an explicit FP64 residual, preconditioned by
        block-Jacobi or, when given, by the dense SPD blocks `preconditioner` (float64, d x d per block, as
        LearnedPreconditioner.blocks returns them). x is updated in place and returned with the run's PCGResult."""
        if preconditioner is not None:
            _dev(preconditioner, "preconditioner", self.ndiag, torch.float64)
        check(_lib.gpu().bls_pcg_set_preconditioner(self.handle, dptr(preconditioner)))
        try:
            return self._solve(S, g, x, tol=tol, maxit=maxit, graph=graph)
        finally:
            _lib.gpu().bls_pcg_set_preconditioner(self._h, None)

    def _solve(self, S, g, x, *, tol, maxit, graph):
        T = self._S(S)
        nr = self.structure.nr
        _dev(g, "g", nr, torch.float64)
        if x is None:
            x = torch.zeros(nr, dtype=torch.float64, device=g.device)
        _dev(x, "x", nr, torch.float64)
        if maxit is None:
            maxit = 10 * nr
        it, rel, fb = C.c_int64(0), C.c_double(0.0), C.c_int64(0)
        rc = check(_lib.gpu().bls_pcg_solve(self.handle, T, dptr(S), dptr(g), dptr(x), float(tol), int(maxit), int(graph), C.byref(it),
                                            C.byref(rel), C.byref(fb)))
        return x, PCGResult(rc == 0, int(it.value), float(rel.value), int(fb.value))

    def solve_refined(self, S: torch.Tensor, S0: torch.Tensor, scaling_r: torch.Tensor, lam: float, C_data: torch.Tensor,
                      g: torch.Tensor, schur_ws, x: torch.Tensor | None = None, *, tol: float = 1e-12, inner_tol: float = 1e-6,
                      max_outer: int = 20, inner_maxit: int | None = None) -> tuple[torch.Tensor, RefinedResult]:
        """Solve A x = g, A = S0 + lam diag(scaling_r) - C' E^-1 C in FP64 (the reduced operator of `schur_ws`'s last
        reduction, applied from its stored blocks), by PCG corrections on the stored S (e.g. the FP32 reduction) until
        ||g - A x|| <= tol ||g||. S0 is R on S's pattern (a reset with lam = 0)."""
        T = self._S(S)
        if S0.dtype != S.dtype:
            raise ArgumentError("S0 must have S's dtype")
        self._S(S0)
        st = self.structure
        nr = st.nr
        _dev(g, "g", nr, torch.float64)
        _dev(scaling_r, "scaling_r", nr, torch.float64)
        _dev(C_data, "C_data", st.C_length, S.dtype)
        if x is None:
            x = torch.zeros(nr, dtype=torch.float64, device=g.device)
        _dev(x, "x", nr, torch.float64)
        if inner_maxit is None:
            inner_maxit = 10 * nr
        o, i, rel, fb = C.c_int64(0), C.c_int64(0), C.c_double(0.0), C.c_int64(0)
        rc = check(_lib.gpu().bls_pcg_solve_refined(self.handle, schur_ws.handle, T, dptr(S), dptr(S0), dptr(scaling_r), float(lam),
                                                    dptr(C_data), dptr(g), dptr(x), float(tol), float(inner_tol), int(max_outer),
                                                    int(inner_maxit), C.byref(o), C.byref(i), C.byref(rel), C.byref(fb)))
        return x, RefinedResult(rc == 0, int(o.value), int(i.value), float(rel.value), int(fb.value))
