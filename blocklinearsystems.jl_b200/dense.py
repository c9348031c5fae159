"""Dense reduced solve on the device: the Cholesky factorisation S = L L' of a dense reduced system (the output of
reduce_schur_dense!) and the solve x = S^-1 g, in FP64 whatever S's storage type. The reference hands its dense S to
DampedLinearSolve's Cholesky (src/schur_linear_systems.jl:312-320)."""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import BLS_NOT_PD, ArgumentError, check, dptr
from .reduction import _dev, _dtype_code, context


class DenseCholesky:
    """The device solver of an n x n dense reduced system (n <= 16384). failed_column: the column (1-based) whose pivot
    was not positive in the last factor(), 0 when it succeeded."""

    def __init__(self, n: int, *, device: int = 0):
        self.n, self.device = int(n), device
        h = C.c_void_p()
        check(_lib.gpu().bls_dense_solver_create(context(device), self.n, C.byref(h)))
        self._h = h
        self.failed_column = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_dense_solver_destroy(h)
            self._h = None

    @property
    def handle(self):
        context(self.device)
        return self._h

    def factor(self, S: torch.Tensor, lam: float | None = None, s_r: torch.Tensor | None = None) -> bool:
        """Factor S (column-major n x n, float64 or float32, its upper triangle read), or S + lam diag(s_r) when s_r is
        given (the QR route's damped reduced normal equations, src/qr_linear_systems.jl:315-322). False: not positive
        definite."""
        T = _dtype_code(_dev(S, "S", self.n * self.n))
        fc = C.c_int64(0)
        if s_r is None:
            rc = check(_lib.gpu().bls_dense_cholesky(self.handle, T, dptr(S), C.byref(fc)))
        else:
            _dev(s_r, "s_r", self.n, torch.float64)
            rc = check(_lib.gpu().bls_dense_cholesky_shifted(self.handle, T, dptr(S), float(0.0 if lam is None else lam), dptr(s_r),
                                                             C.byref(fc)))
        self.failed_column = int(fc.value)
        return rc != BLS_NOT_PD

    def solve(self, g: torch.Tensor, x: torch.Tensor | None = None) -> torch.Tensor:
        """x = S^-1 g from the last successful factor()."""
        _dev(g, "g", self.n, torch.float64)
        if x is None:
            x = torch.empty_like(g)
        _dev(x, "x", self.n, torch.float64)
        check(_lib.gpu().bls_dense_cholesky_solve(self.handle, dptr(g), dptr(x)))
        return x
