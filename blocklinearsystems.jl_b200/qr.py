"""QR elimination on the device, mirroring the reference's Jacobian-path API (0-based layout, torch CUDA tensors).

SchurJacobianStructure    src/schur_jacobian.jl:30-160, src/schur_description.jl:137-189 (layout built natively)
SchurBlockJacobian        src/schur_jacobian.jl:194-208 (raw tables `data` in T, residual `r` in float64)
QRReductionWorkspace      src/qr_reduction.jl:11-24 (here: the device plan plus the factored tables)
reduce_qr                 src/qr_reduction.jl:162-187 -> bool
qr_backsubstitute         src/qr_reduced.jl:97-110 (the reference's backsubstitute!(x_e, x_r, ws))
reduced_normal_sparse     src/qr_reduced.jl:438-480
reduced_normal_dense      src/qr_reduced.jl:407-436
reduced_diagonal_blocks   src/qr_reduced.jl:482-512
free_block_pairs          src/qr_reduced.jl:5-16
reduced_nrows             src/qr_reduced.jl:1-3
reduced_residual          src/qr_reduced.jl:227-243
reduced_mul / reduced_tmul  src/qr_reduced.jl:159-223 (J~ v and J~' w from the factored tables)
reduced_jacobian          src/qr_reduced.jl:245-272 (dense) and 336-370 (sparse: reduced_jacobian_sparse)
build_reduced_jacobian_pattern  src/qr_reduced.jl:284-310

Element type T is the dtype of the Jacobian's tables: torch.float64, or torch.float32 (the mixed form: FP32 tables with
FP64 column norms, reflector scalars and reflector application, rounded once per entry; the residual is FP64 in both).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import BLS_NOT_CONVERGED, BLS_NOT_PD, ArgumentError, DimensionMismatch, check, dptr, ptr64
from .layout import DEFAULT_MIN_WORK, SchurPattern, SchurStructure, _csr
from .reduction import _dev, _dtype_code, context


class SchurJacobianStructure:
    """The layout of a QR elimination: one table per eliminated block, then one per free group (0-based fields).

    SchurJacobianStructure(blocksizes, rowblocks, rowblocksizes, eliminated=...) lays out a description in the caller's
    numbering; SchurJacobianStructure.positional(structure, e_rows, free_rows, free_retained) is the positional form.
    """

    _FIELDS = ("e_rows", "free_rows", "table_nrows", "table_ncols", "table_top", "table_offsets", "raw_offsets",
               "residual_offsets", "reduced_offsets", "table_ptr", "entry_retained", "entry_col", "entry_table", "retained_ptr",
               "retained_entry", "doffsets", "col_chunks", "row_table", "row_first", "row_nrows", "row_ptr", "row_blocks")
    _SCALARS = ("ntables", "raw_length", "residual_length")

    def __init__(self, blocksizes=None, rowblocks=None, rowblocksizes=None, *, eliminated=None, nchunks: int = 1,
                 min_work: int = DEFAULT_MIN_WORK, _handle=None):
        L = _lib.gpu()
        if _handle is None:
            if eliminated is None:
                raise TypeError("eliminated is required")
            bs = np.ascontiguousarray(blocksizes, np.int64)
            el = np.ascontiguousarray(np.asarray(eliminated, bool), np.uint8)
            if len(el) != len(bs):
                raise DimensionMismatch(f"eliminated has length {len(el)}, but there are {len(bs)} column blocks")
            ptr, idx = _csr(rowblocks)
            rbs = np.ascontiguousarray(rowblocksizes, np.int64)
            if len(rbs) != len(ptr) - 1:
                raise DimensionMismatch(f"rowblocksizes has length {len(rbs)}, but there are {len(ptr) - 1} row blocks")
            h = C.c_void_p()
            check(L.bls_qr_structure_from_description(len(bs), ptr64(bs), len(ptr) - 1, ptr64(ptr), ptr64(idx), ptr64(rbs),
                                                      el.ctypes.data_as(C.POINTER(C.c_uint8)), int(nchunks), int(min_work),
                                                      C.byref(h)))
            _handle = h
        self._h = _handle
        for f in self._SCALARS:
            setattr(self, f, int(self._field(f)[0]))
        for f in self._FIELDS:
            setattr(self, f, self._field(f))
        sh = C.c_void_p()
        check(L.bls_qr_structure_schur(self._h, C.byref(sh)))
        self.schur = SchurStructure(_handle=sh)

    @classmethod
    def positional(cls, structure: SchurStructure, e_rows, free_rows=(), free_retained=(), *, nchunks: int = 1):
        er = np.ascontiguousarray(e_rows, np.int64)
        fr = np.ascontiguousarray(free_rows, np.int64)
        if len(er) != structure.neblocks:
            raise DimensionMismatch(f"Number of eliminated row counts ({len(er)}) must match the number of eliminated blocks "
                                    f"({structure.neblocks})")
        if len(free_retained) != len(fr):
            raise DimensionMismatch("Number of free groups' retained lists must match the number of free row counts")
        ptr, idx = _csr([list(x) for x in free_retained])
        h = C.c_void_p()
        check(_lib.gpu().bls_qr_structure_positional(structure.handle, ptr64(er), len(fr), ptr64(fr), ptr64(ptr), ptr64(idx),
                                                     int(nchunks), C.byref(h)))
        return cls(_handle=h)

    def _field(self, name: str) -> np.ndarray:
        L = _lib.gpu()
        n = L.bls_qr_structure_field(self._h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, np.int64)
        if n:
            L.bls_qr_structure_field(self._h, name.encode(), ptr64(out))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_qr_structure_destroy(h)
            self._h = None

    # accessors (src/schur_description.jl:199-214)
    def blockorder(self) -> np.ndarray:
        return self.schur.blockorder()

    def nretained(self) -> int:
        return self.schur.nrblocks

    def nblocks(self) -> int:
        return self.schur.nrblocks + self.schur.neblocks

    @property
    def handle(self):
        return self._h


def free_block_pairs(jst: SchurJacobianStructure) -> list[tuple[int, int]]:
    """Pairs of retained blocks coupled through a free group (src/qr_reduced.jl:5-16), in the reference's order."""
    pairs: list[tuple[int, int]] = []
    seen = set()
    for t in range(jst.schur.neblocks, jst.ntables):
        lo, hi = int(jst.table_ptr[t]), int(jst.table_ptr[t + 1])
        for u2 in range(lo, hi):
            for u1 in range(lo, u2):
                p = (int(jst.entry_retained[u1]), int(jst.entry_retained[u2]))
                if p not in seen:
                    seen.add(p)
                    pairs.append(p)
    return pairs


def reduced_nrows(jst: SchurJacobianStructure) -> int:
    """Rows of the reduced Jacobian J~ (src/qr_reduced.jl:1-3)."""
    return int(jst.reduced_offsets[-1])


class SchurBlockJacobian:
    """The raw tables (`data`, T, length raw_length) and the residual (`r`, float64, length residual_length) on the
    device, zero-initialised as SchurBlockJacobian(structure, T) (src/schur_jacobian.jl:194-208)."""

    def __init__(self, structure: SchurJacobianStructure, dtype=torch.float64, device: int = 0, data=None, r=None):
        self.structure = structure
        dev = torch.device("cuda", device)
        self.data = torch.zeros(structure.raw_length, dtype=dtype, device=dev) if data is None else data
        self.r = torch.zeros(structure.residual_length, dtype=torch.float64, device=dev) if r is None else r
        _dev(self.data, "J.data", structure.raw_length)
        _dev(self.r, "J.r", structure.residual_length, torch.float64)


class QRReductionWorkspace:
    """The device plan of a QR elimination plus its factored tables (`factored`, T) and factored residual (`fres`,
    float64). `pattern` (build_schur_pattern(structure.schur, extra_blocks=free_block_pairs(structure))) is needed for
    reduced_normal_sparse. `failed_block`: the lowest failing eliminated block of the last reduce_qr, 1-based, 0 none."""

    def __init__(self, structure: SchurJacobianStructure, pattern: SchurPattern | None = None, dtype=torch.float64,
                 *, device: int = 0):
        self.structure, self.pattern, self.device, self.dtype = structure, pattern, device, dtype
        ctx = context(device)
        st = structure.schur
        keep = []

        def arr(a):
            a = np.ascontiguousarray(a, np.int64)
            keep.append(a)
            return ptr64(a)

        d = _lib.bls_qr_plan_desc()
        d.nrblocks, d.neblocks, d.ntables = st.nrblocks, st.neblocks, structure.ntables
        d.r_dims, d.e_dims = arr(st.r_dims), arr(st.e_dims)
        d.table_nrows, d.table_ncols, d.table_top = arr(structure.table_nrows), arr(structure.table_ncols), arr(structure.table_top)
        d.table_ptr, d.entry_retained, d.entry_col = arr(structure.table_ptr), arr(structure.entry_retained), arr(structure.entry_col)
        d.raw_offsets, d.residual_offsets = arr(structure.raw_offsets), arr(structure.residual_offsets)
        if pattern is not None:
            d.block_colptr, d.block_rowval = arr(pattern.block_colptr), arr(pattern.block_rowval)
            d.block_row_offsets, d.col_heights, d.S_colptr = arr(pattern.block_row_offsets), arr(pattern.col_heights), arr(pattern.S_colptr)
        h = C.c_void_p()
        check(_lib.gpu().bls_qr_plan_create(ctx, C.byref(d), C.byref(h)))
        self._h = h
        dev = torch.device("cuda", device)
        self.factored = torch.zeros(structure.raw_length, dtype=dtype, device=dev)
        self.fres = torch.zeros(structure.residual_length, dtype=torch.float64, device=dev)
        self.failed_block = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_qr_plan_destroy(h)
            self._h = None

    @property
    def handle(self):
        context(self.device)
        return self._h

    @property
    def _T(self) -> int:
        return _dtype_code(self.factored)

    def query_status(self) -> bool:
        """Verdict of the last reduce_qr (synchronises); sets failed_block."""
        fb = C.c_int64(0)
        rc = check(_lib.gpu().bls_qr_query_status(self.handle, C.byref(fb)))
        self.failed_block = int(fb.value)
        return rc != BLS_NOT_PD

    def launches(self) -> int:
        """Device kernel launches since the last call."""
        return int(_lib.gpu().bls_qr_plan_counters(self._h))

    def set_staging(self, bulk: bool) -> None:
        """Stage each table into shared memory with one bulk (TMA) copy per contiguous span (True, the default) or with
        element-wise asynchronous copies (False); the results are the same."""
        check(_lib.gpu().bls_qr_plan_set_staging(self._h, int(bulk)))


def reduce_qr(ws: QRReductionWorkspace, J: SchurBlockJacobian, scaling_e: torch.Tensor, lam: float, s: torch.Tensor | None = None,
              *, sync: bool = True) -> bool:
    """QR elimination of every eliminated block (src/qr_reduction.jl:162-187); conditioned by `s` (over all the
    variables, [s_r; s_e]) when given. False: a non-finite table or a numerically singular U (ws.failed_block).
    sync=False launches without waiting for the verdict (read it with ws.query_status())."""
    jst = ws.structure
    if J.structure is not jst:
        raise ArgumentError("The Jacobian and the workspace were built for different structures")
    if J.data.dtype != ws.dtype:
        raise ArgumentError(f"the Jacobian is {J.data.dtype}, the workspace {ws.dtype}")
    st = jst.schur
    _dev(scaling_e, "scaling_e", st.ne, torch.float64)
    if s is not None:
        _dev(s, "s", st.nr + st.ne, torch.float64)
    fb = C.c_int64(0)
    rc = check(_lib.gpu().bls_reduce_qr(ws.handle, ws._T, dptr(ws.factored), dptr(ws.fres), dptr(J.data), dptr(J.r), dptr(scaling_e),
                                        float(lam), dptr(s), C.byref(fb) if sync else None))
    if not sync:
        return True
    ws.failed_block = int(fb.value)
    return rc != BLS_NOT_PD


def qr_backsubstitute(x_e: torch.Tensor, x_r: torch.Tensor, ws: QRReductionWorkspace) -> None:
    """x_e = U^-1 (q - B x_r) per eliminated block, in float64 (src/qr_reduced.jl:24-110)."""
    st = ws.structure.schur
    _dev(x_e, "x_e", st.ne, torch.float64)
    _dev(x_r, "x_r", st.nr, torch.float64)
    check(_lib.gpu().bls_qr_backsubstitute(ws.handle, ws._T, dptr(x_e), dptr(x_r), dptr(ws.factored), dptr(ws.fres)))


def reduced_normal_dense(S: torch.Tensor, g_S: torch.Tensor, ws: QRReductionWorkspace) -> bool:
    """Overwrite the upper triangle of the column-major nr x nr S with J~'J~ and g_S with J~'r~ (src/qr_reduced.jl:407-436)."""
    nr = ws.structure.schur.nr
    if S.dtype != ws.dtype:
        raise ArgumentError(f"S must be {ws.dtype}")
    _dev(S, "S", nr * nr)
    _dev(g_S, "g_S", nr, torch.float64)
    check(_lib.gpu().bls_reduced_normal_dense(ws.handle, ws._T, dptr(S), dptr(g_S), dptr(ws.factored), dptr(ws.fres)))
    return True


def reduced_normal_sparse(S_nzval: torch.Tensor, g_S: torch.Tensor, ws: QRReductionWorkspace, pattern: SchurPattern | None = None) -> bool:
    """Sparse counterpart of reduced_normal_dense into S.nzval on the workspace's pattern (src/qr_reduced.jl:438-480)."""
    pat = ws.pattern
    if pat is None:
        raise ArgumentError("the workspace was built without a sparse pattern")
    if pattern is not None and pattern is not pat and len(pattern.S_rowval) != len(pat.S_rowval):
        raise DimensionMismatch("the pattern does not match the workspace's")
    if S_nzval.dtype != ws.dtype:
        raise ArgumentError(f"S must be {ws.dtype}")
    _dev(S_nzval, "S.nzval", pat.nnz)
    _dev(g_S, "g_S", ws.structure.schur.nr, torch.float64)
    check(_lib.gpu().bls_reduced_normal_sparse(ws.handle, ws._T, dptr(S_nzval), dptr(g_S), dptr(ws.factored), dptr(ws.fres)))
    return True


def reduced_diagonal_blocks(D: torch.Tensor, ws: QRReductionWorkspace) -> torch.Tensor:
    """The full d_r x d_r diagonal blocks of J~'J~, at doffsets (src/qr_reduced.jl:482-512)."""
    if D.dtype != ws.dtype:
        raise ArgumentError(f"D must be {ws.dtype}")
    _dev(D, "D", int(ws.structure.doffsets[-1]))
    check(_lib.gpu().bls_reduced_diagonal_blocks(ws.handle, ws._T, dptr(D), dptr(ws.factored)))
    return D


def assemble_hessian(J: SchurBlockJacobian, ws: QRReductionWorkspace, *, dense: bool = False):
    """H = J'J and b = J'r of the raw Jacobian J in the SchurBlockHessian layout of the same structure, on the device:
    (E_data, C_data, R, b) with R the retained blocks on the reduced pattern (dense: column-major nr x nr), upper
    triangle, and b = [b_r; b_e] in float64. What a caller fills with addblock! from its Jacobian (the reference's
    fixtures form it as J64'J64, test/fixtures/QRFixtures.jl:109-120). R resets a SchurReductionWorkspace built with
    r_to_s_map = identity (sparse) like any R on the pattern."""
    jst = J.structure
    st = jst.schur
    if J.data.dtype != ws.dtype:
        raise ArgumentError(f"J must be {ws.dtype}")
    if not dense and ws.pattern is None:
        raise ArgumentError("the workspace was built without a sparse pattern")
    dev = J.data.device
    E = torch.empty(st.E_length, dtype=ws.dtype, device=dev)
    Cd = torch.empty(st.C_length, dtype=ws.dtype, device=dev)
    R = torch.empty(st.nr * st.nr if dense else ws.pattern.nnz, dtype=ws.dtype, device=dev)
    b = torch.empty(st.nr + st.ne, dtype=torch.float64, device=dev)
    check(_lib.gpu().bls_assemble_hessian(ws.handle, ws._T, dptr(J.data), dptr(J.r), dptr(E), dptr(Cd), dptr(R), int(dense), dptr(b)))
    return E, Cd, R, b


def _tables(src, ws):
    """(plan, tables, residual, dtype code) of a SchurBlockJacobian (raw tables, with the workspace `ws` that holds the
    plan) or of a QRReductionWorkspace (its factored tables)."""
    if isinstance(src, QRReductionWorkspace):
        return src, src.factored, src.fres
    if ws is None:
        raise ArgumentError("a SchurBlockJacobian needs the QRReductionWorkspace of its structure")
    if src.data.dtype != ws.dtype:
        raise ArgumentError(f"J must be {ws.dtype}")
    return ws, src.data, src.r


def jtr(g: torch.Tensor, src, ws: QRReductionWorkspace | None = None) -> torch.Tensor:
    """jtr!(g, src) (src/qr_reduced.jl:575-584): the gradient g = J'r = [g_r; g_e] of the full problem, from the raw
    tables of a SchurBlockJacobian or the factored tables of a QRReductionWorkspace (every row, FP64 sums)."""
    w, D, Rv = _tables(src, ws)
    st = w.structure.schur
    _dev(g, "g", st.nr + st.ne, torch.float64)
    check(_lib.gpu().bls_jtr(w.handle, w._T, dptr(g), dptr(D), dptr(Rv)))
    return g


def jtj_diag(d: torch.Tensor, src, ws: QRReductionWorkspace | None = None) -> torch.Tensor:
    """jtj_diag!(d, src) (src/qr_reduced.jl:586-595): the squared column norms of J, diag(J'J) = [d_r; d_e], FP64."""
    w, D, _ = _tables(src, ws)
    st = w.structure.schur
    _dev(d, "d", st.nr + st.ne, torch.float64)
    check(_lib.gpu().bls_jtj_diag(w.handle, w._T, dptr(d), dptr(D)))
    return d


def jtj_quadform(src, v: torch.Tensor, ws: QRReductionWorkspace | None = None) -> float:
    """jtj_quadform(src, v) (src/qr_reduced.jl:597-640): ||J v||^2 = v'(J'J)v for v = [v_r; v_e], FP64."""
    w, D, _ = _tables(src, ws)
    st = w.structure.schur
    _dev(v, "v", st.nr + st.ne, torch.float64)
    out = C.c_double(0.0)
    check(_lib.gpu().bls_jtj_quadform(w.handle, w._T, dptr(D), dptr(v), C.byref(out)))
    return float(out.value)


def build_reduced_jacobian_pattern(jst: SchurJacobianStructure):
    """build_reduced_jacobian_pattern(jst) (src/qr_reduced.jl:284-310): the CSC pattern of J~ (reduced_nrows x nr),
    0-based (colptr, rowval) on the host."""
    L = _lib.gpu()
    n = L.bls_reduced_jacobian_pattern(jst.handle, None, None)
    check(int(n) if n < 0 else 0)
    colptr = np.empty(jst.schur.nr + 1, np.int64)
    rowval = np.empty(n, np.int64)
    L.bls_reduced_jacobian_pattern(jst.handle, ptr64(colptr), ptr64(rowval))
    return colptr, rowval


def reduced_residual(rt: torch.Tensor, ws: QRReductionWorkspace) -> torch.Tensor:
    """reduced_residual!(rt, ws) (src/qr_reduced.jl:227-243): rt = r~ (float64, reduced_nrows entries)."""
    _dev(rt, "rt", None, torch.float64)
    check(_lib.gpu().bls_reduced_residual(ws.handle, dptr(ws.fres), dptr(rt) if rt.numel() else None, rt.numel()))
    return rt


def reduced_jacobian(Jt: torch.Tensor, rt: torch.Tensor, ws: QRReductionWorkspace) -> torch.Tensor:
    """reduced_jacobian!(Jt::Matrix, rt, ws) (src/qr_reduced.jl:245-272): Jt = J~ column-major (reduced_nrows x nr, a
    flat tensor of the workspace's dtype, or the transposed view of an (nr, reduced_nrows) tensor) and rt = r~."""
    if Jt.dtype != ws.dtype:
        raise ArgumentError(f"Jt must be {ws.dtype}")
    _dev(rt, "rt", None, torch.float64)
    m, nr = reduced_nrows(ws.structure), ws.structure.schur.nr
    if Jt.dim() == 2:
        rows, cols = Jt.shape
        if not Jt.t().is_contiguous():
            raise ArgumentError("a 2-d Jt must be column-major (the transpose of a contiguous tensor)")
    else:
        _dev(Jt, "Jt")
        rows, cols = (m, nr) if Jt.numel() == m * nr else (Jt.numel(), 1)
    check(_lib.gpu().bls_reduced_jacobian_dense(ws.handle, ws._T, dptr(ws.factored), dptr(ws.fres), dptr(Jt) if Jt.numel() else None,
                                                rows, cols, dptr(rt) if rt.numel() else None, rt.numel()))
    return Jt


def reduced_jacobian_sparse(nzval: torch.Tensor, colptr, rowval, rt: torch.Tensor, ws: QRReductionWorkspace,
                            nrows: int | None = None, ncols: int | None = None) -> torch.Tensor:
    """reduced_jacobian!(Jt::SparseMatrixCSC, rt, ws) (src/qr_reduced.jl:336-370): nzval (device, the workspace's
    dtype) of J~ on the CSC pattern (colptr, rowval: 0-based host arrays, build_reduced_jacobian_pattern's), and
    rt = r~. The pattern and the sizes are checked before any work (DimensionMismatch, ArgumentError)."""
    if nzval.dtype != ws.dtype:
        raise ArgumentError(f"nzval must be {ws.dtype}")
    _dev(rt, "rt", None, torch.float64)
    cp = np.ascontiguousarray(colptr, np.int64)
    rv = np.ascontiguousarray(rowval, np.int64)
    m = reduced_nrows(ws.structure) if nrows is None else nrows
    n = len(cp) - 1 if ncols is None else ncols
    check(_lib.gpu().bls_reduced_jacobian_sparse(ws.handle, ws._T, dptr(ws.factored), dptr(ws.fres), m, n, ptr64(cp),
                                                 ptr64(rv) if len(rv) else None, dptr(nzval) if nzval.numel() else None,
                                                 dptr(rt) if rt.numel() else None, rt.numel()))
    return nzval


def reduced_mul(y: torch.Tensor, ws: QRReductionWorkspace, v: torch.Tensor) -> torch.Tensor:
    """reduced_mul!(y, ws, v) (src/qr_reduced.jl:159-192): y = J~ v (float64), without forming J~."""
    _dev(y, "y", None, torch.float64)
    _dev(v, "v", None, torch.float64)
    check(_lib.gpu().bls_reduced_mul(ws.handle, ws._T, dptr(ws.factored), dptr(v) if v.numel() else None, v.numel(),
                                     dptr(y) if y.numel() else None, y.numel()))
    return y


def reduced_tmul(g: torch.Tensor, ws: QRReductionWorkspace, w: torch.Tensor) -> torch.Tensor:
    """reduced_tmul!(g, ws, w) (src/qr_reduced.jl:194-223): g = J~' w (float64), without forming J~."""
    _dev(g, "g", None, torch.float64)
    _dev(w, "w", None, torch.float64)
    check(_lib.gpu().bls_reduced_tmul(ws.handle, ws._T, dptr(ws.factored), dptr(w) if w.numel() else None, w.numel(),
                                      dptr(g) if g.numel() else None, g.numel()))
    return g


@dataclass
class LsmrResult:
    """The outcome of lsmr_reduced: `solved` (the reference's Success), the iterations, Fong & Saunders' istop (1, 2, 4,
    5 solved; 3, 6 cond(A) above conlim; 7 itmax) and their estimates for the preconditioned operator."""
    solved: bool
    iterations: int
    istop: int
    normr: float
    normar: float
    normA: float
    condA: float
    normx: float


def lsmr_reduced(x_r: torch.Tensor, ws: QRReductionWorkspace, lam: float, s_r: torch.Tensor | None = None, *,
                 atol: float | None = None, btol: float | None = None, conlim: float | None = None,
                 itmax: int | None = None) -> LsmrResult:
    """The reduced system's LSMR solve (ext/KrylovExt.jl:97-132) on the device: x_r = argmin ||[J~; sqrt(lam s_r)] x -
    [r~; 0]|| from the workspace's factored tables (reduce_qr first), block-Jacobi preconditioned by the diagonal blocks
    of J~'J~ + lam diag(s_r). Tolerances default to the reference's: sqrt(eps(T)) and conlim 1/sqrt(eps(T)) for the
    workspace's storage type T; itmax to reduced_nrows + nr. `solved` is False where the reference returns
    NotPositiveDefinite (a non-finite r~, lam == 0 with fewer reduced rows than retained variables, a diagonal block
    that is not positive definite, cond(A) above conlim, itmax reached)."""
    nr = ws.structure.schur.nr
    _dev(x_r, "x_r", nr, torch.float64)
    if s_r is not None:
        _dev(s_r, "s_r", nr, torch.float64)
    eps = float(np.finfo(np.float32 if ws.dtype == torch.float32 else np.float64).eps)
    tol = np.sqrt(eps)
    it, ist, stats = C.c_int64(0), C.c_int(0), (C.c_double * 5)()
    rc = _lib.gpu().bls_lsmr_reduced(ws.handle, ws._T, dptr(ws.factored), dptr(ws.fres) if ws.fres.numel() else None, float(lam),
                                     dptr(s_r) if s_r is not None and s_r.numel() else None,
                                     dptr(x_r) if x_r.numel() else None, x_r.numel(), tol if atol is None else atol,
                                     tol if btol is None else btol, 1.0 / tol if conlim is None else conlim,
                                     -1 if itmax is None else itmax, C.byref(it), C.byref(ist), stats)
    if rc not in (BLS_NOT_PD, BLS_NOT_CONVERGED):
        check(rc)
    return LsmrResult(rc == 0, int(it.value), int(ist.value), *[float(v) for v in stats])


@dataclass
class RefineResult:
    """Outcome of qr_refine: steps taken (the first is the plain reduced solve), ||d|| / ||J'r|| after each step (d the
    FP64 normal-equation residual of the damped problem), and whether the last one is within the tolerance."""
    steps: int
    rel_residuals: list
    converged: bool


def qr_refine(x: torch.Tensor, ws: QRReductionWorkspace, J: SchurBlockJacobian, scaling_r: torch.Tensor, scaling_e: torch.Tensor,
              lam: float, solve_reduced, *, tol: float = 1e-12, maxit: int = 5) -> RefineResult:
    """Iterative refinement of the QR route (no reference counterpart: the reference solves the reduced system once,
    src/qr_linear_systems.jl:250-300). x = [x_r; x_e] (float64, nr + ne) solves the damped least-squares problem
    min ||J x - r||^2 + lam x' diag([scaling_r; scaling_e]) x of the raw tables J to `tol` in the normal equations:
    each step forms d = J'(r - J x) - lam scaling .* x in FP64 from the raw tables, reduces it through the factored
    tables of the last reduce_qr(ws, J, scaling_e, lam) (U' w = d_e, d_r -= B' w), solves the reduced system with
    `solve_reduced(d_r) -> dx_r` (e.g. DenseCholesky.solve after factor(J~'J~, lam, scaling_r)), back-substitutes
    dx_e = U^-1 (w - B dx_r) and adds dx. The first step from x = 0 is the plain QR-route solve; with FP32 tables the
    following steps recover what FP32 lost, the residual being FP64. Unconditioned tables only (reduce_qr with s = None)."""
    st = ws.structure.schur
    nr, ne = st.nr, st.ne
    if J.data.dtype != ws.dtype:
        raise ArgumentError(f"J must be {ws.dtype}")
    _dev(x, "x", nr + ne, torch.float64)
    _dev(scaling_r, "scaling_r", nr, torch.float64)
    _dev(scaling_e, "scaling_e", ne, torch.float64)
    dev = x.device
    sc = torch.cat([scaling_r, scaling_e])
    y = torch.empty(ws.structure.residual_length, dtype=torch.float64, device=dev)
    d = torch.empty(nr + ne, dtype=torch.float64, device=dev)
    w = torch.empty(max(ne, 1), dtype=torch.float64, device=dev)
    d_r = torch.empty(nr, dtype=torch.float64, device=dev)
    dx_e = torch.empty(max(ne, 1), dtype=torch.float64, device=dev)
    L = _lib.gpu()
    h, T = ws.handle, ws._T
    x.zero_()
    rels = []
    bnorm = None
    for k in range(maxit + 1):
        check(L.bls_qr_normal_residual(h, T, dptr(J.data), dptr(J.r), dptr(sc), float(lam), dptr(x), dptr(y), dptr(d)))
        dn = float(torch.linalg.vector_norm(d))
        if bnorm is None:
            bnorm = max(dn, 1e-300)     # x = 0: d = J'r
        else:
            rels.append(dn / bnorm)
            if rels[-1] <= tol or k == maxit:
                break
        check(L.bls_qr_reduce_rhs(h, T, dptr(ws.factored), dptr(d), dptr(w), dptr(d_r)))
        dx_r = solve_reduced(d_r)
        check(L.bls_qr_backsubstitute_rhs(h, T, dptr(ws.factored), dptr(w), dptr(dx_r), dptr(dx_e)))
        x[:nr] += dx_r
        x[nr:] += dx_e[:ne]
    return RefineResult(len(rels), rels, bool(rels) and rels[-1] <= tol)
