"""ctypes wrapper of the oracle (liboracle.so): a CPU restatement of BlockLinearSystems.jl's elimination path.

Test and baseline infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it as the checker
or the timed CPU reference. The product never imports it. Integers are 0-based at this boundary.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_L = None
i64, p64, vp, pd = C.c_int64, C.POINTER(C.c_int64), C.c_void_p, C.POINTER(C.c_double)
pf = C.POINTER(C.c_float)
pu8 = C.POINTER(C.c_uint8)


class OracleError(Exception):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return HERE / "liboracle.so"


def lib() -> C.CDLL:
    global _L
    if _L is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        L.orc_last_error.restype = C.c_char_p
        L.orc_structure_field.restype = i64
        L.orc_pattern_field.restype = i64
        L.orc_work_field.restype = i64
        L.orc_qr_field.restype = i64
        L.orc_sparse_indices.restype = i64
        L.orc_reduced_jacobian_pattern.restype = i64
        _L = L
    return _L


def _p(a):
    if a is None:
        return None
    if a.dtype == np.int64:
        return a.ctypes.data_as(p64)
    if a.dtype == np.float64:
        return a.ctypes.data_as(pd)
    if a.dtype == np.float32:
        return a.ctypes.data_as(pf)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(pu8)
    raise TypeError(a.dtype)


def _chk(rc):
    if rc < 0:
        raise OracleError(rc, lib().orc_last_error().decode())
    return rc


def _csr(lists):
    if isinstance(lists, tuple):
        return np.ascontiguousarray(lists[0], np.int64), np.ascontiguousarray(lists[1], np.int64)
    ptr = np.zeros(len(lists) + 1, np.int64)
    ptr[1:] = np.cumsum([len(x) for x in lists])
    idx = np.array([v for x in lists for v in x], np.int64)
    return ptr, idx


class Structure:
    SCALARS = ("nr", "nrblocks", "neblocks", "max_coupled_dim")
    FIELDS = ("r_dims", "e_dims", "boffsets_r", "boffsets_e", "eoffsets", "eliminated_ptr", "entry_retained", "coffsets",
              "order", "retained_pairs", "chunks")

    def __init__(self, h):
        self.h = h
        for f in self.SCALARS:
            setattr(self, f, int(self.field(f)[0]))
        for f in self.FIELDS:
            setattr(self, f, self.field(f))
        self.ne = int(self.e_dims.sum())
        self.E_length = int((self.e_dims ** 2).sum())
        self.C_length = int(sum(self.r_dims[r] * self.e_dims[e] for e in range(self.neblocks)
                                for r in self.entry_retained[self.eliminated_ptr[e]:self.eliminated_ptr[e + 1]]))

    @classmethod
    def from_description(cls, blocksizes, rowblocks, eliminated, nchunks=1, min_work=4096):
        bs = np.ascontiguousarray(blocksizes, np.int64)
        el = np.ascontiguousarray(np.asarray(eliminated, bool), np.uint8)
        ptr, idx = _csr(rowblocks)
        h = vp()
        _chk(lib().orc_structure_from_description(i64(len(bs)), _p(bs), i64(len(ptr) - 1), _p(ptr), _p(idx), _p(el), i64(nchunks),
                                                  i64(min_work), C.byref(h)))
        return cls(h)

    @classmethod
    def positional(cls, r_dims, e_dims, couplings, nchunks=1, min_work=4096):
        rd = np.ascontiguousarray(r_dims, np.int64)
        ed = np.ascontiguousarray(e_dims, np.int64)
        ptr, idx = _csr(couplings)
        h = vp()
        _chk(lib().orc_structure_positional(i64(len(rd)), _p(rd), i64(len(ed)), _p(ed), _p(ptr), _p(idx), i64(nchunks), i64(min_work),
                                            C.byref(h)))
        return cls(h)

    def field(self, name):
        n = lib().orc_structure_field(self.h, name.encode(), None)
        out = np.empty(n, np.int64)
        if n:
            lib().orc_structure_field(self.h, name.encode(), _p(out))
        return out

    def __del__(self):
        if self.h and _L is not None:
            _L.orc_structure_free(self.h)
            self.h = None


class Pattern:
    FIELDS = ("block_colptr", "block_rowval", "block_row_offsets", "col_heights", "S_colptr", "S_rowval", "diag_inds", "R_block_start")

    def __init__(self, st: Structure, extra=()):
        ex = np.ascontiguousarray(np.asarray(list(extra), np.int64).reshape(-1, 2))
        h = vp()
        _chk(lib().orc_schur_pattern(st.h, i64(len(ex)), _p(ex) if len(ex) else None, C.byref(h)))
        self.h = h
        self.st = st
        for f in self.FIELDS:
            n = lib().orc_pattern_field(h, f.encode(), None)
            a = np.empty(n, np.int64)
            if n:
                lib().orc_pattern_field(h, f.encode(), _p(a))
            setattr(self, f, a)
        a = np.empty(1, np.int64)
        lib().orc_pattern_field(h, b"R_length", _p(a))
        self.R_length = int(a[0])
        self.nnz = int(self.S_colptr[-1])

    def r_to_s_map(self):
        out = np.empty(self.R_length, np.int64)
        _chk(lib().orc_r_to_s_map(self.st.h, self.h, _p(out)))
        return out

    def sparse_indices(self, symmetric=False):
        n = lib().orc_sparse_indices(self.st.h, self.h, int(symmetric), None, None, None)
        colptr = np.empty(self.st.nr + 1, np.int64)
        rowval = np.empty(n, np.int64)
        m = np.empty(n, np.int64)
        lib().orc_sparse_indices(self.st.h, self.h, int(symmetric), _p(colptr), _p(rowval), _p(m))
        return colptr, rowval, m

    def __del__(self):
        if getattr(self, "h", None) and _L is not None:
            _L.orc_pattern_free(self.h)
            self.h = None


class Work:
    def __init__(self, st: Structure, nchunks=1, f32=False):
        h = vp()
        _chk(lib().orc_work_new(st.h, i64(nchunks), int(f32), C.byref(h)))
        self.h, self.st, self.f32 = h, st, f32

    def field(self, name):
        n = lib().orc_work_field(self.h, name.encode(), None)
        out = np.empty(n, np.int64)
        if n:
            lib().orc_work_field(self.h, name.encode(), _p(out))
        return out

    def caches(self):
        Einv = np.empty(self.st.E_length, np.float32 if self.f32 else np.float64)
        z = np.empty(self.st.ne)
        lib().orc_work_caches(self.h, Einv.ctypes.data_as(vp), _p(z))
        return Einv, z

    def __del__(self):
        if self.h and _L is not None:
            _L.orc_work_free(self.h)
            self.h = None


def _sfx(a):
    return "f32" if a.dtype == np.float32 else "f64"


def reset_schur_sparse(st, pat, nzval, R, scaling_r, lam, s_r=None):
    f = getattr(lib(), "orc_reset_schur_sparse_" + _sfx(nzval))
    return _chk(f(st.h, pat.h, _p(nzval), _p(R), _p(scaling_r), C.c_double(lam), _p(s_r)))


def reset_schur_dense(st, S, R, scaling_r, lam, s_r=None):
    f = getattr(lib(), "orc_reset_schur_dense_" + _sfx(S))
    return _chk(f(st.h, _p(S), _p(R), _p(scaling_r), C.c_double(lam), _p(s_r)))


def reduce_schur_sparse(st, pat, work, nzval, g, b_r, b_e, scaling_e, lam, E, Cd, s_r=None, s_e=None, nthreads=1):
    fb = C.c_int64(0)
    f = getattr(lib(), "orc_reduce_schur_sparse_" + _sfx(nzval))
    rc = _chk(f(st.h, pat.h, work.h, _p(nzval), _p(g), _p(b_r), _p(b_e), _p(scaling_e), C.c_double(lam), _p(E), _p(Cd), _p(s_r), _p(s_e),
                C.c_int(nthreads), C.byref(fb)))
    return rc == 0, int(fb.value)


def reduce_schur_dense(st, work, S, g, b_r, b_e, scaling_e, lam, E, Cd, s_r=None, s_e=None, nthreads=1):
    fb = C.c_int64(0)
    f = getattr(lib(), "orc_reduce_schur_dense_" + _sfx(S))
    rc = _chk(f(st.h, work.h, _p(S), _p(g), _p(b_r), _p(b_e), _p(scaling_e), C.c_double(lam), _p(E), _p(Cd), _p(s_r), _p(s_e),
                C.c_int(nthreads), C.byref(fb)))
    return rc == 0, int(fb.value)


def backsubstitute(st, work, x_e, x_r, Cd, s_r=None, s_e=None, nthreads=1):
    f = getattr(lib(), "orc_backsubstitute_" + _sfx(Cd))
    return _chk(f(st.h, work.h, _p(x_e), _p(x_r), _p(Cd), _p(s_r), _p(s_e), C.c_int(nthreads)))


def symmetrify_full(blocksizes, it_colptr, it_rowval, it_nzval, data, blocks=None, m=None):
    """symmetrifyfull!(mat, bsm, blocks) (src/SparseBlockLinearSystem.jl:299-341) of the block system given by its
    block sizes and indicestransposed (0-based CSC over block rows; it_nzval = 0-based block starts in data). blocks:
    0-based block list, a boolean mask, or None for all. m: the order of the target (default: the expected one).
    Returns the m x m matrix."""
    bsz = np.ascontiguousarray(blocksizes, np.int64)
    cp, rv, nz = (np.ascontiguousarray(a, np.int64) for a in (it_colptr, it_rowval, it_nzval))
    d = np.ascontiguousarray(data, np.float64)
    if blocks is not None:
        blocks = np.asarray(blocks)
        if blocks.dtype == bool:
            blocks = np.flatnonzero(blocks)
        blocks = np.ascontiguousarray(blocks, np.int64)
    if m is None:
        m = int(bsz.sum()) if blocks is None else int(bsz[blocks[(blocks >= 0) & (blocks < len(bsz))]].sum())
    mat = np.zeros(max(m, 0) * max(m, 0))
    _chk(lib().orc_symmetrify_full(i64(len(bsz)), _p(bsz), _p(cp), _p(rv), _p(nz), _p(d), None if blocks is None else _p(blocks),
                                   i64(0 if blocks is None else len(blocks)), _p(mat), i64(m)))
    return mat.reshape(m, m, order="F")


def retained_block_pairs(it_colptr, it_rowval):
    """retained_block_pairs(R) (src/schur_structure.jl:325-334): off-diagonal stored blocks, 0-based (row, col)."""
    return [(r, int(it_rowval[k])) for r in range(len(it_colptr) - 1) for k in range(int(it_colptr[r]), int(it_colptr[r + 1]))
            if int(it_rowval[k]) != r]


def r_to_s_map_csc(R_colptr, R_rowval, S_colptr, S_rowval):
    """build_r_to_s_map(R_sparse, S_sparse) (src/schur_structure.jl:336-353), 0-based."""
    rc, rr, sc, sr = (np.ascontiguousarray(a, np.int64) for a in (R_colptr, R_rowval, S_colptr, S_rowval))
    out = np.empty(len(rr), np.int64)
    _chk(lib().orc_r_to_s_map_csc(i64(len(rc) - 1), _p(rc), _p(rr), _p(sc), _p(sr), i64(len(sc) - 1), _p(out)))
    return out


def r_to_s_map_blocks_csc(sizes, it_colptr, it_rowval, it_nzval, data_len, S_colptr, S_rowval, boffsets_r):
    """build_r_to_s_map(R_sys, S_sparse, boffsets_r) (src/schur_structure.jl:363-397), 0-based, -1 unmapped."""
    a = [np.ascontiguousarray(x, np.int64) for x in (sizes, it_colptr, it_rowval, it_nzval, S_colptr, S_rowval, boffsets_r)]
    out = np.empty(int(data_len), np.int64)
    _chk(lib().orc_r_to_s_map_blocks_csc(i64(len(a[0])), _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), i64(data_len), _p(a[4]), _p(a[5]),
                                         i64(len(a[4]) - 1), _p(a[6]), _p(out)))
    return out


def sort_schur_blocks(is_elim, sizes, couplings):
    el = np.ascontiguousarray(np.asarray(is_elim, bool), np.uint8)
    sz = np.ascontiguousarray(sizes, np.int64)
    ptr, idx = _csr(couplings)
    out = np.empty(len(sz), np.int64)
    _chk(lib().orc_sort_schur_blocks(i64(len(sz)), _p(el), _p(sz), _p(ptr), _p(idx), _p(out)))
    return out


def expand_block_perm(perm, sizes):
    pm = np.ascontiguousarray(perm, np.int64)
    sz = np.ascontiguousarray(sizes, np.int64)
    out = np.empty(int(sz.sum()), np.int64)
    _chk(lib().orc_expand_block_perm(i64(len(sz)), _p(pm), _p(sz), _p(out)))
    return out


def inv_sym_block(H, damp, generic=False):
    H = np.asfortranarray(H)
    d = H.shape[0]
    inv = np.zeros((d, d), H.dtype, order="F")
    hp = np.ascontiguousarray(H.ravel(order="F"))
    dm = np.ascontiguousarray(damp, H.dtype)
    out = np.zeros(d * d, H.dtype)
    if generic:
        ok = lib().orc_inv_sym_block_generic_f64(C.c_int(d), _p(hp), _p(dm), _p(out))
    else:
        f = lib().orc_inv_sym_block_f32 if H.dtype == np.float32 else lib().orc_inv_sym_block_f64
        ok = f(C.c_int(d), _p(hp), _p(dm), _p(out))
    return bool(ok), out.reshape(d, d, order="F")


def max_threads():
    return lib().orc_max_threads()


class QRStructure:
    """The oracle's SchurJacobianStructure (src/schur_jacobian.jl:59-160), 0-based fields."""

    SCALARS = ("ntables",)
    FIELDS = ("table_nrows", "table_ncols", "table_top", "table_offsets", "raw_offsets", "residual_offsets", "reduced_offsets",
              "table_ptr", "entry_retained", "entry_col", "entry_table", "retained_ptr", "retained_entry", "doffsets", "e_rows",
              "free_rows", "col_chunks")

    def __init__(self, h, st: Structure):
        self.h, self.st = h, st
        for f in self.SCALARS:
            setattr(self, f, int(self.field(f)[0]))
        for f in self.FIELDS:
            setattr(self, f, self.field(f))
        self.raw_length = int(self.raw_offsets[-1])
        self.residual_length = int(self.residual_offsets[-1])

    @classmethod
    def from_description(cls, blocksizes, rowblocks, rowblocksizes, eliminated, nchunks=1, min_work=4096):
        bs = np.ascontiguousarray(blocksizes, np.int64)
        el = np.ascontiguousarray(np.asarray(eliminated, bool), np.uint8)
        rbs = np.ascontiguousarray(rowblocksizes, np.int64)
        ptr, idx = _csr(rowblocks)
        q, s = vp(), vp()
        _chk(lib().orc_qr_structure_from_description(i64(len(bs)), _p(bs), i64(len(rbs)), _p(ptr), _p(idx), _p(rbs), _p(el), i64(nchunks),
                                                     i64(min_work), C.byref(q), C.byref(s)))
        return cls(q, Structure(s))

    @classmethod
    def positional(cls, st: Structure, e_rows, free_rows=(), free_retained=(), nchunks=1):
        er = np.ascontiguousarray(e_rows, np.int64)
        fr = np.ascontiguousarray(free_rows, np.int64)
        ptr, idx = _csr([list(x) for x in free_retained])
        q = vp()
        _chk(lib().orc_qr_structure_positional(st.h, _p(er), i64(len(fr)), _p(fr) if len(fr) else None, _p(ptr) if len(fr) else None,
                                               _p(idx) if len(idx) else None, i64(nchunks), C.byref(q)))
        return cls(q, st)

    def field(self, name):
        n = lib().orc_qr_field(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, np.int64)
        if n:
            lib().orc_qr_field(self.h, name.encode(), _p(out))
        return out

    def __del__(self):
        if self.h and _L is not None:
            _L.orc_qr_free(self.h)
            self.h = None


def reduce_qr(q: QRStructure, F, Fr, Rw, Rr, scaling_e, lam, s=None, nthreads=1):
    """reduce_qr! (src/qr_reduction.jl:162-187) into F / Fr; returns (ok, failed_block 1-based)."""
    fb = C.c_int64(0)
    f = getattr(lib(), "orc_reduce_qr_" + _sfx(F))
    rc = _chk(f(q.h, _p(F), _p(Fr), _p(Rw), _p(Rr), _p(scaling_e), i64(len(scaling_e)), C.c_double(lam), _p(s), C.c_int(nthreads),
                C.byref(fb)))
    return rc == 0, int(fb.value)


def qr_backsubstitute(q: QRStructure, x_e, x_r, F, Fr):
    return _chk(getattr(lib(), "orc_qr_backsubstitute_" + _sfx(F))(q.h, _p(x_e), _p(x_r), _p(F), _p(Fr)))


def reduced_normal_sparse(q: QRStructure, pat: Pattern, nzval, g, F, Fr):
    return _chk(getattr(lib(), "orc_reduced_normal_sparse_" + _sfx(F))(q.h, pat.h, _p(nzval), _p(g), _p(F), _p(Fr)))


def reduced_normal_dense(q: QRStructure, S, g, F, Fr):
    return _chk(getattr(lib(), "orc_reduced_normal_dense_" + _sfx(F))(q.h, _p(S), _p(g), _p(F), _p(Fr)))


def reduced_nrows(q: QRStructure) -> int:
    """reduced_nrows (src/qr_reduced.jl:1-3): rows of the reduced problem."""
    return int(q.reduced_offsets[-1])


def reduced_residual(q: QRStructure, rt, Fr):
    """reduced_residual!(rt, ws) (src/qr_reduced.jl:227-243)."""
    return _chk(lib().orc_reduced_residual(q.h, _p(rt), i64(len(rt)), _p(Fr)))


def reduced_jacobian_pattern(q: QRStructure):
    """build_reduced_jacobian_pattern(jst) (src/qr_reduced.jl:284-310): the CSC pattern of J~, 0-based (colptr, rowval)."""
    n = lib().orc_reduced_jacobian_pattern(q.h, None, None)
    _chk(int(n) if n < 0 else 0)
    colptr = np.empty(q.st.nr + 1, np.int64)
    rowval = np.empty(n, np.int64)
    lib().orc_reduced_jacobian_pattern(q.h, _p(colptr), _p(rowval))
    return colptr, rowval


def reduced_mul(q: QRStructure, y, v, F):
    """reduced_mul!(y, ws, v) (src/qr_reduced.jl:159-192): y = J~ v."""
    return _chk(getattr(lib(), "orc_reduced_mul_" + _sfx(F))(q.h, _p(y), i64(len(y)), _p(v), i64(len(v)), _p(F)))


def reduced_tmul(q: QRStructure, g, w, F):
    """reduced_tmul!(g, ws, w) (src/qr_reduced.jl:194-223): g = J~' w."""
    return _chk(getattr(lib(), "orc_reduced_tmul_" + _sfx(F))(q.h, _p(g), i64(len(g)), _p(w), i64(len(w)), _p(F)))


def reduced_jacobian_dense(q: QRStructure, Jt, nrows, ncols, rt, F, Fr):
    """reduced_jacobian!(Jt::Matrix, rt, ws) (src/qr_reduced.jl:245-272): Jt column-major nrows x ncols, flat."""
    return _chk(getattr(lib(), "orc_reduced_jacobian_dense_" + _sfx(F))(q.h, _p(Jt), i64(nrows), i64(ncols), _p(rt), i64(len(rt)), _p(F),
                                                                          _p(Fr)))


def reduced_jacobian_sparse(q: QRStructure, nrows, ncols, colptr, rowval, nzval, rt, F, Fr):
    """reduced_jacobian!(Jt::SparseMatrixCSC, rt, ws) (src/qr_reduced.jl:336-370) on a 0-based CSC pattern."""
    cp = np.ascontiguousarray(colptr, np.int64)
    rv = np.ascontiguousarray(rowval, np.int64)
    return _chk(getattr(lib(), "orc_reduced_jacobian_sparse_" + _sfx(F))(q.h, i64(nrows), i64(ncols), _p(cp), _p(rv), _p(nzval), _p(rt),
                                                                           i64(len(rt)), _p(F), _p(Fr)))


def reduced_diagonal_blocks(q: QRStructure, D, F):
    return _chk(getattr(lib(), "orc_reduced_diagonal_blocks_" + _sfx(F))(q.h, _p(D), _p(F)))


def factor_diagonal_blocks(D, dims):
    dm = np.ascontiguousarray(dims, np.int64)
    return _chk(getattr(lib(), "orc_factor_diagonal_blocks_" + _sfx(D))(_p(D), _p(dm), i64(len(dm)))) == 0


def solve_diagonal_blocks(y, D, dims, x):
    dm = np.ascontiguousarray(dims, np.int64)
    getattr(lib(), "orc_solve_diagonal_blocks_" + _sfx(D))(_p(y), _p(D), _p(dm), i64(len(dm)), _p(x))


def pcg_solve(st: Structure, pat: Pattern, S, g, x, tol=1e-8, maxit=100000, nthreads=None):
    """Block-Jacobi PCG on S x = g (S's upper triangle on the pattern); x updated in place. Returns
    (status, iterations, rel_residual): status 0 converged, 1 a diagonal block not PD, 2 not converged."""
    it, rel = C.c_int64(0), C.c_double(0.0)
    f = getattr(lib(), "orc_pcg_solve_" + _sfx(S))
    rc = _chk(f(st.h, pat.h, _p(S), _p(g), _p(x), C.c_double(tol), i64(maxit), C.c_int(nthreads or max_threads()), C.byref(it), C.byref(rel)))
    return rc, int(it.value), float(rel.value)


def assemble_hessian(q: QRStructure, Rw, Rr, pat: Pattern | None = None):
    """H = J'J and b = J'r of the raw tables in the SchurBlockHessian layout (the reference's fixtures form
    H = J64'J64 and b = J64'r, test/fixtures/QRFixtures.jl:109-120, and fill E_data / C_data / R by the layout of
    add_eliminated! / add_coupling! / add_retained_pair!, src/schur_assembly.jl:189-246): per table, over its data rows
    (the damping rows of an eliminated table are its last d_e rows), G = J_t'J_t and v = J_t'r_t in FP64, then
    E_e = G[point, point] (column-major), C_c = G[point, entry] (d_e x d_r column-major), b = [v over retained
    columns summed per block; v over the point's columns], and the retained blocks of G summed into R: on `pat`'s
    S.nzval layout (upper triangle of diagonal blocks) or, with pat None, a column-major dense nr x nr upper triangle."""
    st = q.st
    nr, ne = int(st.nr), int(st.ne)
    E, Cd, b = np.zeros(st.E_length), np.zeros(st.C_length), np.zeros(nr + ne)
    R = np.zeros(pat.nnz if pat is not None else nr * nr)
    for t in range(q.ntables):
        M, C1, top = int(q.table_nrows[t]), int(q.table_ncols[t]) - 1, int(q.table_top[t])
        n = M - top
        off, ro = int(q.raw_offsets[t]), int(q.residual_offsets[t])
        Jt = np.asarray(Rw[off:off + M * C1], np.float64).reshape(C1, M).T[:n]
        rt = np.asarray(Rr[ro:ro + n], np.float64)
        G, v = Jt.T @ Jt, Jt.T @ rt
        u0, u1e = int(q.table_ptr[t]), int(q.table_ptr[t + 1])
        cols = [(int(q.entry_col[u]), int(st.r_dims[q.entry_retained[u]]), int(q.entry_retained[u])) for u in range(u0, u1e)]
        if t < st.neblocks:
            de = int(st.e_dims[t])
            pc = slice(C1 - de, C1)
            eo = int(st.eoffsets[t])
            E[eo:eo + de * de] = G[pc, pc].ravel(order="F")
            b[nr + int(st.boffsets_e[t]):nr + int(st.boffsets_e[t]) + de] = v[pc]
            for k, (c0, dr, r) in enumerate(cols):
                co = int(st.coffsets[int(st.eliminated_ptr[t]) + k])
                Cd[co:co + de * dr] = G[pc, c0:c0 + dr].ravel(order="F")
        for k2, (c2, d2, r2) in enumerate(cols):
            o2 = int(st.boffsets_r[r2])
            b[o2:o2 + d2] += v[c2:c2 + d2]
            for k1 in range(k2 + 1):
                c1, d1, r1 = cols[k1]
                o1 = int(st.boffsets_r[r1])
                blk = G[c1:c1 + d1, c2:c2 + d2]
                if pat is not None:
                    lo, hi = int(pat.block_colptr[r2]), int(pat.block_colptr[r2 + 1])
                    kb = lo + int(np.searchsorted(pat.block_rowval[lo:hi], r1))
                    assert pat.block_rowval[kb] == r1
                for w in range(d2):
                    for a in range(d1):
                        if k1 == k2 and a > w:
                            continue
                        if pat is not None:
                            R[int(pat.S_colptr[o2 + w]) + int(pat.block_row_offsets[kb]) + a] += blk[a, w]
                        else:
                            R[o1 + a + nr * (o2 + w)] += blk[a, w]
    return E, Cd, R, b


def _table(q: QRStructure, D, t):
    M, C1 = int(q.table_nrows[t]), int(q.table_ncols[t]) - 1
    off = int(q.raw_offsets[t])
    return np.asarray(D[off:off + M * C1], np.float64).reshape(C1, M).T, M, C1


def jtr(q: QRStructure, D, Rv, *, diag=False):
    """jtr!(g, src) (src/qr_reduced.jl:575-584), or with diag=True jtj_diag!(d, src) (:586-595), from tables D (raw or
    factored) and their residual Rv: per retained block the sum over its entries, in retained_entry order, of each
    column's dot with the residual (or itself) over every row of the entry's table (sum_retained_columns!, :536-560);
    per eliminated block its point columns' dots (foreach_eliminated_column, :562-573). FP64."""
    st = q.st
    nr = int(st.nr)
    out = np.zeros(nr + int(st.ne))
    for r in range(int(st.nrblocks)):
        ro, dr = int(st.boffsets_r[r]), int(st.r_dims[r])
        for k in range(int(q.retained_ptr[r]), int(q.retained_ptr[r + 1])):
            u = int(q.retained_entry[k])
            t = int(q.entry_table[u])
            A, M, _ = _table(q, D, t)
            rv = None if diag else np.asarray(Rv[int(q.residual_offsets[t]):int(q.residual_offsets[t]) + M], np.float64)
            for j in range(dr):
                c = A[:, int(q.entry_col[u]) + j]
                out[ro + j] += float(np.dot(c, c if diag else rv))
    for e in range(int(st.neblocks)):
        A, M, C1 = _table(q, D, e)
        de = int(st.e_dims[e])
        rv = np.asarray(Rv[int(q.residual_offsets[e]):int(q.residual_offsets[e]) + M], np.float64) if not diag else None
        for k in range(de):
            c = A[:, C1 - de + k]
            out[nr + int(st.boffsets_e[e]) + k] = float(np.dot(c, c if diag else rv))
    return out


def jtj_quadform(q: QRStructure, D, v):
    """jtj_quadform(src, v) (src/qr_reduced.jl:597-640): sum over tables, in order, of sum over rows of (row . v)^2."""
    st = q.st
    nr = int(st.nr)
    total = 0.0
    for t in range(q.ntables):
        A, M, C1 = _table(q, D, t)
        x = np.zeros(C1)
        for u in range(int(q.table_ptr[t]), int(q.table_ptr[t + 1])):
            r = int(q.entry_retained[u])
            x[int(q.entry_col[u]):int(q.entry_col[u]) + int(st.r_dims[r])] = v[int(st.boffsets_r[r]):int(st.boffsets_r[r]) + int(st.r_dims[r])]
        if t < int(st.neblocks):
            de = int(st.e_dims[t])
            x[C1 - de:] = v[nr + int(st.boffsets_e[t]):nr + int(st.boffsets_e[t]) + de]
        total += float(np.sum((A @ x) ** 2))
    return total


_COND_EPS, _COND_BOUND = 1e-12, 2.0 ** 16
_FLOATMIN = {"f64": 2.2250738585072014e-308, "f32": float(np.finfo(np.float32).tiny)}


def conditioning_scale(d: float, T: str = "f64") -> float:
    """conditioning_scale (src/conditioning.jl:29-36): the power of two nearest, on a log scale, to
    1 / (1e-12 + sqrt|d|), at least floatmin(T); 1.0 for a non-finite d."""
    import math
    dd = abs(float(d))
    if not math.isfinite(dd):
        return 1.0
    f, e = math.frexp(1.0 / (_COND_EPS + math.sqrt(dd)))
    s = math.ldexp(1.0, e) if f >= math.sqrt(0.5) else math.ldexp(1.0, e - 1)
    return max(s, _FLOATMIN[T])


def prepare_scale(s, d, lam, sc, T: str = "f64", *, stale: bool) -> bool:
    """prepare_scale! (src/conditioning.jl:60-87) on the vector s in place; returns whether it was rewritten."""
    lam = max(float(lam), 0.0)
    dj = [float(d[j]) + lam * float(sc[j]) for j in range(len(s))]
    if not stale:
        drifted = False
        for j in range(len(s)):
            v = abs(dj[j]) * (float(s[j]) * float(s[j]))
            if not (1.0 / _COND_BOUND <= v <= _COND_BOUND) and conditioning_scale(dj[j], T) != s[j]:
                drifted = True
                break
        if not drifted:
            return False
    for j in range(len(s)):
        s[j] = conditioning_scale(dj[j], T)
    return True


def hessian_dense(st: Structure, R, E, Cd, pat: Pattern | None = None):
    """The full symmetric H of a SchurBlockHessian from R on the reduced pattern (its upper part; dense column-major
    nr x nr when pat is None), E_data and C_data in the structure's layout (add_eliminated! / add_coupling! /
    add_retained_pair!, src/schur_assembly.jl:189-246). dot(x, H, y) (src/linalg.jl:133-262) is x @ H @ y."""
    nr, ne = int(st.nr), int(st.ne)
    H = np.zeros((nr + ne, nr + ne))
    if pat is None:
        A = np.asarray(R, np.float64).reshape(nr, nr, order="F")
        U = np.triu(A)
    else:
        U = np.zeros((nr, nr))
        for j in range(nr):
            for q in range(int(pat.S_colptr[j]), int(pat.S_colptr[j + 1])):
                i = int(pat.S_rowval[q])
                if i <= j:
                    U[i, j] = R[q]
    H[:nr, :nr] = U + np.triu(U, 1).T
    for e in range(int(st.neblocks)):
        de, eo, so = int(st.e_dims[e]), int(st.eoffsets[e]), nr + int(st.boffsets_e[e])
        H[so:so + de, so:so + de] = np.asarray(E[eo:eo + de * de], np.float64).reshape(de, de, order="F")
        for c in range(int(st.eliminated_ptr[e]), int(st.eliminated_ptr[e + 1])):
            r = int(st.entry_retained[c])
            dr, ro, co = int(st.r_dims[r]), int(st.boffsets_r[r]), int(st.coffsets[c])
            B = np.asarray(Cd[co:co + de * dr], np.float64).reshape(de, dr, order="F")
            H[so:so + de, ro:ro + dr] = B
            H[ro:ro + dr, so:so + de] = B.T
    return H


def lsmr_reduced(Jt, rt, r_dims, lam, s_r=None, atol=1e-8, btol=1e-8, conlim=1e8, itmax=None):
    """The LSMR solve of the reduced problem (ext/KrylovExt.jl:97-132) restated with numpy on the written-out J~ (dense,
    m x nr) and r~: min ||[J~; sqrt(lam s_r)] x - [r~; 0]|| with the block-Jacobi N = D^-1 (D the diagonal blocks of
    A'A, blocks of sizes r_dims) as the change of variables x = L^-T y, D = L L'. The recurrences are Fong & Saunders'
    LSMR (SIAM J. Sci. Comput. 33, 2011: two plane rotations per step, the estimates of ||r||, ||A'r||, ||A||,
    cond(A), stopping tests 1-7) without internal damping, ||x|| taken in the original variables. Returns
    (x, status, iterations, istop) with status "ok", "not_pd" (the reference's NotPositiveDefinite: non-finite r~, lam
    == 0 with fewer rows than columns, a block of D not positive definite, istop 3 or 6) or "itmax"."""
    Jt = np.asarray(Jt, np.float64)
    m, nr = Jt.shape
    itmax = m + nr if itmax is None else itmax
    sqd = np.sqrt(lam * (np.ones(nr) if s_r is None else np.asarray(s_r, np.float64)))
    A = np.vstack([Jt, np.diag(sqd)])
    b = np.concatenate([np.asarray(rt, np.float64), np.zeros(nr)])
    if not np.all(np.isfinite(rt)):
        return np.zeros(nr), "not_pd", 0, 0
    if lam == 0 and m < nr:
        return np.zeros(nr), "not_pd", 0, 0
    Linv = np.zeros((nr, nr))   # block diagonal L^-1
    o = 0
    for d in r_dims:
        d = int(d)
        Db = A[:, o:o + d].T @ A[:, o:o + d]
        try:
            Lb = np.linalg.cholesky(Db)
        except np.linalg.LinAlgError:
            return np.zeros(nr), "not_pd", 0, 0
        Linv[o:o + d, o:o + d] = np.linalg.inv(Lb)
        o += d
    C = Linv.T                  # x = C y
    B = A @ C
    x = np.zeros(nr)
    beta = np.linalg.norm(b)
    if beta == 0:
        return x, "ok", 0, 0
    u = b / beta
    v = B.T @ u
    alpha = np.linalg.norm(v)
    if alpha > 0:
        v = v / alpha
    h, hbar = C @ v, np.zeros(nr)
    zetabar, alphabar, rho, rhobar, cbar, sbar = alpha * beta, alpha, 1.0, 1.0, 1.0, 0.0
    betadd, betad, rhodold, tautildeold, thetatilde, zeta = beta, 0.0, 1.0, 0.0, 0.0, 0.0
    normA2, maxrbar, minrbar = alpha * alpha, 0.0, 1e100
    normb, ctol = beta, (1.0 / conlim if conlim > 0 else 0.0)
    if alpha * beta == 0:
        return x, "ok", 0, 0
    if itmax == 0:
        return x, "itmax", 0, 7
    itn, istop = 0, 0
    while istop == 0:
        itn += 1
        u = B @ v - alpha * u
        beta = np.linalg.norm(u)
        if beta > 0:
            u = u / beta
            v = B.T @ u - beta * v
            alpha = np.linalg.norm(v)
            if alpha > 0:
                v = v / alpha
        rhoold = rho
        rho = np.hypot(alphabar, beta)
        c, s = alphabar / rho, beta / rho
        thetanew = s * alpha
        alphabar = c * alpha
        rhobarold, zetaold, thetabar, rhotemp = rhobar, zeta, sbar * rho, cbar * rho
        rhobar = np.hypot(cbar * rho, thetanew)
        cbar, sbar = cbar * rho / rhobar, thetanew / rhobar
        zeta, zetabar = cbar * zetabar, -sbar * zetabar
        hbar = h - (thetabar * rho / (rhoold * rhobarold)) * hbar
        x = x + (zeta / (rho * rhobar)) * hbar
        h = C @ v - (thetanew / rho) * h
        betahat, betadd = c * betadd, -s * betadd
        thetatildeold, rhotildeold = thetatilde, np.hypot(rhodold, thetabar)
        ctildeold, stildeold = rhodold / rhotildeold, thetabar / rhotildeold
        thetatilde, rhodold = stildeold * rhobar, ctildeold * rhobar
        betad = -stildeold * betad + ctildeold * betahat
        tautildeold = (zetaold - thetatildeold * tautildeold) / rhotildeold
        taud = (zeta - thetatilde * tautildeold) / rhodold
        normr = np.sqrt((betad - taud) ** 2 + betadd ** 2)
        normA2 += beta * beta
        normA = np.sqrt(normA2)
        normA2 += alpha * alpha
        maxrbar = max(maxrbar, rhobarold)
        if itn > 1:
            minrbar = min(minrbar, rhobarold)
        condA = max(maxrbar, rhotemp) / min(minrbar, rhotemp)
        normar, normx = abs(zetabar), np.linalg.norm(x)
        test1 = normr / normb
        test2 = normar / (normA * normr) if normA * normr != 0 else np.inf
        test3 = 1.0 / condA
        t1 = test1 / (1.0 + normA * normx / normb)
        rtol = btol + atol * normA * normx / normb
        if itn >= itmax:
            istop = 7
        if 1.0 + test3 <= 1.0:
            istop = 6
        if 1.0 + test2 <= 1.0:
            istop = 5
        if 1.0 + t1 <= 1.0:
            istop = 4
        if test3 <= ctol:
            istop = 3
        if test2 <= atol:
            istop = 2
        if test1 <= rtol:
            istop = 1
    status = "itmax" if istop == 7 else ("not_pd" if istop in (3, 6) else "ok")
    return x, status, itn, istop
