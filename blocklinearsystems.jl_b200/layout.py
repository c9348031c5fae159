"""Host-side layout of an elimination, mirroring BlockLinearSystems.jl's structure API (0-based).

SchurStructure            src/schur_structure.jl:50-166, src/schur_description.jl:16-101
build_schur_pattern       src/schur_structure.jl:241-323
build_r_to_s_map          src/schur_structure.jl:406-431 (block-level form)
sparse_with_map           src/SparseBlockLinearSystem.jl:233-282, 343-354 (makesparseindices + the scatter map)

All integer results are computed by the native library (libblsgpu.so); this module only marshals arrays.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, ptr64

DEFAULT_MIN_WORK = 4096   # src/threading.jl:24


def _csr(lists) -> tuple[np.ndarray, np.ndarray]:
    """A list of index lists, or a (ptr, idx) pair, as int64 CSR arrays."""
    if isinstance(lists, tuple) and len(lists) == 2 and isinstance(lists[0], np.ndarray):
        return np.ascontiguousarray(lists[0], np.int64), np.ascontiguousarray(lists[1], np.int64)
    ptr = np.zeros(len(lists) + 1, np.int64)
    ptr[1:] = np.cumsum([len(x) for x in lists])
    idx = np.fromiter((int(v) for x in lists for v in x), np.int64, count=int(ptr[-1]))
    return ptr, idx


class SchurStructure:
    """The layout of an elimination on the Hessian path (src/schur_structure.jl:1-49).

    SchurStructure(blocksizes, rowblocks, eliminated=..., nchunks=1, min_work=4096) lays out a description in the
    caller's numbering (0-based column blocks; `rowblocks` a list of index lists or a (ptr, idx) CSR pair).
    SchurStructure.positional(r_dims, e_dims, couplings) is the positional constructor. Array attributes are 0-based
    int64 numpy arrays; `chunks` / `col_chunks` are flattened half-open ranges.
    """

    _FIELDS = ("r_dims", "e_dims", "boffsets_r", "boffsets_e", "eoffsets", "eliminated_ptr", "entry_retained", "coffsets",
               "order", "chunks", "retained_ptr", "retained_entry", "entry_eliminated", "col_chunks", "retained_pairs")
    _SCALARS = ("nr", "ne", "nrblocks", "neblocks", "max_coupled_dim", "E_length", "C_length", "nchunks", "min_work")

    def __init__(self, blocksizes=None, rowblocks=None, *, eliminated=None, nchunks: int = 1, min_work: int = DEFAULT_MIN_WORK,
                 _handle=None):
        L = _lib.gpu()
        if _handle is None:
            if eliminated is None:
                raise TypeError("eliminated is required")
            bs = np.ascontiguousarray(blocksizes, np.int64)
            el = np.ascontiguousarray(np.asarray(eliminated, bool), np.uint8)
            if len(el) != len(bs):
                raise _lib.DimensionMismatch(f"eliminated has length {len(el)}, but there are {len(bs)} column blocks")
            ptr, idx = _csr(rowblocks)
            h = C.c_void_p()
            check(L.bls_structure_from_description(len(bs), ptr64(bs), len(ptr) - 1, ptr64(ptr), ptr64(idx),
                                                   el.ctypes.data_as(C.POINTER(C.c_uint8)), int(nchunks), int(min_work),
                                                   C.byref(h)))
            _handle = h
        self._h = _handle
        for f in self._SCALARS:
            setattr(self, f, int(self._field(f)[0]))
        for f in self._FIELDS:
            setattr(self, f, self._field(f))
        self.retained_pairs = self.retained_pairs.reshape(-1, 2)

    @classmethod
    def positional(cls, r_dims, e_dims, couplings, *, nchunks: int = 1, min_work: int = DEFAULT_MIN_WORK) -> "SchurStructure":
        rd = np.ascontiguousarray(r_dims, np.int64)
        ed = np.ascontiguousarray(e_dims, np.int64)
        ptr, idx = _csr(couplings)
        h = C.c_void_p()
        check(_lib.gpu().bls_structure_positional(len(rd), ptr64(rd), len(ed), ptr64(ed), ptr64(ptr), ptr64(idx), int(nchunks),
                                                  int(min_work), C.byref(h)))
        return cls(_handle=h)

    def _field(self, name: str) -> np.ndarray:
        L = _lib.gpu()
        n = L.bls_structure_field(self._h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, np.int64)
        if n:
            L.bls_structure_field(self._h, name.encode(), ptr64(out))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_structure_destroy(h)
            self._h = None

    # accessors (src/schur_description.jl:199-214)
    def blockorder(self) -> np.ndarray:
        return self.order.copy()

    def nretained(self) -> int:
        return self.nrblocks

    def nblocks(self) -> int:
        return self.nrblocks + self.neblocks

    def blocksizes(self) -> np.ndarray:
        return np.concatenate([self.r_dims, self.e_dims])

    def position(self) -> np.ndarray:
        """Layout position of each caller block (invperm of blockorder)."""
        p = np.empty_like(self.order)
        p[self.order] = np.arange(len(self.order))
        return p

    @property
    def handle(self):
        return self._h


@dataclass
class SchurPattern:
    """build_schur_pattern's result (src/schur_structure.jl:314-322), 0-based, plus the sparse retained storage laid
    out on it (src/schur_hessian.jl:286): R_block_start per block (the block (r2, r1) of R for the k-th pattern block
    (r1, r2)) and R_length."""
    block_colptr: np.ndarray
    block_rowval: np.ndarray
    block_row_offsets: np.ndarray
    col_heights: np.ndarray
    S_colptr: np.ndarray
    S_rowval: np.ndarray
    diag_inds: np.ndarray
    R_block_start: np.ndarray
    R_length: int
    _h: object = None

    @property
    def nnz(self) -> int:
        return int(self.S_colptr[-1])

    def R_diag_start(self, nrblocks: int) -> np.ndarray:
        """Start of each retained block's diagonal block in the retained storage."""
        out = np.empty(nrblocks, np.int64)
        for r in range(nrblocks):
            lo, hi = self.block_colptr[r], self.block_colptr[r + 1]
            k = lo + np.searchsorted(self.block_rowval[lo:hi], r)
            out[r] = self.R_block_start[k]
        return out

    def __del__(self):
        if self._h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_pattern_destroy(self._h)
            self._h = None


@dataclass
class BlockSystem:
    """The layout of a block-square SparseBlockLinearSystem (src/SparseBlockLinearSystem.jl:11-35), 0-based: its block
    sizes and indicestransposed as a CSC over block rows r (colptr), whose rows are the block columns c (rowval) and
    whose values are the blocks' starts in the data (starts; block (r, c) is blocksizes[r] x blocksizes[c],
    column-major)."""
    blocksizes: np.ndarray
    colptr: np.ndarray
    rowval: np.ndarray
    starts: np.ndarray

    @classmethod
    def retained(cls, structure: "SchurStructure", pattern: "SchurPattern") -> "BlockSystem":
        """The retained storage R on a Schur pattern: block (r2, r1), r1 <= r2, of R for pattern block (r1, r2)."""
        return cls(np.ascontiguousarray(structure.r_dims, np.int64), pattern.block_colptr, pattern.block_rowval,
                   pattern.R_block_start)

    @property
    def size(self) -> int:
        return int(np.sum(self.blocksizes))


def retained_block_pairs(bsys: "BlockSystem") -> list:
    """retained_block_pairs(R) (src/schur_structure.jl:325-334): the off-diagonal stored blocks of R as 0-based
    (row_block, col_block) pairs in indicestransposed's order, to pass as extra_blocks to build_schur_pattern."""
    out = []
    for r in range(len(bsys.blocksizes)):
        for k in range(int(bsys.colptr[r]), int(bsys.colptr[r + 1])):
            c = int(bsys.rowval[k])
            if r != c:
                out.append((r, c))
    return out


def build_r_to_s_map_scalar(R_colptr, R_rowval, S_colptr, S_rowval) -> np.ndarray:
    """build_r_to_s_map(R_sparse, S_sparse) (src/schur_structure.jl:336-353): for each stored entry of the CSC R (0-based
    colptr / rowval) its position in S.nzval (the scalar CSC S_colptr / S_rowval, rows sorted). ArgumentError if an
    entry of R is not in S."""
    rc, rr, sc, sr = (np.ascontiguousarray(a, np.int64) for a in (R_colptr, R_rowval, S_colptr, S_rowval))
    out = np.empty(len(rr), np.int64)
    check(_lib.gpu().bls_r_to_s_map_csc(len(rc) - 1, ptr64(rc), ptr64(rr) if len(rr) else None, ptr64(sc), ptr64(sr) if len(sr) else None,
                                        ptr64(out) if len(out) else None))
    return out


def build_r_to_s_map_blocks(bsys: "BlockSystem", S_colptr, S_rowval, boffsets_r, data_len: int) -> np.ndarray:
    """build_r_to_s_map(R_sys, S_sparse, boffsets_r) (src/schur_structure.jl:363-397): for each entry of R's block storage
    (data_len entries) its position in the scalar S.nzval: a diagonal block's upper triangle and every entry of a block
    below the diagonal (in S's upper triangle); -1 elsewhere (the reference's 0). ArgumentError if S lacks one."""
    bs, cp, rv, st = (np.ascontiguousarray(a, np.int64) for a in (bsys.blocksizes, bsys.colptr, bsys.rowval, bsys.starts))
    sc, sr, bo = (np.ascontiguousarray(a, np.int64) for a in (S_colptr, S_rowval, boffsets_r))
    out = np.empty(int(data_len), np.int64)
    check(_lib.gpu().bls_r_to_s_map_blocks_csc(len(bs), ptr64(bs), ptr64(cp), ptr64(rv) if len(rv) else None, ptr64(st) if len(st) else None,
                                               int(data_len), ptr64(sc), ptr64(sr) if len(sr) else None, ptr64(bo),
                                               ptr64(out) if len(out) else None))
    return out


def build_schur_pattern(structure: SchurStructure, extra_blocks=()) -> SchurPattern:
    """build_schur_pattern(structure; extra_blocks) (src/schur_structure.jl:241-323)."""
    L = _lib.gpu()
    ex = np.ascontiguousarray(np.asarray(list(extra_blocks), np.int64).reshape(-1, 2))
    h = C.c_void_p()
    check(L.bls_schur_pattern_build(structure.handle, len(ex), ptr64(ex) if len(ex) else None, C.byref(h)))

    def f(name):
        n = L.bls_pattern_field(h, name.encode(), None)
        out = np.empty(n, np.int64)
        if n:
            L.bls_pattern_field(h, name.encode(), ptr64(out))
        return out

    return SchurPattern(f("block_colptr"), f("block_rowval"), f("block_row_offsets"), f("col_heights"), f("S_colptr"),
                        f("S_rowval"), f("diag_inds"), f("R_block_start"), int(f("R_length")[0]), h)


def build_r_to_s_map(structure: SchurStructure, pattern: SchurPattern) -> np.ndarray:
    """build_r_to_s_map(R, pattern, boffsets_r) (src/schur_structure.jl:406-431) for the retained storage on the
    pattern; -1 marks an unmapped entry (the reference's 0)."""
    out = np.empty(pattern.R_length, np.int64)
    check(_lib.gpu().bls_build_r_to_s_map(structure.handle, pattern._h, ptr64(out)))
    return out


def sparse_with_map(structure: SchurStructure, pattern: SchurPattern, symmetric: bool = False):
    """makesparseindices + sparse_with_map (src/SparseBlockLinearSystem.jl:233-282, 343-354) for the retained storage:
    returns (colptr, rowval, scatter_map), 0-based; the CSC values are storage[scatter_map]."""
    L = _lib.gpu()
    n = L.bls_sparse_indices(structure.handle, pattern._h, int(symmetric), None, None, None)
    check(int(n) if n < 0 else 0)
    colptr = np.empty(structure.nr + 1, np.int64)
    rowval = np.empty(n, np.int64)
    smap = np.empty(n, np.int64)
    L.bls_sparse_indices(structure.handle, pattern._h, int(symmetric), ptr64(colptr), ptr64(rowval), ptr64(smap))
    return colptr, rowval, smap
