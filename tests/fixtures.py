"""Test problems: the structures of the reference's own test fixtures, with values drawn from numpy's seeded generators.

The block structures are those of BlockLinearSystems.jl's tests (0-based here); the values cannot be the reference's
(its tests draw from Julia's Xoshiro, which is not available), so every value test checks an identity instead: the
Schur path's solution against a dense FP64 solve of the full system, as test/schur.jl:223-237 does.
"""
from __future__ import annotations

import numpy as np

# test/schur.jl:10-52: retained blocks 6, 3, 6, 9; eliminated 8 of size 3 and 2 of size 1
SCHUR_JL = dict(r_dims=[6, 3, 6, 9], e_dims=[3] * 8 + [1, 1],
                couplings=[[0, 1], [0, 2], [1, 2, 3], [0, 3], [0, 1, 2], [1, 3], [2, 3], [0, 1, 2, 3], [0, 2], [1, 3]])
# test/fixtures/SchurFixtures.jl:119-130 standard_problem
STANDARD = dict(r_dims=[6, 6, 6, 6], e_dims=[3] * 7 + [2] * 5 + [1] * 8,
                couplings=[[0, 1], [0, 1], [0, 1, 2], [1, 2], [2, 3], [2, 3], [0, 3], [0, 1], [1, 2], [2, 3], [0, 1, 2, 3], [3],
                           [0], [1], [2], [3], [0, 1], [2, 3], [1, 2], [0, 3]])
# test/fixtures/SchurFixtures.jl:134-140 coupled_groups_problem (retained-retained pairs without a shared point)
COUPLED_GROUPS = dict(r_dims=[6, 6, 6, 6], e_dims=[3, 3, 3, 3, 2, 2, 1, 1],
                      couplings=[[0, 1], [0, 1], [2, 3], [2, 3], [0], [3], [1, 0], [2, 3]], rr_pairs=[(2, 0), (3, 1), (1, 0)])
# test/fixtures/SchurFixtures.jl:189-208 gauge_problem (couplings only)
GAUGE = dict(r_dims=[6, 6, 6, 6], e_dims=[3] * 6, couplings=[[0, 1], [0, 1, 2], [1, 2, 3], [2, 3], [0, 3], [0, 1, 2, 3]])

# test/fixtures/SchurFixtures.jl:144-151 mixed_dims_problem: point blocks of 1 to 12 variables (the Cholesky forms above
# 3, and the reference's LAPACK form above 8), each coupled to up to three of four retained blocks (numpy's draws)
_mrng = np.random.default_rng(11)
MIXED_DIMS = dict(r_dims=[6, 3, 9, 6], e_dims=[12, 12, 9, 9, 8, 8, 5, 5, 4, 4, 3, 3, 2, 2, 1, 1],
                  couplings=[sorted(set(int(x) for x in _mrng.integers(0, 4, 3))) for _ in range(16)])

DEVICE_FIXTURES = {"schur_jl": SCHUR_JL, "standard": STANDARD, "coupled_groups": COUPLED_GROUPS, "gauge": GAUGE}


def make_problem(rng: np.random.Generator, r_dims, e_dims, couplings, rr_pairs=()):
    """A strictly diagonally dominant bipartite system, retained variables first (SchurTestProblem,
    test/fixtures/SchurFixtures.jl:26-54): blocks U(-1, 1), symmetrised from the upper triangle, diagonal made
    dominant by 0.5 + U(0, 1). Returns (H, b)."""
    nr, ne = sum(r_dims), sum(e_dims)
    n = nr + ne
    roff = np.concatenate([[0], np.cumsum(r_dims)[:-1]])
    eoff = nr + np.concatenate([[0], np.cumsum(e_dims)[:-1]])
    H = np.zeros((n, n))

    def fill(r0, nrow, c0, ncol):
        H[r0:r0 + nrow, c0:c0 + ncol] = 2 * rng.random((nrow, ncol)) - 1

    for r, d in enumerate(r_dims):
        fill(roff[r], d, roff[r], d)
    for e, d in enumerate(e_dims):
        fill(eoff[e], d, eoff[e], d)
    for e, cs in enumerate(couplings):
        for r in cs:
            fill(roff[r], r_dims[r], eoff[e], e_dims[e])
    for r1, r2 in rr_pairs:
        a, b = min(r1, r2), max(r1, r2)
        fill(roff[a], r_dims[a], roff[b], r_dims[b])
    H = np.triu(H) + np.triu(H, 1).T
    for i in range(n):
        H[i, i] = np.abs(H[i]).sum() - abs(H[i, i]) + 0.5 + rng.random()
    return H, rng.standard_normal(n)


def gauge_problem(rng: np.random.Generator, prior: float = 1e-8):
    """Singular along a gauge direction up to a tiny prior (test/fixtures/SchurFixtures.jl:189-208)."""
    r_dims, e_dims, couplings = GAUGE["r_dims"], GAUGE["e_dims"], GAUGE["couplings"]
    nr, ne = sum(r_dims), sum(e_dims)
    H = np.zeros((nr + ne, nr + ne))
    for e, cs in enumerate(couplings):
        for r in cs:
            w = 0.5 + rng.random()
            ri = 6 * r + np.arange(3)
            ei = nr + 3 * e + np.arange(3)
            H[np.ix_(ri, ri)] += w * np.eye(3)
            H[np.ix_(ei, ei)] += w * np.eye(3)
            H[np.ix_(ri, ei)] -= w * np.eye(3)
            H[np.ix_(ei, ri)] -= w * np.eye(3)
    for r in range(4):
        ri = 6 * r + np.arange(3, 6)
        H[np.ix_(ri, ri)] += prior * np.eye(3)
    return H, rng.standard_normal(nr + ne)


def split_hessian(H, st, pattern=None, dtype=np.float64):
    """E_data, C_data and R (dense column-major, or the sparse storage on `pattern`) of a full H laid out by the
    structure `st` (retained blocks first in H, in layout order). `st` may be the product's or the oracle's structure."""
    nr = int(st.nr)
    E = np.zeros(int(st.E_length), dtype)
    Cd = np.zeros(int(st.C_length), dtype)
    for e in range(int(st.neblocks)):
        de = int(st.e_dims[e])
        eo, so = int(st.eoffsets[e]), nr + int(st.boffsets_e[e])
        E[eo:eo + de * de] = H[so:so + de, so:so + de].ravel(order="F")
        for c in range(int(st.eliminated_ptr[e]), int(st.eliminated_ptr[e + 1])):
            r = int(st.entry_retained[c])
            dr, ro, co = int(st.r_dims[r]), int(st.boffsets_r[r]), int(st.coffsets[c])
            # stored d_e x d_r column-major: C[co + row*de + col] = H[retained row, eliminated col]
            Cd[co:co + dr * de] = H[ro:ro + dr, so:so + de].ravel(order="C")
    if pattern is None:
        R = np.asfortranarray(H[:nr, :nr]).ravel(order="F").astype(dtype)
    else:
        R = np.zeros(pattern.R_length, dtype)
        for r2 in range(int(st.nrblocks)):
            d2, o2 = int(st.r_dims[r2]), int(st.boffsets_r[r2])
            for k in range(int(pattern.block_colptr[r2]), int(pattern.block_colptr[r2 + 1])):
                r1 = int(pattern.block_rowval[k])
                d1, o1 = int(st.r_dims[r1]), int(st.boffsets_r[r1])
                # R block (row r2, column r1): d2 x d1 column-major
                R[int(pattern.R_block_start[k]):int(pattern.R_block_start[k]) + d2 * d1] = H[o2:o2 + d2, o1:o1 + d1].ravel(order="F")
    return E, Cd, R


def csc_to_dense_upper(nr, colptr, rowval, nzval):
    """Symmetric dense matrix from the upper triangle stored in a CSC (lower entries of diagonal blocks ignored)."""
    A = np.zeros((nr, nr))
    for j in range(nr):
        for q in range(int(colptr[j]), int(colptr[j + 1])):
            i = int(rowval[q])
            if i <= j:
                A[i, j] = nzval[q]
    return np.triu(A) + np.triu(A, 1).T


def dense_upper_sym(S_colmajor, nr):
    A = np.asarray(S_colmajor, np.float64).reshape(nr, nr, order="F")
    return np.triu(A) + np.triu(A, 1).T
