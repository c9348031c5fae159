"""QR test problems: the structures of the reference's QR fixtures (test/fixtures/QRFixtures.jl:55-80), 0-based, with the
random parts (couplings of the bundle-adjustment problem, extra rows of the mixed one) and every value drawn from
numpy's seeded generators, since the reference draws them from Julia's Xoshiro.
"""
from __future__ import annotations

import numpy as np


def _bundle(rng):
    c = [sorted(int(x) for x in rng.permutation(8)[: rng.integers(2, 5)]) for _ in range(60)]
    return dict(r_dims=[6] * 8, e_dims=[3] * 60, couplings=c, e_rows=[2 * len(x) for x in c])


def _mixed(rng):
    e = [12, 9, 8, 5, 3, 2, 1, 1]
    return dict(r_dims=[6, 3, 9, 6], e_dims=e, couplings=[[0, 2], [1, 3], [0, 1, 3], [2], [0, 3], [1, 2], [0], [3]],
                e_rows=[d + 4 + int(rng.integers(0, 7)) for d in e])


def _free(rng):
    return dict(r_dims=[6, 6, 6, 6, 3], e_dims=[3, 3, 3, 2, 2, 1], couplings=[[0, 1], [1, 2], [2, 3], [0, 3], [1], [0, 2]],
                e_rows=[8, 8, 7, 6, 5, 4], free_rows=[7, 3, 6], free_retained=[[1, 0], [2], [4, 3, 1]])


def _all(rng):
    return dict(r_dims=[6, 6, 3, 6], e_dims=[3, 3, 3, 3], couplings=[[0, 1, 2, 3], [0, 1], [2, 3], [1, 3]], e_rows=[24, 8, 8, 8])


def _single(rng):
    return dict(r_dims=[6, 3], e_dims=[4], couplings=[[0, 1]], e_rows=[20])


QR_FIXTURES = {"bundle adjustment": _bundle, "mixed dimensions": _mixed, "free groups": _free, "coupled to all": _all,
               "single eliminated block": _single}


def fill_tables(jst, rng, dtype=np.float64):
    """Raw tables and residual of a Jacobian on the structure `jst` (product or oracle fields): every data row of every
    entry's block, eliminated block and residual N(0, 1); damping rows zero (QRTestProblem, QRFixtures.jl:26-52).
    Also returns the dense J (rows in table order, columns [x_r; x_e]) and r."""
    st = jst.schur if hasattr(jst, "schur") else jst.st
    nr, ne = int(st.nr), int(np.sum(st.e_dims))
    rows = int(sum(int(jst.table_nrows[t]) - int(jst.table_top[t]) for t in range(jst.ntables)))
    Rw = np.zeros(int(jst.raw_offsets[-1]), dtype)
    Rr = np.zeros(int(jst.residual_offsets[-1]))
    Jf = np.zeros((rows, nr + ne))
    rf = np.zeros(rows)
    row = 0
    for t in range(jst.ntables):
        M, C, top = int(jst.table_nrows[t]), int(jst.table_ncols[t]) - 1, int(jst.table_top[t])
        mt = M - top
        T = np.zeros((M, C))
        for u in range(int(jst.table_ptr[t]), int(jst.table_ptr[t + 1])):
            r = int(jst.entry_retained[u])
            d, c0 = int(st.r_dims[r]), int(jst.entry_col[u])
            B = rng.standard_normal((mt, d))
            T[:mt, c0:c0 + d] = B
            Jf[row:row + mt, int(st.boffsets_r[r]):int(st.boffsets_r[r]) + d] = B
        if t < int(st.neblocks):
            de = int(st.e_dims[t])
            E = rng.standard_normal((mt, de))
            T[:mt, C - de:] = E
            Jf[row:row + mt, nr + int(st.boffsets_e[t]):nr + int(st.boffsets_e[t]) + de] = E
        rv = rng.standard_normal(mt)
        Rr[int(jst.residual_offsets[t]):int(jst.residual_offsets[t]) + mt] = rv
        rf[row:row + mt] = rv
        Rw[int(jst.raw_offsets[t]):int(jst.raw_offsets[t + 1])] = T.ravel(order="F")
        row += mt
    return Rw, Rr, Jf, rf
