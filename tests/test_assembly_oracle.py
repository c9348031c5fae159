"""The oracle's assembly of H = J'J, b = J'r from the raw tables, pinned against the reference's own definition: its QR
fixtures form the Hessian side as the dense J64'J64 and J64'r (test/fixtures/QRFixtures.jl:109-120) and store it in the
SchurBlockHessian layout of add_eliminated! / add_coupling! / add_retained_pair! (src/schur_assembly.jl:189-246).
Every E block, coupling block, retained block (on the reduced pattern and dense) and b entry is compared with the dense
product at 1e-14.
"""
import numpy as np
import pytest

import oracle as orc
from qr_fixtures import QR_FIXTURES, fill_tables


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("name", list(QR_FIXTURES))
def test_assembly_is_dense_jtj(name):
    rng = np.random.default_rng(5)
    fx = QR_FIXTURES[name](rng)
    st = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    q = orc.QRStructure.positional(st, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    Rw, Rr, Jf, rf = fill_tables(q, rng)
    H, b = Jf.T @ Jf, Jf.T @ rf
    nr = int(st.nr)
    pat = orc.Pattern(st, orc_free_pairs(q))
    E, Cd, R, bb = orc.assemble_hessian(q, Rw, Rr, pat)
    _, _, Rd, _ = orc.assemble_hessian(q, Rw, Rr, None)
    assert relerr(bb, b) < 1e-14
    # E and the coupling blocks at the structure's offsets
    for e in range(st.neblocks):
        de, eo, so = int(st.e_dims[e]), int(st.eoffsets[e]), nr + int(st.boffsets_e[e])
        assert relerr(E[eo:eo + de * de], H[so:so + de, so:so + de].ravel(order="F")) < 1e-14
        for c in range(int(st.eliminated_ptr[e]), int(st.eliminated_ptr[e + 1])):
            r = int(st.entry_retained[c])
            dr, ro, co = int(st.r_dims[r]), int(st.boffsets_r[r]), int(st.coffsets[c])
            assert relerr(Cd[co:co + de * dr], H[so:so + de, ro:ro + dr].ravel(order="F")) < 1e-14
    # retained blocks: dense upper triangle, and on the pattern (upper triangle of diagonal blocks, zero below)
    A = Rd.reshape(nr, nr, order="F")
    assert relerr(A, np.triu(H[:nr, :nr])) < 1e-14
    ref = np.zeros(pat.nnz)
    for j in range(nr):
        for k in range(int(pat.S_colptr[j]), int(pat.S_colptr[j + 1])):
            i = int(pat.S_rowval[k])
            ref[k] = H[i, j] if i <= j else 0.0
    assert relerr(R, ref) < 1e-14


def orc_free_pairs(q):
    """The retained pairs of the free tables (free_block_pairs, src/qr_reduced.jl:7-22), 0-based (r1, r2)."""
    out = set()
    for t in range(int(q.st.neblocks), q.ntables):
        rs = [int(q.entry_retained[u]) for u in range(int(q.table_ptr[t]), int(q.table_ptr[t + 1]))]
        for a in rs:
            for b in rs:
                if a < b:
                    out.add((a, b))
    return sorted(out)
