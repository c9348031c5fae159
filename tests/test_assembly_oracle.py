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
    # and the oracle's dense H of that Hessian (the layout dot(x, H, y) reads) is J'J itself
    assert relerr(orc.hessian_dense(st, R, E, Cd, pat), H) < 1e-14
    assert relerr(orc.hessian_dense(st, Rd, E, Cd, None), H) < 1e-14


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


@pytest.mark.parametrize("name", list(QR_FIXTURES))
def test_jacobian_queries_are_dense(name):
    """jtr!, jtj_diag! and jtj_quadform of the oracle against J'r, diag(J'J) and ||J v||^2 of the dense J (the fixture's
    damping rows are zero, so every row of the tables is a row of J)."""
    rng = np.random.default_rng(6)
    fx = QR_FIXTURES[name](rng)
    st = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    q = orc.QRStructure.positional(st, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    Rw, Rr, Jf, rf = fill_tables(q, rng)
    assert relerr(orc.jtr(q, Rw, Rr), Jf.T @ rf) < 1e-14
    assert relerr(orc.jtr(q, Rw, None, diag=True), np.sum(Jf * Jf, axis=0)) < 1e-14
    v = rng.standard_normal(Jf.shape[1])
    assert abs(orc.jtj_quadform(q, Rw, v) - np.sum((Jf @ v) ** 2)) <= 1e-13 * np.sum((Jf @ v) ** 2)


def test_conditioning_scale_rule():
    """conditioning_scale (src/conditioning.jl:29-36): a power of two, the nearest on a log scale to
    1/(1e-12 + sqrt|d|), floored at floatmin(T), 1 for a non-finite d; prepare_scale! (:60-87) keeps the scale while
    |d + lambda sc| s^2 stays in [2^-16, 2^16] and recomputes every entry once one entry leaves it."""
    import math
    rng = np.random.default_rng(7)
    for d in list(10.0 ** rng.uniform(-300, 300, 500)) + [0.0, -3.0, 1e-320, 5e-324]:
        s = orc.conditioning_scale(d)
        m, e = math.frexp(s)
        assert m == 0.5
        target = 1.0 / (1e-12 + math.sqrt(abs(d)))
        assert abs(math.log2(s) - math.log2(target)) <= 0.5 + 1e-12
    assert orc.conditioning_scale(float("inf")) == 1.0 and orc.conditioning_scale(float("nan")) == 1.0
    assert orc.conditioning_scale(1e300, "f32") == float(np.finfo(np.float32).tiny)
    d = 10.0 ** rng.uniform(-4, 4, 50)
    sc = np.ones(50)
    s = np.zeros(50)
    assert orc.prepare_scale(s, d, 1e-3, sc, stale=True)
    s0 = s.copy()
    assert not orc.prepare_scale(s, d, 2e-3, sc, stale=False) and (s == s0).all()   # a small change of damping
    assert orc.prepare_scale(s, d, 1e6, sc, stale=False) and not (s == s0).all()    # one far enough to drift
