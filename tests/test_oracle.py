"""The oracle (CPU restatement of the reference) against the reference's own known answers and tolerances.

Known answers: tests/golden/known_answers.json (transcribed from the reference's tests). Value checks: the Schur
path's solution against a dense FP64 solve of the full system (test/schur.jl:223-237: 1e-12; K=4 vs K=1: 1e-14 dense,
1e-13 sparse, :255-256, :399-400), the rank-1 failure (:405-425), QR identities (test/qr_reduction.jl:20-58).
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from fixtures import COUPLED_GROUPS, SCHUR_JL, STANDARD, csc_to_dense_upper, dense_upper_sym, gauge_problem, make_problem, split_hessian

KA = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())


def test_doctest_structure():
    c = KA["doctest_structure"]
    st = orc.Structure.from_description(c["blocksizes"], c["rowblocks"], c["eliminated"])
    assert list(st.order) == c["blockorder"]
    assert st.nrblocks == c["nretained"]
    assert list(np.concatenate([st.r_dims, st.e_dims])) == c["layout_blocksizes"]


def test_doctest_jacobian_structure():
    import ctypes as C
    c = KA["doctest_jacobian_structure"]
    bs = np.array(c["blocksizes"], np.int64)
    ptr, idx = orc._csr(c["rowblocks"])
    rbs = np.array(c["rowblocksizes"], np.int64)
    el = np.array(c["eliminated"], np.uint8)
    q, s = C.c_void_p(), C.c_void_p()
    orc._chk(orc.lib().orc_qr_structure_from_description(orc.i64(len(bs)), orc._p(bs), orc.i64(len(rbs)), orc._p(ptr), orc._p(idx),
                                                         orc._p(rbs), orc._p(el), orc.i64(1), orc.i64(4096), C.byref(q), C.byref(s)))
    st = orc.Structure(s)
    assert list(st.order) == c["blockorder"] and st.nrblocks == c["nretained"] and st.nrblocks + st.neblocks == c["nblocks"]
    orc.lib().orc_qr_free(q)


def test_expand_block_perm_and_sort():
    c = KA["expand_block_perm"]
    assert list(orc.expand_block_perm(c["perm"], c["sizes"])) == c["expected"]
    c = KA["sort_schur_blocks"]
    assert list(orc.sort_schur_blocks(c["is_elim"], c["sizes"], c["couplings"])) == c["expected"]


def _hand_pattern(r_dims, couplings, extra=()):
    """The hand-built pattern of test/schur.jl:270-302."""
    nrb = len(r_dims)
    cols = [set([r]) for r in range(nrb)]
    for cs in couplings:
        s = sorted(cs)
        for j in range(len(s)):
            for i in range(j + 1):
                cols[s[j]].add(s[i])
    for a, b in extra:
        cols[max(a, b)].add(min(a, b))
    colptr = [0]
    rowval, offs, heights = [], [], []
    for c in range(nrb):
        h = 0
        for r in sorted(cols[c]):
            rowval.append(r)
            offs.append(h)
            h += r_dims[r]
        heights.append(h)
        colptr.append(len(rowval))
    return colptr, rowval, offs, heights


def test_pattern_equals_hand_built():
    st = orc.Structure.positional(SCHUR_JL["r_dims"], SCHUR_JL["e_dims"], SCHUR_JL["couplings"])
    pat = orc.Pattern(st)
    colptr, rowval, offs, heights = _hand_pattern(SCHUR_JL["r_dims"], SCHUR_JL["couplings"])
    assert list(pat.block_colptr) == colptr and list(pat.block_rowval) == rowval
    assert list(pat.block_row_offsets) == offs and list(pat.col_heights) == heights
    # diagonal indices: the diagonal entry's position in each scalar column
    for j in range(st.nr):
        lo, hi = pat.S_colptr[j], pat.S_colptr[j + 1]
        assert pat.S_rowval[pat.diag_inds[j]] == j and lo <= pat.diag_inds[j] < hi


def test_coupled_groups_extra_blocks_and_map_count():
    c = KA["coupled_groups_extra"]
    st = orc.Structure.positional(COUPLED_GROUPS["r_dims"], COUPLED_GROUPS["e_dims"], COUPLED_GROUPS["couplings"])
    plain = orc.Pattern(st)
    withextra = orc.Pattern(st, c["extra"])
    assert len(withextra.block_rowval) == len(plain.block_rowval) + c["added_blocks"]
    with pytest.raises(orc.OracleError):
        orc.Pattern(st, [(0, 4)])
    rr = COUPLED_GROUPS["rr_pairs"]
    pat = orc.Pattern(st, rr)
    m = pat.r_to_s_map()
    # R on the pattern stores every pattern block; the reference's R stores the couplings' blocks plus rr_pairs. The
    # count law (4*21 + 36*npairs) applies per stored block: diagonal blocks map 21 entries, off-diagonal blocks 36.
    nb = len(pat.block_rowval)
    ndiag = st.nrblocks
    k = KA["coupled_groups_r_to_s_count"]
    assert int((m >= 0).sum()) == ndiag * k["diag_upper_per_block"] + (nb - ndiag) * k["offdiag_per_block"]
    mapped = m[m >= 0]
    assert len(np.unique(mapped)) == len(mapped)
    cols = np.repeat(np.arange(st.nr), np.diff(pat.S_colptr))
    assert np.all(pat.S_rowval[mapped] <= cols[mapped])


def test_qr_bytes_formula():
    import ctypes as C
    c = KA["qr_bytes"]
    st = orc.Structure.positional([6] * c["nret"], [3] * c["nelim"], [list(range(c["nret"]))] * c["nelim"])
    q = C.c_void_p()
    e_rows = np.full(c["nelim"], c["rows"], np.int64)
    orc._chk(orc.lib().orc_qr_structure_positional(st.h, orc._p(e_rows), orc.i64(0), None, None, None, orc.i64(1), C.byref(q)))
    raw = np.empty(c["nelim"] + 1, np.int64)
    res = np.empty(c["nelim"] + 1, np.int64)
    orc.lib().orc_qr_field(q, b"raw_offsets", orc._p(raw))
    orc.lib().orc_qr_field(q, b"residual_offsets", orc._p(res))
    assert 2 * 8 * (raw[-1] + res[-1]) == c["expected_bytes"]
    orc.lib().orc_qr_free(q)


def test_inv_sym_block_known_answers():
    c = KA["inv_sym_2x2"]
    H = np.array(c["H"])
    assert orc.inv_sym_block(H.astype(np.float32), np.zeros(2, np.float32))[0] == c["f32_success"]
    assert orc.inv_sym_block(H, np.zeros(2))[0] == c["f64_success"]
    for A in KA["inv_sym_not_pd"]["cases"]:
        A = np.array(A, float)
        assert not orc.inv_sym_block(A, np.zeros(len(A)))[0]
        assert not orc.inv_sym_block(A, np.zeros(len(A)), generic=True)[0]


@pytest.mark.parametrize("kind", ["pd", "indefinite", "nd", "nearsingular"])
@pytest.mark.parametrize("damped", [False, True])
def test_closed_forms_agree_with_cholesky(kind, damped):
    """test/kernels.jl:11-49: the closed forms accept exactly what the Cholesky path accepts."""
    rng = np.random.default_rng(1)
    for D in (1, 2, 3):
        for _ in range(50):
            Q, _r = np.linalg.qr(rng.standard_normal((D, D)))
            if kind == "pd":
                ev = rng.random(D) + 0.1
            elif kind == "nd":
                ev = -(rng.random(D) + 0.1)
            elif kind == "indefinite":
                ev = rng.standard_normal(D)
                ev[0] = abs(ev[0]) + 0.1
                ev[-1] = -abs(ev[-1]) - 0.1
            else:
                ev = rng.random(D) + 0.1
                ev[0] = rng.choice([1e-3, 1e-8, 1e-16, 0.0, -1e-16])
            A = Q @ np.diag(ev) @ Q.T
            A = (A + A.T) / 2
            lam = rng.choice([1e-6, 1e-2, 1.0]) if damped else 0.0
            damp = lam * np.abs(np.diag(A)) if damped else np.zeros(D)
            ok1, inv1 = orc.inv_sym_block(A, damp)
            ok2, inv2 = orc.inv_sym_block(A, damp, generic=True)
            assert ok1 == ok2
            if ok1:
                assert np.allclose(inv1, inv2, rtol=np.sqrt(np.finfo(float).eps) * 1e3)


def _schur_solve(p, lam, scaling, dense, nchunks=1, nthreads=1, extra=()):
    """Reduce with the oracle, solve S densely, back-substitute; returns (x, S-as-dense, g)."""
    H, b, r_dims, e_dims, couplings = p
    st = orc.Structure.positional(r_dims, e_dims, couplings, nchunks=nchunks, min_work=0)
    nr = st.nr
    pat = None if dense else orc.Pattern(st, extra)
    E, Cd, R = split_hessian(H, st, pat)
    work = orc.Work(st, nchunks)
    sr, se = scaling[:nr].copy(), scaling[nr:].copy()
    g = np.zeros(nr)
    if dense:
        S = np.zeros(nr * nr)
        orc.reset_schur_dense(st, S, R, sr, lam)
        ok, fb = orc.reduce_schur_dense(st, work, S, g, b[:nr].copy(), b[nr:].copy(), se, lam, E, Cd, nthreads=nthreads)
        Sd = dense_upper_sym(S, nr)
    else:
        S = np.zeros(pat.nnz)
        orc.reset_schur_sparse(st, pat, S, R, sr, lam)
        ok, fb = orc.reduce_schur_sparse(st, pat, work, S, g, b[:nr].copy(), b[nr:].copy(), se, lam, E, Cd, nthreads=nthreads)
        Sd = csc_to_dense_upper(nr, pat.S_colptr, pat.S_rowval, S)
    if not ok:
        return None, fb
    x_r = np.linalg.solve(Sd, g)
    x_e = np.zeros(st.ne)
    orc.backsubstitute(st, work, x_e, x_r, Cd, nthreads=nthreads)
    return np.concatenate([x_r, x_e]), (S, g)


@pytest.mark.parametrize("name", ["schur_jl", "standard", "coupled_groups"])
@pytest.mark.parametrize("dense", [True, False])
def test_schur_path_matches_dense_solve(name, dense):
    fx = {"schur_jl": SCHUR_JL, "standard": STANDARD, "coupled_groups": COUPLED_GROUPS}[name]
    rng = np.random.default_rng(7)
    rr = fx.get("rr_pairs", [])
    H, b = make_problem(rng, fx["r_dims"], fx["e_dims"], fx["couplings"], rr)
    lam = 0.5
    scaling = 1.0 + rng.random(len(b))
    x, _ = _schur_solve((H, b, fx["r_dims"], fx["e_dims"], fx["couplings"]), lam, scaling, dense, extra=rr)
    x_ref = np.linalg.solve(H + lam * np.diag(scaling), b)
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-12


@pytest.mark.parametrize("dense", [True, False])
@pytest.mark.parametrize("lam", [1e-6, 1e-3, 0.1])
def test_gauge_problem_backward_stable(dense, lam):
    """test/schur_problems.jl:43-58: on the gauge-deficient problem the relative residual stays at rounding level."""
    rng = np.random.default_rng(21)
    H, b = gauge_problem(rng)
    x, _ = _schur_solve((H, b, [6] * 4, [3] * 6, [[0, 1], [0, 1, 2], [1, 2, 3], [2, 3], [0, 3], [0, 1, 2, 3]]), lam, np.ones(len(b)), dense)
    Hd = H + lam * np.eye(len(b))
    rel_res = np.linalg.norm(Hd @ x - b) / (np.linalg.norm(Hd, 2) * np.linalg.norm(x) + np.linalg.norm(b))
    assert rel_res <= 1e-13


@pytest.mark.parametrize("dense", [True, False])
def test_threaded_equals_serial(dense):
    rng = np.random.default_rng(3)
    H, b = make_problem(rng, SCHUR_JL["r_dims"], SCHUR_JL["e_dims"], SCHUR_JL["couplings"])
    sc = 1.0 + rng.random(len(b))
    p = (H, b, SCHUR_JL["r_dims"], SCHUR_JL["e_dims"], SCHUR_JL["couplings"])
    _, (S1, g1) = _schur_solve(p, 0.5, sc, dense, nchunks=1, nthreads=1)
    _, (S4, g4) = _schur_solve(p, 0.5, sc, dense, nchunks=4, nthreads=4)
    tol = 1e-14 if dense else 1e-13
    assert np.linalg.norm(S4 - S1) <= tol * np.linalg.norm(S1)
    assert np.linalg.norm(g4 - g1) <= tol * np.linalg.norm(g1)


def test_rank_one_block_fails_with_lowest_index():
    rng = np.random.default_rng(5)
    fx = SCHUR_JL
    H, b = make_problem(rng, fx["r_dims"], fx["e_dims"], fx["couplings"])
    nr = sum(fx["r_dims"])
    v = rng.standard_normal(3)
    H[nr:nr + 3, nr:nr + 3] = np.outer(v, v)
    x, fb = _schur_solve((H, b, fx["r_dims"], fx["e_dims"], fx["couplings"]), 0.0, np.ones(len(b)), True)
    assert x is None and fb == 1
    # two bad blocks: the lowest wins, threaded or not
    H[nr + 9:nr + 12, nr + 9:nr + 12] = np.outer(v, v)
    for nch in (1, 4):
        x, fb = _schur_solve((H, b, fx["r_dims"], fx["e_dims"], fx["couplings"]), 0.0, np.ones(len(b)), False, nchunks=nch, nthreads=nch)
        assert x is None and fb == 1


def test_bad_damping_rejected_before_any_write():
    st = orc.Structure.positional(SCHUR_JL["r_dims"], SCHUR_JL["e_dims"], SCHUR_JL["couplings"])
    nr = st.nr
    S = np.full(nr * nr, 7.0)
    R = np.zeros(nr * nr)
    for sc, lam in ((np.ones(nr), -0.1), (np.ones(nr), np.nan), (np.r_[np.ones(nr - 1), -1.0], 0.1), (np.r_[np.nan, np.ones(nr - 1)], 0.1)):
        with pytest.raises(orc.OracleError):
            orc.reset_schur_dense(st, S, R, sc, lam)
        assert np.all(S == 7.0)
