"""Device QR elimination through the C ABI against the oracle (the reference's qr_table!/reduce_qr! restated on the CPU).

FP64: factored tables, factored residual, J~'J~ (sparse and dense), J~'r~, the diagonal blocks and the back-substituted
x_e within 1e-12 relative of the oracle (the device sums the column norms in another order; the reference's own
identities, test/qr_reduction.jl:20-58, hold at 1e-10 and are checked too: J~'J~ is the Schur complement of the damped
normal equations). Mixed form (FP32 tables, FP64 norms and reflector arithmetic): against the FP64 oracle on the same
FP32-rounded tables, within 1e-5 relative on the reference's fixtures (condition numbers near 10) and within the
bound stated in the scene test on the ill-conditioned QR workload.
Failure reporting (the lowest failing table, non-finite and singular), argument checks, conditioning scales.
"""
import numpy as np
import pytest
import torch

import oracle as orc
from qr_fixtures import QR_FIXTURES, fill_tables

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def cu(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(DEV)


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def fixture(bls, name, seed=3):
    rng = np.random.default_rng(seed)
    fx = QR_FIXTURES[name](rng)
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    ost = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    j = bls.SchurJacobianStructure.positional(st, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    o = orc.QRStructure.positional(ost, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    Rw, Rr, Jf, rf = fill_tables(j, rng)
    sc_e = 0.5 + rng.random(j.schur.ne)
    return j, o, Rw, Rr, Jf, rf, sc_e


def run_both(bls, j, o, Rw, Rr, sc_e, lam, dtype, s=None, sparse=True):
    npdt = np.float32 if dtype == torch.float32 else np.float64
    Rw_s = Rw.astype(npdt)
    pairs = bls.free_block_pairs(j)
    pat = bls.build_schur_pattern(j.schur, pairs) if sparse else None
    opat = orc.Pattern(o.st, pairs) if sparse else None
    ws = bls.QRReductionWorkspace(j, pat, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw_s), r=cu(Rr))
    ok = bls.reduce_qr(ws, J, cu(sc_e), lam, None if s is None else cu(s))
    F, Fr = np.zeros(o.raw_length), np.zeros(o.residual_length)
    ook, ofb = orc.reduce_qr(o, F, Fr, Rw_s.astype(np.float64), Rr, sc_e, lam, s)
    out = dict(ok=ok, fb=ws.failed_block, ook=ook, ofb=ofb, ws=ws, F=ws.factored.double().cpu().numpy(), oF=F,
               Fr=ws.fres.cpu().numpy(), oFr=Fr, pat=pat, opat=opat)
    if not (ok and ook):
        return out
    nr, ne = j.schur.nr, j.schur.ne
    # J~'J~ and J~'r~, dense and sparse
    Sd = torch.zeros(nr * nr, dtype=dtype, device=DEV)
    gd = torch.zeros(nr, dtype=torch.float64, device=DEV)
    bls.reduced_normal_dense(Sd, gd, ws)
    oSd, ogd = np.zeros(nr * nr), np.zeros(nr)
    orc.reduced_normal_dense(o, oSd, ogd, F, Fr)
    out.update(Sd=Sd.double().cpu().numpy(), oSd=oSd, gd=gd.cpu().numpy(), ogd=ogd)
    if sparse:
        Ss = torch.zeros(pat.nnz, dtype=dtype, device=DEV)
        gs = torch.zeros(nr, dtype=torch.float64, device=DEV)
        bls.reduced_normal_sparse(Ss, gs, ws, pat)
        oSs, ogs = np.zeros(opat.nnz), np.zeros(nr)
        orc.reduced_normal_sparse(o, opat, oSs, ogs, F, Fr)
        out.update(Ss=Ss.double().cpu().numpy(), oSs=oSs, gs=gs.cpu().numpy(), ogs=ogs)
    D = torch.zeros(int(j.doffsets[-1]), dtype=dtype, device=DEV)
    bls.reduced_diagonal_blocks(D, ws)
    oD = np.zeros(int(o.doffsets[-1]))
    orc.reduced_diagonal_blocks(o, oD, F)
    x_r = np.random.default_rng(11).standard_normal(nr)
    x_e = torch.zeros(ne, dtype=torch.float64, device=DEV)
    bls.qr_backsubstitute(x_e, cu(x_r), ws)
    ox_e = np.zeros(ne)
    orc.qr_backsubstitute(o, ox_e, x_r, F, Fr)
    out.update(D=D.double().cpu().numpy(), oD=oD, x_r=x_r, x_e=x_e.cpu().numpy(), ox_e=ox_e)
    return out


def check_close(out, tol, sparse=True, keys=("F", "Fr", "Sd", "gd", "D", "x_e")):
    assert out["ok"] and out["ook"] and out["fb"] == 0
    for k in keys + (("Ss", "gs") if sparse else ()):
        t = tol[k] if isinstance(tol, dict) else tol
        e = relerr(out[k], out["o" + k])
        assert e <= t, f"{k}: relative error {e:.3e} > {t:.1e}"


@pytest.mark.parametrize("name", list(QR_FIXTURES))
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_fixtures_vs_oracle(bls, name, dtype):
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, name)
    out = run_both(bls, j, o, Rw, Rr, sc_e, 0.3, dtype)
    check_close(out, 1e-12 if dtype == torch.float64 else 1e-5)


@pytest.mark.parametrize("name", ["bundle adjustment", "free groups", "mixed dimensions"])
def test_schur_identity(bls, name):
    """J~'J~ = the Schur complement of the damped normal equations, J~'r~ the reduced right-hand side
    (test/qr_reduction.jl:20-58), and x_e solves the eliminated rows: U x_e = q - B x_r."""
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, name)
    lam = 0.3
    out = run_both(bls, j, o, Rw, Rr, sc_e, lam, torch.float64)
    nr = j.schur.nr
    H = Jf.T @ Jf
    b = Jf.T @ rf
    H[nr:, nr:] += lam * np.diag(sc_e)
    X = np.linalg.solve(H[nr:, nr:], np.hstack([H[nr:, :nr], b[nr:, None]]))
    S = H[:nr, :nr] - H[:nr, nr:] @ X[:, :nr]
    g = b[:nr] - H[:nr, nr:] @ X[:, nr]
    Sd = out["Sd"].reshape(nr, nr, order="F")
    Sd = np.triu(Sd) + np.triu(Sd, 1).T
    assert relerr(Sd, S) <= 1e-10
    assert relerr(out["gd"], g) <= 1e-10
    # back-substitution: the eliminated variables of the full damped solve given its retained ones
    x_full = np.linalg.solve(H, b)
    x_e = torch.zeros(j.schur.ne, dtype=torch.float64, device=DEV)
    bls.qr_backsubstitute(x_e, cu(x_full[:nr]), out["ws"])
    assert relerr(x_e.cpu().numpy(), x_full[nr:]) <= 1e-10


def test_conditioning_scales(bls):
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, "free groups")
    rng = np.random.default_rng(5)
    s = 2.0 ** rng.integers(-3, 4, j.schur.nr + j.schur.ne).astype(np.float64)
    for dtype, tol in ((torch.float64, 1e-12), (torch.float32, 1e-5)):
        check_close(run_both(bls, j, o, Rw, Rr, sc_e, 0.2, dtype, s=s), tol)


def test_dense_only_plan(bls):
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, "coupled to all")
    out = run_both(bls, j, o, Rw, Rr, sc_e, 0.1, torch.float64, sparse=False)
    check_close(out, 1e-12, sparse=False)
    with pytest.raises(bls.ArgumentError):
        bls.reduced_normal_sparse(torch.zeros(4, dtype=torch.float64, device=DEV), torch.zeros(j.schur.nr, dtype=torch.float64, device=DEV),
                                  out["ws"])


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_lowest_failure(bls, dtype):
    """A non-finite table and a singular one (zero eliminated columns, no damping): the lowest is reported
    (test/schur_qr.jl:395-428); free tables are then not copied."""
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, "bundle adjustment")
    for spoil in ([(41, "nan"), (17, "zero"), (30, "inf")], [(5, "zero"), (9, "nan")], [(59, "nan")]):
        W = Rw.copy()
        for t, how in spoil:
            M, C = int(j.table_nrows[t]), int(j.table_ncols[t]) - 1
            T = W[j.raw_offsets[t]:j.raw_offsets[t + 1]].reshape(C, M).T.copy()
            if how == "zero":
                T[:, C - 3:] = 0.0
            else:
                T[0, 0] = np.nan if how == "nan" else np.inf
            W[j.raw_offsets[t]:j.raw_offsets[t + 1]] = T.T.ravel()
        out = run_both(bls, j, o, W, Rr, sc_e, 0.0, dtype)
        low = min(t for t, _ in spoil) + 1
        assert not out["ok"] and not out["ook"]
        assert out["fb"] == out["ofb"] == low


def test_argument_errors_write_nothing(bls):
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, "single eliminated block")
    ws = bls.QRReductionWorkspace(j, None, torch.float64)
    J = bls.SchurBlockJacobian(j, torch.float64, data=cu(Rw), r=cu(Rr))
    ws.factored.fill_(7.0)
    for bad_sc, lam in ((-sc_e, 0.1), (sc_e, -1.0), (sc_e, float("nan")), (np.full_like(sc_e, np.inf), 0.1)):
        with pytest.raises(bls.ArgumentError):
            bls.reduce_qr(ws, J, cu(bad_sc), lam)
    torch.cuda.synchronize()
    assert bool((ws.factored == 7.0).all())
    with pytest.raises(bls.DimensionMismatch):
        bls.reduce_qr(ws, J, cu(sc_e[:-1]), 0.1)
    with pytest.raises(bls.ArgumentError):
        bls.reduce_qr(bls.QRReductionWorkspace(j, None, torch.float32), J, cu(sc_e), 0.1)


def _qr_scene(bls):
    spec = bls.scenes.scaled_down(bls.scenes.workload("qr_500x100k"), ncams=60, npoints=4000)
    p = bls.scenes.jacobian_problem(spec)
    sc = bls.scenes.Scene(spec)
    bs, el, ptr, idx = sc.description()
    o = orc.QRStructure.from_description(bs, (ptr, idx), np.full(len(ptr) - 1, 2), el)
    return spec, p, o, (bs, el, ptr, idx)


def test_qr_scene_f64(bls):
    """The QR workload's distributions (point Jacobians with singular values log-uniform in [1e-7, 1], damping rows
    sqrt(1e-6) I) scaled down to 60 cameras and 4,000 points, FP64: everything within 1e-11 of the oracle."""
    spec, p, o, _ = _qr_scene(bls)
    check_close(run_both(bls, p.structure, o, p.Rw, p.Rr, p.scaling_e, p.lam, torch.float64), 1e-11)


def test_qr_scene_mixed(bls):
    """The same scene in the mixed form against the FP64 oracle on the FP32-rounded tables. With singular values down
    to 1e-7, the third pivot of a table is at FP32 rounding level (~1e-7 against the damping entry 1e-3), so the
    Householder sign choice (beta = -sign(a) |x|) may differ from the FP64 one: the factored tables are then another
    valid factorisation, equal in magnitude (|F| within 1e-3) but not entrywise. What is unique is checked tightly:
    J~'J~ (both forms), J~'r~ and the diagonal blocks within 1e-6 relative, the back-substituted x_e within 1e-4
    (U's smallest diagonal entries are ~1e-3)."""
    spec, p, o, _ = _qr_scene(bls)
    out = run_both(bls, p.structure, o, p.Rw, p.Rr, p.scaling_e, p.lam, torch.float32)
    check_close(out, {"Sd": 1e-6, "gd": 1e-6, "D": 1e-6, "x_e": 1e-4, "Ss": 1e-6, "gs": 1e-6}, keys=("Sd", "gd", "D", "x_e"))
    assert relerr(np.abs(out["F"]), np.abs(out["oF"])) <= 1e-3


def test_qr_mixed_beats_schur_mixed(bls):
    """On the ill-conditioned QR scene, the mixed QR path's reduced normal equations are closer to the FP64 ones than
    the mixed Schur path's (FP32 E = J_p'J_p squares the condition number the QR path works with): at least 10x."""
    spec, p, o, (bs, el, ptr, idx) = _qr_scene(bls)
    qr = run_both(bls, p.structure, o, p.Rw, p.Rr, p.scaling_e, p.lam, torch.float32)
    hp = bls.scenes.hessian_problem(spec)
    st, pat = hp.structure, hp.pattern
    ost = orc.Structure.from_description(bs, (ptr, idx), el)
    opat = orc.Pattern(ost)
    sc_r, sc_e = np.zeros(st.nr), np.ones(st.ne)     # the QR tables' damping: lambda I on the points only
    ws = bls.SchurReductionWorkspace(st, pat)
    S = torch.zeros(pat.nnz, dtype=torch.float32, device=DEV)
    g = torch.zeros(st.nr, dtype=torch.float64, device=DEV)
    bls.reset_schur_sparse(S, cu(hp.R, torch.float32), None, None, cu(sc_r), p.lam, ws)
    assert bls.reduce_schur_sparse(S, g, cu(hp.b_r), cu(hp.b_e), cu(sc_e), p.lam, st, cu(hp.E, torch.float32), cu(hp.C, torch.float32),
                                   None, None, None, None, ws)
    oS, og = np.zeros(opat.nnz), np.zeros(st.nr)
    orc.reset_schur_sparse(ost, opat, oS, hp.R, sc_r, p.lam)
    assert orc.reduce_schur_sparse(ost, opat, orc.Work(ost, 1), oS, og, hp.b_r, hp.b_e, sc_e, p.lam, hp.E, hp.C)[0]
    err_schur = relerr(S.double().cpu().numpy(), oS)
    err_qr = relerr(qr["Ss"], qr["oSs"])
    print(f"mixed J~'J~ vs FP64: {err_qr:.2e}; mixed Schur S vs FP64: {err_schur:.2e}")
    assert err_qr * 10 <= err_schur, (err_qr, err_schur)


@pytest.mark.parametrize("name", list(QR_FIXTURES))
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_assembly_vs_oracle(bls, name, dtype):
    """H = J'J, b = J'r from the raw tables into the Hessian layout (E, C, R on the pattern and dense, b) against the
    oracle's FP64 assembly of the same stored tables: 1e-13 in FP64; FP32 rounded once (E, C) or per table (R)."""
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, name)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    Rw_s = Rw.astype(npdt)
    pairs = bls.free_block_pairs(j)
    pat = bls.build_schur_pattern(j.schur, pairs)
    opat = orc.Pattern(o.st, pairs)
    ws = bls.QRReductionWorkspace(j, pat, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw_s), r=cu(Rr))
    oE, oC, oR, ob = orc.assemble_hessian(o, Rw_s.astype(np.float64), Rr, opat)
    _, _, oRd, _ = orc.assemble_hessian(o, Rw_s.astype(np.float64), Rr, None)
    tol = 1e-13 if dtype == torch.float64 else 2e-6
    for dense, oRx in ((False, oR), (True, oRd)):
        E, Cd, R, b = bls.assemble_hessian(J, ws, dense=dense)
        assert relerr(E.double().cpu().numpy(), oE) <= tol
        assert relerr(Cd.double().cpu().numpy(), oC) <= tol
        assert relerr(R.double().cpu().numpy(), oRx) <= tol
        assert relerr(b.cpu().numpy(), ob) <= 1e-13


@pytest.mark.parametrize("name", ["bundle adjustment", "free groups", "coupled to all"])   # d_e <= 3 (the Schur path's limit)
def test_assembled_schur_equals_qr_reduction(bls, name):
    """The two elimination paths from one Jacobian on the device: assemble H = J'J, reduce it by the Schur complement
    (R reset from the pattern through the identity map, the eliminated blocks damped by lambda * scaling_e), and the
    QR path's J~'J~ and J~'r~ agree at 1e-10 (the reference's own identity, test/qr_reduction.jl:20-58)."""
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, name)
    lam = 0.3
    pairs = bls.free_block_pairs(j)
    pat = bls.build_schur_pattern(j.schur, pairs)
    qws = bls.QRReductionWorkspace(j, pat, torch.float64)
    J = bls.SchurBlockJacobian(j, torch.float64, data=cu(Rw), r=cu(Rr))
    E, Cd, R, b = bls.assemble_hessian(J, qws)
    st, nr = j.schur, j.schur.nr
    sws = bls.SchurReductionWorkspace(st, pat, r_to_s_map=np.arange(pat.nnz))
    S = torch.zeros(pat.nnz, dtype=torch.float64, device=DEV)
    g = torch.zeros(nr, dtype=torch.float64, device=DEV)
    bls.reset_schur_sparse(S, R, None, None, torch.zeros(nr, dtype=torch.float64, device=DEV), lam, sws)
    assert bls.reduce_schur_sparse(S, g, b[:nr].contiguous(), b[nr:].contiguous(), cu(sc_e), lam, st, E, Cd, None, None, None, None, sws)
    assert bls.reduce_qr(qws, J, cu(sc_e), lam)
    Sq = torch.zeros(pat.nnz, dtype=torch.float64, device=DEV)
    gq = torch.zeros(nr, dtype=torch.float64, device=DEV)
    bls.reduced_normal_sparse(Sq, gq, qws, pat)
    assert relerr(S.cpu().numpy(), Sq.cpu().numpy()) <= 1e-10
    assert relerr(g.cpu().numpy(), gq.cpu().numpy()) <= 1e-10


@pytest.mark.parametrize("name", list(QR_FIXTURES))
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_jacobian_queries_vs_oracle(bls, name, dtype):
    """jtr!, jtj_diag! and jtj_quadform on the raw tables and on the factored ones against the oracle on the same
    stored values (FP64 sums in both, so 1e-13 whatever the storage type)."""
    j, o, Rw, Rr, Jf, rf, sc_e = fixture(bls, name)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    Rw_s = Rw.astype(npdt)
    pat = bls.build_schur_pattern(j.schur, bls.free_block_pairs(j))
    ws = bls.QRReductionWorkspace(j, pat, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw_s), r=cu(Rr))
    assert bls.reduce_qr(ws, J, cu(sc_e), 0.3)
    n = j.schur.nr + j.schur.ne
    v = np.random.default_rng(9).standard_normal(n)
    for src, D, Rv in ((J, Rw_s, Rr), (ws, ws.factored.cpu().numpy(), ws.fres.cpu().numpy())):
        g = bls.jtr(torch.empty(n, dtype=torch.float64, device=DEV), src, ws)
        d = bls.jtj_diag(torch.empty(n, dtype=torch.float64, device=DEV), src, ws)
        qf = bls.jtj_quadform(src, cu(v), ws)
        assert relerr(g.cpu().numpy(), orc.jtr(o, D, Rv)) <= 1e-13
        assert relerr(d.cpu().numpy(), orc.jtr(o, D, None, diag=True)) <= 1e-13
        oq = orc.jtj_quadform(o, D, v)
        assert abs(qf - oq) <= 1e-13 * oq


def test_prepare_scale_bit_identical(bls):
    """prepare_scale! on the device against the oracle, bit for bit: scales from a diagonal over 600 decades with zeros,
    negatives, subnormals and non-finite entries (FP64 and FP32 floors), then the drift rule at two later dampings."""
    rng = np.random.default_rng(12)
    d = np.concatenate([10.0 ** rng.uniform(-300, 300, 4000), [0.0, -2.5, 5e-324, 1e-310, np.inf, -np.inf, np.nan, 1e300]])
    sc = rng.random(len(d))
    for dtype, T in ((torch.float64, "f64"), (torch.float32, "f32")):
        s = torch.zeros(len(d), dtype=torch.float64, device=DEV)
        os_ = np.zeros(len(d))
        assert bls.prepare_scale(s, cu(d), 1e-3, cu(sc), dtype, stale=True)
        orc.prepare_scale(os_, d, 1e-3, sc, T, stale=True)
        assert (s.cpu().numpy() == os_).all()
        for lam in (2e-3, 1e8):
            rec = bls.prepare_scale(s, cu(d), lam, cu(sc), dtype, stale=False)
            orec = orc.prepare_scale(os_, d, lam, sc, T, stale=False)
            assert rec == orec and (s.cpu().numpy() == os_).all()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_bulk_staging_matches_element_staging(bls, dtype):
    """The table kernels stage each table with one bulk (TMA) copy per contiguous span by default; element-wise
    staging (the other mode) must give bit-identical factored tables and residual, and the same J~'J~, J~'r~,
    diagonal blocks and assembled Hessian up to the order of their atomic sums, on the scaled QR scene and on a table
    buffer offset by one element from a 16-byte boundary (which falls back to element staging)."""
    spec, p, o, _ = _qr_scene(bls)
    j = p.structure
    pat = bls.build_schur_pattern(j.schur, bls.free_block_pairs(j))
    nr = j.schur.nr
    outs = []
    for bulk, shift in ((True, 0), (False, 0), (True, 1)):
        ws = bls.QRReductionWorkspace(j, pat, dtype)
        ws.set_staging(bulk)
        raw = torch.zeros(len(p.Rw) + 1, dtype=dtype, device=DEV)
        raw[shift:shift + len(p.Rw)] = cu(p.Rw, dtype)
        J = bls.SchurBlockJacobian(j, dtype, data=raw[shift:shift + len(p.Rw)], r=cu(p.Rr))
        assert bls.reduce_qr(ws, J, cu(p.scaling_e), p.lam)
        S = torch.zeros(pat.nnz, dtype=dtype, device=DEV)
        g = torch.zeros(nr, dtype=torch.float64, device=DEV)
        bls.reduced_normal_sparse(S, g, ws, pat)
        D = torch.zeros(int(j.doffsets[-1]), dtype=dtype, device=DEV)
        bls.reduced_diagonal_blocks(D, ws)
        E, Cd, R, b = bls.assemble_hessian(J, ws)
        outs.append([t.double().cpu().numpy().copy() for t in (ws.factored, ws.fres, S, g, D, E, Cd, R, b)])
    # the factored tables and their residual come from each table's own staged copy: bit-identical; the Gram,
    # diagonal-block and assembly outputs add per-table contributions with atomics, whose order varies from run to run:
    # equal to a few units in the last place
    names = ("factored", "fres", "S", "g", "D", "E", "C", "R", "b")
    tol = 1e-14 if dtype == torch.float64 else 1e-6
    for other in outs[1:]:
        for name, a, b_ in zip(names, outs[0], other):
            if name in ("factored", "fres"):
                assert np.array_equal(a, b_), name
            else:
                assert np.linalg.norm(a - b_) <= tol * np.linalg.norm(a), name
