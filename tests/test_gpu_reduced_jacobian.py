"""The reduced problem written out on the device (src/qr_reduced.jl:227-370), through the C ABI, against the oracle's
restatement applied to the device's own factored tables (a gather: bit-exact): reduced_residual! (r~),
reduced_jacobian! dense (J~ column-major) and sparse (J~ on build_reduced_jacobian_pattern's CSC, every stored entry
written), in FP64 and the mixed form's FP32, on the reference's QR fixtures and a scaled QR scene; then the reference's
rejections (test/schur_qr.jl:256-269): a wrong size or residual length (DimensionMismatch), columns of the wrong height
or a run that starts at the wrong row (ArgumentError), each before anything is written."""
import numpy as np
import pytest
import torch

import oracle as orc
from qr_fixtures import QR_FIXTURES, fill_tables

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def cu(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).to(DEV)


def _fixture(bls, name, seed=5):
    rng = np.random.default_rng(seed)
    fx = QR_FIXTURES[name](rng)
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    ost = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    j = bls.SchurJacobianStructure.positional(st, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    o = orc.QRStructure.positional(ost, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    Rw, Rr, _, _ = fill_tables(j, rng)
    return j, o, Rw, Rr, 0.5 + rng.random(j.schur.ne)


def _check(bls, j, o, Rw, Rr, sc_e, dtype, lam=0.3):
    npdt = np.float32 if dtype == torch.float32 else np.float64
    ws = bls.QRReductionWorkspace(j, None, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw.astype(npdt)), r=cu(Rr))
    assert bls.reduce_qr(ws, J, cu(sc_e), lam)
    F = ws.factored.cpu().numpy()
    Fr = ws.fres.cpu().numpy()
    m, nr = bls.reduced_nrows(j), j.schur.nr
    # the oracle's gather of the same factored tables
    oJt, ort = np.zeros(m * nr, npdt), np.zeros(m)
    orc.reduced_jacobian_dense(o, oJt, m, nr, ort, F, Fr)
    colptr, rowval = bls.build_reduced_jacobian_pattern(j)
    onz, ort2 = np.full(len(rowval), np.nan, npdt), np.full(m, np.nan)
    orc.reduced_jacobian_sparse(o, m, nr, colptr, rowval, onz, ort2, F, Fr)
    # the device
    rt = torch.full((m,), float("nan"), dtype=torch.float64, device=DEV)
    assert np.array_equal(bls.reduced_residual(rt, ws).cpu().numpy(), ort)
    Jt = torch.full((m * nr,), float("nan"), dtype=dtype, device=DEV)
    rt.fill_(float("nan"))
    bls.reduced_jacobian(Jt, rt, ws)
    assert np.array_equal(Jt.cpu().numpy(), oJt) and np.array_equal(rt.cpu().numpy(), ort)
    nz = torch.full((len(rowval),), float("nan"), dtype=dtype, device=DEV)
    rt.fill_(float("nan"))
    bls.reduced_jacobian_sparse(nz, colptr, rowval, rt, ws)
    nzh = nz.cpu().numpy()
    assert not np.isnan(nzh).any()                     # every stored entry is written
    assert np.array_equal(nzh, onz) and np.array_equal(rt.cpu().numpy(), ort)
    dense = np.zeros((m, nr), npdt)
    for c in range(nr):
        dense[rowval[colptr[c]:colptr[c + 1]], c] = nzh[colptr[c]:colptr[c + 1]]
    assert np.array_equal(dense, Jt.cpu().numpy().reshape(m, nr, order="F"))   # identical, not just close
    # J~'J~ and J~'r~ from the written-out problem agree with reduced_normal_dense
    if dtype == torch.float64:
        S = torch.zeros(nr * nr, dtype=dtype, device=DEV)
        g = torch.zeros(nr, dtype=torch.float64, device=DEV)
        bls.reduced_normal_dense(S, g, ws)
        A = dense
        Su = S.cpu().numpy().reshape(nr, nr, order="F")
        scale = max(np.abs(Su).max(), 1e-300)
        assert np.abs(np.triu(A.T @ A) - np.triu(Su)).max() <= 1e-12 * scale
        assert np.abs(A.T @ ort - g.cpu().numpy()).max() <= 1e-12 * max(np.abs(g.cpu().numpy()).max(), 1e-300)
    return ws, colptr, rowval, m, nr


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
@pytest.mark.parametrize("name", list(QR_FIXTURES))
def test_reduced_problem_fixtures(bls, name, dtype):
    j, o, Rw, Rr, sc_e = _fixture(bls, name)
    _check(bls, j, o, Rw, Rr, sc_e, dtype)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_reduced_problem_scene(bls, dtype):
    spec = bls.scenes.scaled_down(bls.scenes.workload("qr_500x100k"), ncams=30, npoints=600)
    p = bls.scenes.jacobian_problem(spec)
    sc = bls.scenes.Scene(spec)
    bs, el, ptr, idx = sc.description()
    o = orc.QRStructure.from_description(bs, (ptr, idx), np.full(len(ptr) - 1, 2), el)
    _check(bls, p.structure, o, p.Rw, p.Rr, p.scaling_e, dtype, lam=p.lam)


def test_rejections_before_any_write(bls):
    j, o, Rw, Rr, sc_e = _fixture(bls, "bundle adjustment")
    ws, colptr, rowval, m, nr = _check(bls, j, o, Rw, Rr, sc_e, torch.float64)
    nz = torch.full((len(rowval),), 7.0, dtype=torch.float64, device=DEV)
    rt = torch.full((m,), 7.0, dtype=torch.float64, device=DEV)
    # sizes: one column too many, one residual entry too many
    with pytest.raises(bls.DimensionMismatch):
        bls.reduced_jacobian_sparse(nz, np.concatenate([colptr, colptr[-1:]]), rowval, rt, ws)
    with pytest.raises(bls.DimensionMismatch):
        bls.reduced_jacobian_sparse(nz, colptr, rowval, torch.zeros(m + 1, dtype=torch.float64, device=DEV), ws)
    with pytest.raises(bls.DimensionMismatch):
        bls.reduced_jacobian(torch.zeros((m + 1) * nr, dtype=torch.float64, device=DEV), rt, ws)
    with pytest.raises(bls.DimensionMismatch):
        bls.reduced_residual(torch.zeros(m + 1, dtype=torch.float64, device=DEV), ws)
    # heights: a full pattern
    full_cp = np.arange(nr + 1, dtype=np.int64) * m
    full_rv = np.tile(np.arange(m, dtype=np.int64), nr)
    if len(rowval) < m * nr:
        with pytest.raises(bls.ArgumentError, match="entries, expected"):
            bls.reduced_jacobian_sparse(torch.zeros(m * nr, dtype=torch.float64, device=DEV), full_cp, full_rv, rt, ws)
    # a run that starts at the wrong row
    c = int(np.flatnonzero(np.diff(colptr) > 0)[0])
    bad = rowval.copy()
    q = colptr[c]
    bad[q] = 0 if bad[q] == m - 1 else m - 1
    with pytest.raises(bls.ArgumentError, match="stores row"):
        bls.reduced_jacobian_sparse(nz, colptr, bad, rt, ws)
    assert bool((nz == 7.0).all()) and bool((rt == 7.0).all())


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
@pytest.mark.parametrize("name", list(QR_FIXTURES))
def test_reduced_mul_tmul(bls, name, dtype):
    """reduced_mul! / reduced_tmul! (src/qr_reduced.jl:159-223): J~ v and J~' w from the factored tables, against the
    oracle on the device's own tables (FP64 accumulation; J~ v in the reference's order per row, the runs' dot products
    of J~' w as warp sums: within 1e-14 relative), and J~'(J~ v) against S v with S = J~'J~ from reduced_normal_dense."""
    j, o, Rw, Rr, sc_e = _fixture(bls, name)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    ws = bls.QRReductionWorkspace(j, None, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw.astype(npdt)), r=cu(Rr))
    assert bls.reduce_qr(ws, J, cu(sc_e), 0.3)
    F = ws.factored.cpu().numpy()
    m, nr = bls.reduced_nrows(j), j.schur.nr
    rng = np.random.default_rng(9)
    v, w = rng.standard_normal(nr), rng.standard_normal(m)
    y = bls.reduced_mul(torch.full((m,), float("nan"), dtype=torch.float64, device=DEV), ws, cu(v)).cpu().numpy()
    g = bls.reduced_tmul(torch.full((nr,), float("nan"), dtype=torch.float64, device=DEV), ws, cu(w)).cpu().numpy()
    oy, og = np.zeros(m), np.zeros(nr)
    orc.reduced_mul(o, oy, v, F)
    orc.reduced_tmul(o, og, w, F)
    assert np.abs(y - oy).max() <= 1e-14 * max(np.abs(oy).max(), 1e-300)
    assert np.abs(g - og).max() <= 1e-14 * max(np.abs(og).max(), 1e-300)
    if dtype == torch.float64:
        S = torch.zeros(nr * nr, dtype=dtype, device=DEV)
        bls.reduced_normal_dense(S, torch.zeros(nr, dtype=torch.float64, device=DEV), ws)
        Su = S.cpu().numpy().reshape(nr, nr, order="F")
        Sf = np.triu(Su) + np.triu(Su, 1).T
        tt = bls.reduced_tmul(torch.zeros(nr, dtype=torch.float64, device=DEV), ws, cu(y)).cpu().numpy()
        assert np.abs(tt - Sf @ v).max() <= 1e-12 * max(np.abs(Sf @ v).max(), 1e-300)
    with pytest.raises(bls.DimensionMismatch):
        bls.reduced_mul(torch.zeros(m + 1, dtype=torch.float64, device=DEV), ws, cu(v))
    with pytest.raises(bls.DimensionMismatch):
        bls.reduced_tmul(torch.zeros(nr, dtype=torch.float64, device=DEV), ws, cu(np.zeros(m + 1)))
