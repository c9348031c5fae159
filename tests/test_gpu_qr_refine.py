"""Iterative refinement of the QR route (qr_refine): the mixed route (FP32 tables, FP64 reflector arithmetic and
residual) followed by refinement steps whose normal-equation residual d = J'(r - J x) - lambda scaling .* x is FP64
from the raw tables, reduced through the factored tables and solved with the dense Cholesky of
J~'J~ + lambda diag(scaling_r).

On the ill-conditioned QR workload scaled down (point Jacobians with singular values down to 1e-7): the plain mixed
solve leaves a relative normal-equation residual far above FP64 level; refinement brings it to <= 1e-11 and the
solution to within 1e-9 of the FP64 route's refined solution of the same FP32-rounded tables. In FP64 one refinement
step reaches <= 1e-12.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def cu(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t.to(dtype) if dtype is not None else t).to(DEV)


def _route(bls, p, dtype, Rw, sc_r):
    j = p.structure
    nr, ne = j.schur.nr, j.schur.ne
    ws = bls.QRReductionWorkspace(j, None, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw, dtype), r=cu(p.Rr))
    sc_e = cu(p.scaling_e)
    assert bls.reduce_qr(ws, J, sc_e, p.lam)
    S = torch.zeros(nr * nr, dtype=dtype, device=DEV)
    g = torch.zeros(nr, dtype=torch.float64, device=DEV)
    bls.reduced_normal_dense(S, g, ws)
    D = bls.DenseCholesky(nr)
    assert D.factor(S, p.lam, sc_r)
    x = torch.zeros(nr + ne, dtype=torch.float64, device=DEV)
    return ws, J, sc_e, D, x


def test_mixed_route_refined_to_fp64(bls):
    spec = bls.scenes.scaled_down(bls.scenes.workload("qr_500x100k"), ncams=60, npoints=4000)
    p = bls.scenes.jacobian_problem(spec)
    nr = p.structure.schur.nr
    Rw32 = p.Rw.astype(np.float32)
    sc_r = cu(np.ones(nr))
    ws, J, sc_e, D, x = _route(bls, p, torch.float32, Rw32, sc_r)
    plain = bls.qr_refine(x, ws, J, sc_r, sc_e, p.lam, lambda d: D.solve(d), maxit=1)
    x_plain = x.clone()
    res = bls.qr_refine(x, ws, J, sc_r, sc_e, p.lam, lambda d: D.solve(d), tol=1e-11, maxit=6)
    ws64, J64, sc_e64, D64, x64 = _route(bls, p, torch.float64, Rw32.astype(np.float64), sc_r)
    res64 = bls.qr_refine(x64, ws64, J64, sc_r, sc_e64, p.lam, lambda d: D64.solve(d), tol=1e-12, maxit=3)
    print(f"plain mixed {plain.rel_residuals}, refined {res.rel_residuals}, fp64 {res64.rel_residuals}")
    assert res64.converged and res64.steps <= 2
    assert plain.rel_residuals[0] > 1e-9          # the plain mixed solve is far from FP64 level
    assert res.converged, res
    xr, x64r = x.cpu().numpy(), x64.cpu().numpy()
    e_ref = np.linalg.norm(xr - x64r) / np.linalg.norm(x64r)
    e_plain = np.linalg.norm(x_plain.cpu().numpy() - x64r) / np.linalg.norm(x64r)
    print(f"solution vs FP64 route: plain {e_plain:.2e}, refined {e_ref:.2e}")
    assert e_ref <= 1e-9 and e_ref < e_plain


def test_refinement_steps_are_the_block_elimination(bls):
    """The first step from x = 0 is the plain QR-route solve: x_r = (J~'J~ + lam D_r)^-1 J~'r~ and x_e by the
    back-substitution of the factored residual (FP64 route, 1e-10)."""
    spec = bls.scenes.scaled_down(bls.scenes.workload("qr_500x100k"), ncams=30, npoints=1200, seed=7)
    p = bls.scenes.jacobian_problem(spec)
    j = p.structure
    nr, ne = j.schur.nr, j.schur.ne
    sc_r = cu(np.ones(nr))
    ws, J, sc_e, D, x = _route(bls, p, torch.float64, p.Rw, sc_r)
    bls.qr_refine(x, ws, J, sc_r, sc_e, p.lam, lambda d: D.solve(d), maxit=1)
    S = torch.zeros(nr * nr, dtype=torch.float64, device=DEV)
    g = torch.zeros(nr, dtype=torch.float64, device=DEV)
    bls.reduced_normal_dense(S, g, ws)
    xr = D.solve(g)
    xe = torch.zeros(ne, dtype=torch.float64, device=DEV)
    bls.qr_backsubstitute(xe, xr, ws)
    ref = torch.cat([xr, xe]).cpu().numpy()
    assert np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref) <= 1e-10
