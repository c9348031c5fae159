"""Dense reduced solve on the device (Cholesky of the dense S that reduce_schur_dense! produces, then x = S^-1 g)
against a dense FP64 solve on the host of the same stored S (the oracle's reduction for the scene), within 1e-10;
random SPD systems across tile boundaries; the first non-positive pivot reported as its 1-based column."""
import numpy as np
import pytest
import torch

import oracle as orc

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def first_bad_pivot(A):
    """The 1-based column of the first pivot of A's unblocked Cholesky that is not positive, 0 if none."""
    A = np.array(A, np.float64)
    n = A.shape[0]
    for j in range(n):
        d = A[j, j] - A[j, :j] @ A[j, :j]
        if not (d > 0) or not np.isfinite(d):
            return j + 1
        A[j, j] = np.sqrt(d)
        A[j + 1:, j] = (A[j + 1:, j] - A[j + 1:, :j] @ A[j, :j]) / A[j, j]
    return 0


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_dense_scene_solve(bls, dtype):
    spec = bls.scenes.workload("dense_50x2000")
    p = bls.scenes.hessian_problem(spec, dense=True)
    st = p.structure
    nr = st.nr
    cu = lambda a, t=dtype: torch.from_numpy(np.ascontiguousarray(a)).to(device=DEV, dtype=t)
    ws = bls.SchurReductionWorkspace(st, None)
    S = torch.zeros(nr * nr, dtype=dtype, device=DEV)
    g = torch.zeros(nr, dtype=torch.float64, device=DEV)
    bls.reset_schur_dense(S, cu(p.R), cu(p.scaling_r, torch.float64), p.lam, ws)
    assert bls.reduce_schur_dense(S, g, cu(p.b_r, torch.float64), cu(p.b_e, torch.float64), cu(p.scaling_e, torch.float64), p.lam, st,
                                  cu(p.E), cu(p.C), ws)
    A = S.double().cpu().numpy().reshape(nr, nr, order="F")
    A = np.triu(A) + np.triu(A, 1).T
    x_ref = np.linalg.solve(A, g.cpu().numpy())
    D = bls.DenseCholesky(nr)
    assert D.factor(S) and D.failed_column == 0
    x = D.solve(g)
    assert relerr(x.cpu().numpy(), x_ref) <= 1e-10
    # a second solve from the same factorisation, another right-hand side
    g2 = torch.from_numpy(np.random.default_rng(3).standard_normal(nr)).to(DEV)
    assert relerr(D.solve(g2).cpu().numpy(), np.linalg.solve(A, g2.cpu().numpy())) <= 1e-10


# sizes on both sides of the 64-column panels and tiles, and two large systems (about 80 and 100 panels)
@pytest.mark.parametrize("n", [1, 7, 32, 33, 63, 64, 65, 100, 127, 128, 129, 517, 5200, 6500])
def test_random_spd_across_tiles(bls, n):
    rng = np.random.default_rng(n)
    B = rng.standard_normal((n, n))
    A = B @ B.T + n * np.eye(n)
    Su = np.triu(A) + np.tril(rng.standard_normal((n, n)), -1)   # only the upper triangle is read
    D = bls.DenseCholesky(n)
    assert D.factor(torch.from_numpy(Su.ravel(order="F")).to(DEV))
    g = rng.standard_normal(n)
    x = D.solve(torch.from_numpy(g).to(DEV))
    assert relerr(x.cpu().numpy(), np.linalg.solve(A, g)) <= 1e-10


def test_not_positive_definite_reports_column(bls):
    rng = np.random.default_rng(8)
    n = 100
    B = rng.standard_normal((n, n))
    A = B @ B.T + n * np.eye(n)
    A[57, 57] = -1e3
    col = first_bad_pivot(A)
    assert col > 0
    D = bls.DenseCholesky(n)
    assert not D.factor(torch.from_numpy(A.ravel(order="F")).to(DEV))
    assert D.failed_column == col
    with pytest.raises(bls.ArgumentError):
        D.solve(torch.zeros(n, dtype=torch.float64, device=DEV))


@pytest.mark.parametrize("n", [200, 3000])
def test_one_solver_many_systems(bls, n):
    """One solver reused (its factorisation and solve are replayed from captured graphs): a system, a system that is
    not positive definite (reported; the solver then holds no factorisation), another system in FP32 storage, each
    against a host solve; solves with x aliasing g."""
    rng = np.random.default_rng(n)
    D = bls.DenseCholesky(n)
    for trial, dt in enumerate([torch.float64, None, torch.float32]):
        B = rng.standard_normal((n, n))
        A = B @ B.T + n * np.eye(n)
        if dt is None:   # a pivot in the third panel (or the last column) that is not positive
            j = min(150, n - 1)
            A[j, j] = -1.0
            assert not D.factor(torch.from_numpy(A.ravel(order="F")).to(DEV))
            assert D.failed_column == first_bad_pivot(A)
            with pytest.raises(bls.ArgumentError):
                D.solve(torch.zeros(n, dtype=torch.float64, device=DEV))
            continue
        S = torch.from_numpy(A.ravel(order="F")).to(DEV, dt)
        As = S.double().cpu().numpy().reshape(n, n, order="F")   # the stored values (FP32-rounded for dt=float32)
        assert D.factor(S) and D.failed_column == 0
        for k in range(2):
            g = rng.standard_normal(n)
            gd = torch.from_numpy(g).to(DEV)
            x = D.solve(gd, gd if k == 1 else None)   # the second solve in place
            assert relerr(x.cpu().numpy(), np.linalg.solve(As, g)) <= 1e-10, (trial, k)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
@pytest.mark.parametrize("name", ["bundle adjustment", "mixed dimensions", "free groups"])
def test_qr_route_damped_normal_equations(bls, name, dtype):
    """The QR route's dense reduced solve on the device (src/qr_linear_systems.jl:315-322): reduce_qr, J~'J~ and J~'r~
    by reduced_normal_dense, then the Cholesky of J~'J~ + lambda diag(s_r) and the solve; against a host solve of the
    same stored J~'J~ damped on the host, within 1e-10. lambda must be finite and non-negative."""
    from qr_fixtures import QR_FIXTURES, fill_tables
    rng = np.random.default_rng(11)
    fx = QR_FIXTURES[name](rng)
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    j = bls.SchurJacobianStructure.positional(st, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    Rw, Rr, _, _ = fill_tables(j, rng)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    ws = bls.QRReductionWorkspace(j, None, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=torch.from_numpy(Rw.astype(npdt)).to(DEV), r=torch.from_numpy(Rr).to(DEV))
    lam = 1e-3
    assert bls.reduce_qr(ws, J, torch.from_numpy(0.5 + rng.random(j.schur.ne)).to(DEV), lam)
    nr = j.schur.nr
    S = torch.zeros(nr * nr, dtype=dtype, device=DEV)
    g = torch.zeros(nr, dtype=torch.float64, device=DEV)
    bls.reduced_normal_dense(S, g, ws)
    s_r = 0.5 + rng.random(nr)
    A = S.double().cpu().numpy().reshape(nr, nr, order="F")
    A = np.triu(A) + np.triu(A, 1).T + np.diag(lam * s_r)
    D = bls.DenseCholesky(nr)
    sr = torch.from_numpy(s_r).to(DEV)
    assert D.factor(S, lam, sr) and D.failed_column == 0
    x = D.solve(g)
    assert relerr(x.cpu().numpy(), np.linalg.solve(A, g.cpu().numpy())) <= 1e-10
    for bad in (-1e-3, float("nan"), float("inf")):
        with pytest.raises(bls.ArgumentError):
            D.factor(S, bad, sr)
