"""LSMR on the reduced problem (ext/KrylovExt.jl:25-132) on the device, through the C ABI. As in the reference's test
(test/dampedlinearsolve_qrelimination.jl:235-247, "LSMR on a badly scaled reduced Jacobian equals QR"), the check is
against the direct solution of the same damped least-squares problem, here numpy's lstsq of the written-out
[J~; sqrt(lambda s_r)] and [r~; 0] (reduced_jacobian! of the same factored tables), at rtol 1e-6 in the norm, for
lambda in {0, 1e-8, 1e-4}, with and without a scaling s_r, on the QR fixtures with retained columns scaled over six
orders of magnitude, in FP64 and the mixed form; then the reference's NotPositiveDefinite cases and an itmax stop;
and against the oracle's restatement of the same LSMR on the same written-out problem (stops, iterations, iterates)."""
import numpy as np
import pytest
import torch

from qr_fixtures import QR_FIXTURES, fill_tables

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
CASES = [(0.0, False), (1e-8, False), (1e-4, False), (1e-8, True), (1e-4, True)]


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def scale_retained_columns(j, Rw, scale):
    """Multiply retained scalar column k of every table entry by scale[k] (a badly scaled Jacobian)."""
    st = j.schur
    Rw = Rw.copy()
    for t in range(j.ntables):
        M, off = int(j.table_nrows[t]), int(j.raw_offsets[t])
        for u in range(int(j.table_ptr[t]), int(j.table_ptr[t + 1])):
            r, c0 = int(j.entry_retained[u]), int(j.entry_col[u])
            for k in range(int(st.r_dims[r])):
                Rw[off + (c0 + k) * M: off + (c0 + k + 1) * M] *= scale[int(st.boffsets_r[r]) + k]
    return Rw


def problem(bls, name, seed=5, badly_scaled=True):
    rng = np.random.default_rng(seed)
    fx = QR_FIXTURES[name](rng)
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    j = bls.SchurJacobianStructure.positional(st, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    Rw, Rr, _, _ = fill_tables(j, rng)
    if badly_scaled:
        Rw = scale_retained_columns(j, Rw, 10.0 ** rng.uniform(-3, 3, j.schur.nr))
    return j, Rw, Rr, 0.5 + rng.random(j.schur.ne), 0.5 + rng.random(j.schur.nr)


def direct(bls, ws, lam, s_r):
    """lstsq of [J~; sqrt(lam s_r)] x = [r~; 0] from the written-out reduced problem (FP64 arithmetic)."""
    m, nr = bls.reduced_nrows(ws.structure), ws.structure.schur.nr
    Jt = torch.zeros(m * nr, dtype=ws.dtype, device=DEV)
    rt = torch.zeros(m, dtype=torch.float64, device=DEV)
    bls.reduced_jacobian(Jt, rt, ws)
    A = Jt.cpu().double().numpy().reshape(m, nr, order="F")
    d = np.sqrt(lam * (np.ones(nr) if s_r is None else s_r))
    Aa = np.vstack([A, np.diag(d)])
    return np.linalg.lstsq(Aa, np.concatenate([rt.cpu().numpy(), np.zeros(nr)]), rcond=None)[0], Aa


def close(x, ref, rtol):
    return np.linalg.norm(x - ref) <= rtol * max(np.linalg.norm(x), np.linalg.norm(ref))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
@pytest.mark.parametrize("name", list(QR_FIXTURES))
def test_lsmr_equals_the_direct_solution(bls, name, dtype):
    j, Rw, Rr, sc_e, s_r = problem(bls, name)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    ws = bls.QRReductionWorkspace(j, None, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw.astype(npdt)), r=cu(Rr))
    m, nr = bls.reduced_nrows(j), j.schur.nr
    for lam, scaled in CASES:
        assert bls.reduce_qr(ws, J, cu(sc_e), lam)
        s = s_r if scaled else None
        ref, Aa = direct(bls, ws, lam, s)
        x = torch.full((nr,), float("nan"), dtype=torch.float64, device=DEV)
        if lam == 0 and m < nr:
            assert not bls.lsmr_reduced(x, ws, lam, None if s is None else cu(s)).solved   # rank deficient: NotPositiveDefinite
            continue
        if lam == 0 and np.linalg.matrix_rank(Aa) < nr:
            continue
        # FP64 vectors with tolerances far below the reference's: the direct solution to 1e-6
        res = bls.lsmr_reduced(x, ws, lam, None if s is None else cu(s), atol=1e-12, btol=1e-12, conlim=1e14)
        assert res.solved and res.istop in (1, 2, 4, 5), (lam, scaled, res)
        assert close(x.cpu().numpy(), ref, 1e-6), (lam, scaled, res)
        # the reference's own tolerances (sqrt(eps(T)), conlim 1/sqrt(eps(T))): solved, and within the reference's
        # bound for LSMR in single precision (test/precision.jl:107) for the mixed form
        x.fill_(float("nan"))
        res = bls.lsmr_reduced(x, ws, lam, None if s is None else cu(s))
        if dtype == torch.float64:
            assert res.solved, (lam, scaled, res)
            assert close(x.cpu().numpy(), ref, 1e-6), (lam, scaled, res)
        elif res.solved:
            tol = np.sqrt(np.finfo(np.float32).eps) * np.linalg.cond(Aa)
            assert close(x.cpu().numpy(), ref, tol), (lam, scaled, res)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_lsmr_on_a_scene(bls, dtype):
    spec = bls.scenes.scaled_down(bls.scenes.workload("qr_500x100k"), ncams=30, npoints=600)
    p = bls.scenes.jacobian_problem(spec)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    ws = bls.QRReductionWorkspace(p.structure, None, dtype)
    J = bls.SchurBlockJacobian(p.structure, dtype, data=cu(p.Rw.astype(npdt)), r=cu(p.Rr))
    nr = p.structure.schur.nr
    s_r = 0.5 + np.random.default_rng(4).random(nr)
    for lam in (1e-6, p.lam):
        assert bls.reduce_qr(ws, J, cu(p.scaling_e), lam)
        ref, _ = direct(bls, ws, lam, s_r)
        x = torch.zeros(nr, dtype=torch.float64, device=DEV)
        res = bls.lsmr_reduced(x, ws, lam, cu(s_r), atol=1e-12, btol=1e-12, conlim=1e14)
        assert res.solved and close(x.cpu().numpy(), ref, 1e-6), (lam, res)


def test_not_positive_definite_and_itmax(bls):
    j, Rw, Rr, sc_e, s_r = problem(bls, "bundle adjustment", badly_scaled=False)
    ws = bls.QRReductionWorkspace(j, None, torch.float64)
    nr = j.schur.nr
    x = torch.zeros(nr, dtype=torch.float64, device=DEV)
    # a retained block whose columns are all zero: its diagonal block of J~'J~ is singular without damping
    Rz = scale_retained_columns(j, Rw, np.where(np.arange(nr) < 6, 0.0, 1.0))
    J = bls.SchurBlockJacobian(j, torch.float64, data=cu(Rz), r=cu(Rr))
    assert bls.reduce_qr(ws, J, cu(sc_e), 0.0)
    assert not bls.lsmr_reduced(x, ws, 0.0).solved
    assert bls.reduce_qr(ws, J, cu(sc_e), 1e-4)
    assert bls.lsmr_reduced(x, ws, 1e-4, atol=1e-12, btol=1e-12, conlim=1e14).solved   # damping makes it definite
    # a non-finite r~ (a non-finite Jacobian is already refused by reduce_qr; the factored residual is poisoned here)
    J = bls.SchurBlockJacobian(j, torch.float64, data=cu(Rw), r=cu(Rr))
    assert bls.reduce_qr(ws, J, cu(sc_e), 1e-4)
    ws.fres.fill_(float("nan"))
    assert not bls.lsmr_reduced(x, ws, 1e-4).solved
    # itmax
    assert bls.reduce_qr(ws, J, cu(sc_e), 1e-4)
    res = bls.lsmr_reduced(x, ws, 1e-4, atol=0.0, btol=0.0, conlim=0.0, itmax=2)
    assert not res.solved and res.istop == 7 and res.iterations == 2
    x.fill_(1.0)
    res = bls.lsmr_reduced(x, ws, 1e-4, itmax=0)
    assert not res.solved and res.istop == 7 and res.iterations == 0 and not bool(x.any())
    with pytest.raises(bls.DimensionMismatch):
        bls.lsmr_reduced(torch.zeros(nr + 1, dtype=torch.float64, device=DEV), ws, 1e-4)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
@pytest.mark.parametrize("name", list(QR_FIXTURES))
def test_lsmr_against_the_oracle(bls, name, dtype):
    """The device's LSMR against the oracle's restatement on the same written-out J~ and r~ (the device's own factored
    tables), at the reference's tolerances for the storage type: the same stop (istop), iteration counts within one,
    solutions within 1e-6 (at equal iteration counts)."""
    import oracle as orc
    j, Rw, Rr, sc_e, s_r = problem(bls, name)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    ws = bls.QRReductionWorkspace(j, None, dtype)
    J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw.astype(npdt)), r=cu(Rr))
    m, nr = bls.reduced_nrows(j), j.schur.nr
    tol = float(np.sqrt(np.finfo(npdt).eps))
    for lam, scaled in CASES:
        if lam == 0 and m < nr:
            continue
        assert bls.reduce_qr(ws, J, cu(sc_e), lam)
        s = s_r if scaled else None
        Jt = torch.zeros(m * nr, dtype=dtype, device=DEV)
        rt = torch.zeros(m, dtype=torch.float64, device=DEV)
        bls.reduced_jacobian(Jt, rt, ws)
        A = Jt.cpu().double().numpy().reshape(m, nr, order="F")
        xo, status, it, istop = orc.lsmr_reduced(A, rt.cpu().numpy(), j.schur.r_dims, lam, s, atol=tol, btol=tol, conlim=1 / tol)
        x = torch.zeros(nr, dtype=torch.float64, device=DEV)
        res = bls.lsmr_reduced(x, ws, lam, None if s is None else cu(s))
        assert res.solved == (status == "ok"), (lam, scaled, res, status)
        assert abs(res.iterations - it) <= 1, (lam, scaled, res.iterations, it)
        if res.iterations == it:
            assert res.istop == istop
        if res.solved:   # the same iterate to rounding; one iteration apart, within the stopping tolerance's reach
            assert close(x.cpu().numpy(), xo, 1e-6 if res.iterations == it else 100 * tol), (lam, scaled, res)
