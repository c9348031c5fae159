"""Device block-Jacobi, y = S x and PCG on the reduced system, through the C ABI.

Block-Jacobi (src/diagonal_blocks.jl:6-61): factor and solve against the oracle at 1e-13 relative on random SPD blocks
of several sizes, and the lowest non-positive-definite block. y = S x against the dense symmetric matrix built from
the same upper storage (1e-13 FP64; FP32 storage with FP64 products at 1e-13 of the same FP32 values). PCG has no
counterpart in the reference: its parity is unpinned and it is judged by the FP64 residual ||g - S x|| / ||g|| <= tol
computed here on the host from the dense matrix, and against the oracle's PCG (the same algorithm on the CPU) and a
dense solve.
"""
import numpy as np
import pytest
import torch

import oracle as orc
from fixtures import csc_to_dense_upper

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


def reduced_system(bls, name="pcg_10000x1M", ncams=120, npoints=6000, seed=None):
    """A scaled-down scene reduced on the device in FP64: (structure, pattern, S (FP64 numpy), g)."""
    spec = bls.scenes.scaled_down(bls.scenes.workload(name), ncams=ncams, npoints=npoints, seed=seed)
    p = bls.scenes.hessian_problem(spec)
    st, pat = p.structure, p.pattern
    ws = bls.SchurReductionWorkspace(st, pat)
    S = torch.zeros(pat.nnz, dtype=torch.float64, device=DEV)
    g = torch.zeros(st.nr, dtype=torch.float64, device=DEV)
    bls.reset_schur_sparse(S, cu(p.R), None, None, cu(p.scaling_r), p.lam, ws)
    assert bls.reduce_schur_sparse(S, g, cu(p.b_r), cu(p.b_e), cu(p.scaling_e), p.lam, st, cu(p.E), cu(p.C), None, None, None, None, ws)
    return st, pat, S.cpu().numpy(), g.cpu().numpy()


def test_block_jacobi_vs_oracle(bls):
    rng = np.random.default_rng(3)
    dims = np.array([6, 3, 9, 1, 6, 2, 16, 6], np.int64)
    blocks = []
    for d in dims:
        A = rng.standard_normal((d, d))
        blocks.append((A @ A.T + d * np.eye(d)).ravel(order="F"))
    D0 = np.concatenate(blocks)
    bj = bls.BlockJacobi(dims)
    for dt in (torch.float64, torch.float32):
        D = cu(D0, dt)
        assert bls.factor_diagonal_blocks(D, bj)
        oD = D0.astype(np.float64 if dt == torch.float64 else np.float32).copy()
        assert orc.factor_diagonal_blocks(oD, dims)
        assert relerr(D.cpu().numpy(), oD) <= (1e-13 if dt == torch.float64 else 1e-6)
        x = rng.standard_normal(int(dims.sum()))
        y = torch.empty(len(x), dtype=torch.float64, device=DEV)
        bls.solve_diagonal_blocks(y, D, bj, cu(x))
        oy = np.zeros(len(x))
        orc.solve_diagonal_blocks(oy, oD, dims, x)
        assert relerr(y.cpu().numpy(), oy) <= (1e-13 if dt == torch.float64 else 1e-6)
        # in place (y is x)
        xt = cu(x)
        bls.solve_diagonal_blocks(xt, D, bj, xt)
        assert relerr(xt.cpu().numpy(), oy) <= (1e-13 if dt == torch.float64 else 1e-6)
    # blocks 3 and 6 (0-based 2 and 5) not positive definite: the lowest is reported
    bad = D0.copy()
    off = np.concatenate([[0], np.cumsum(dims ** 2)])
    for b in (5, 2):
        bad[off[b]] = -1.0
    D = cu(bad)
    assert not bls.factor_diagonal_blocks(D, bj) and bj.failed_block == 3
    bad[off[2]] = np.nan
    assert not bls.factor_diagonal_blocks(cu(bad), bj) and bj.failed_block == 3


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_spmv_and_diagonal_blocks(bls, dtype):
    st, pat, S, g = reduced_system(bls, "sparse_1000x200k", ncams=80, npoints=3000)
    Sd = S.astype(np.float32).astype(np.float64) if dtype == torch.float32 else S
    A = csc_to_dense_upper(st.nr, pat.S_colptr, pat.S_rowval, Sd)
    ws = bls.PCGWorkspace(st, pat)
    x = np.random.default_rng(1).standard_normal(st.nr)
    y = ws.spmv(cu(S, dtype), cu(x))
    assert relerr(y.cpu().numpy(), A @ x) <= 1e-13
    D = ws.diagonal_blocks(cu(S, dtype)).cpu().numpy()
    o = 0
    for r in range(st.nrblocks):
        d, b = int(st.r_dims[r]), int(st.boffsets_r[r])
        np.testing.assert_array_equal(D[o:o + d * d].reshape(d, d, order="F"), A[b:b + d, b:b + d])
        o += d * d


@pytest.mark.parametrize("name", ["pcg_10000x1M", "sparse_1000x200k"])
@pytest.mark.parametrize("graph", [True, False], ids=["graph", "direct"])
def test_pcg_converges(bls, name, graph):
    st, pat, S, g = reduced_system(bls, name)
    A = csc_to_dense_upper(st.nr, pat.S_colptr, pat.S_rowval, S)
    ws = bls.PCGWorkspace(st, pat)
    x, res = ws.solve(cu(S), cu(g), tol=1e-8, graph=graph)
    xh = x.cpu().numpy()
    true_rel = np.linalg.norm(g - A @ xh) / np.linalg.norm(g)
    assert res.converged and res.iterations > 0
    assert true_rel <= 1e-8 and abs(true_rel - res.rel_residual) <= 1e-3 * max(true_rel, 1e-12)
    # the oracle's PCG, same algorithm on the CPU: same iteration count up to rounding, same answer
    ost, opat = orc.Structure.positional(st.r_dims, st.e_dims, [st.entry_retained[st.eliminated_ptr[e]:st.eliminated_ptr[e + 1]]
                                                                  for e in range(st.neblocks)]), None
    opat = orc.Pattern(ost)
    ox = np.zeros(st.nr)
    rc, oit, orel = orc.pcg_solve(ost, opat, S, g, ox, 1e-8)
    assert rc == 0 and abs(oit - res.iterations) <= 2
    xd = np.linalg.solve(A, g)
    assert relerr(xh, xd) <= 1e-5 and relerr(ox, xd) <= 1e-5


def test_pcg_mixed_storage(bls):
    """S stored in FP32 (the mixed reduction's output): the FP64 residual against that FP32 S reaches 1e-8."""
    st, pat, S, g = reduced_system(bls)
    S32 = S.astype(np.float32)
    A = csc_to_dense_upper(st.nr, pat.S_colptr, pat.S_rowval, S32.astype(np.float64))
    ws = bls.PCGWorkspace(st, pat)
    x, res = ws.solve(cu(S32), cu(g), tol=1e-8)
    assert res.converged
    assert np.linalg.norm(g - A @ x.cpu().numpy()) / np.linalg.norm(g) <= 1e-8


def test_pcg_edge_cases(bls):
    st, pat, S, g = reduced_system(bls, ncams=60, npoints=2500)
    ws = bls.PCGWorkspace(st, pat)
    A = csc_to_dense_upper(st.nr, pat.S_colptr, pat.S_rowval, S)
    # warm start from the solution: converged in zero iterations
    xd = np.linalg.solve(A, g)
    x, res = ws.solve(cu(S), cu(g), cu(xd), tol=1e-8)
    assert res.converged and res.iterations == 0
    # g = 0: x = 0
    x, res = ws.solve(cu(S), torch.zeros(st.nr, dtype=torch.float64, device=DEV), cu(np.ones(st.nr)))
    assert res.converged and float(x.abs().max()) == 0.0
    # an iteration limit below what is needed
    x, res = ws.solve(cu(S), cu(g), tol=1e-14, maxit=2)
    assert not res.converged and res.iterations == 2
    # a diagonal block that is not positive definite
    Sb = S.copy()
    Sb[pat.diag_inds[6 * 3]] = -1.0
    x, res = ws.solve(cu(Sb), cu(g))
    assert not res.converged and res.failed_block == 4 and res.iterations == 0
    with pytest.raises(bls.ArgumentError):
        ws.solve(cu(S), cu(g), tol=0.0)


@pytest.mark.parametrize("name,ncams,npoints", [("pcg_10000x1M", 120, 6000), ("sparse_1000x200k", 100, 6000)])
def test_refined_mixed_solve_reaches_fp64_solution(bls, name, ncams, npoints):
    """The mixed (FP32) reduction solved with iterative refinement against the FP64 reduced operator: the solution is
    within 1e-10 of the exact solution of the FP64 oracle's reduced system on the same stored inputs, where PCG on the
    FP32 S alone stops at the FP32 reduction's own error. The operator itself matches the oracle's S at 1e-12."""
    spec = bls.scenes.scaled_down(bls.scenes.workload(name), ncams=ncams, npoints=npoints)
    p = bls.scenes.hessian_problem(spec)
    st, pat = p.structure, p.pattern
    E32, C32, R32 = (a.astype(np.float32) for a in (p.E, p.C, p.R))
    # oracle: FP64 reduction of the FP32-stored values, solved densely
    sc = bls.scenes.Scene(spec)
    bs, el, ptr, idx = sc.description()
    ost = orc.Structure.from_description(bs, (ptr, idx), el)
    opat = orc.Pattern(ost)
    oS, og = np.zeros(opat.nnz), np.zeros(ost.nr)
    orc.reset_schur_sparse(ost, opat, oS, R32.astype(np.float64), p.scaling_r, p.lam)
    ook, _ = orc.reduce_schur_sparse(ost, opat, orc.Work(ost, 1), oS, og, p.b_r, p.b_e, p.scaling_e, p.lam, E32.astype(np.float64),
                                     C32.astype(np.float64))
    assert ook
    Sd = csc_to_dense_upper(st.nr, pat.S_colptr, pat.S_rowval, oS)
    x_star = np.linalg.solve(Sd, og)
    # device: mixed reduction, R on the pattern, refined solve
    ws = bls.SchurReductionWorkspace(st, pat)
    S = torch.zeros(pat.nnz, dtype=torch.float32, device=DEV)
    S0 = torch.zeros(pat.nnz, dtype=torch.float32, device=DEV)
    g = torch.zeros(st.nr, dtype=torch.float64, device=DEV)
    scr, C = cu(p.scaling_r), cu(C32)
    bls.reset_schur_sparse(S0, cu(R32), None, None, scr, 0.0, ws)
    bls.reset_schur_sparse(S, cu(R32), None, None, scr, p.lam, ws)
    assert bls.reduce_schur_sparse(S, g, cu(p.b_r), cu(p.b_e), cu(p.scaling_e), p.lam, st, cu(E32), C, None, None, None, None, ws)
    # the FP64 operator against the oracle's S
    xr = np.random.default_rng(1).standard_normal(st.nr)
    pcg = bls.PCGWorkspace(st, pat)
    y0 = pcg.spmv(S0, cu(xr))
    y0 += p.lam * scr * cu(xr)
    y = ws.apply_elimination(torch.empty_like(y0), y0, cu(xr), C)
    assert relerr(y.cpu().numpy(), Sd @ xr) < 1e-12
    x, res = pcg.solve_refined(S, S0, scr, p.lam, C, g, ws, tol=1e-13)
    assert res.converged and res.rel_residual <= 1e-13, res
    err = relerr(x.cpu().numpy(), x_star)
    xp, pres = pcg.solve(S, g, tol=1e-12)
    err_plain = relerr(xp.cpu().numpy(), x_star)
    print(f"{name}: refined error {err:.2e} ({res.corrections} corrections, {res.iterations} PCG iterations); "
          f"PCG on the FP32 S alone {err_plain:.2e}")
    assert err <= 1e-10
    assert err_plain > 100 * err
