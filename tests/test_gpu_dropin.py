"""The reference's schur_solve! call sequence (src/schur_linear_systems.jl:362-406) through the Julia extension's GPU
methods, mirrored over ctypes in dropin_shim.py with the reference's exact positional signatures:

    reset_schur_sparse!(S.nzval, R.data, r_to_s_map, diag_inds, scaling_r, lambda, ws, s_r, S)
    reduce_schur_sparse!(S, g_S, b_r, b_e, scaling_e, lambda, structure, E_data, C_data,
                         block_colptr, block_rowval, block_row_offsets, col_heights, ws, s_r, s_e) || return NotPositiveDefinite
    (the caller's own sparse factorisation of S on the host)
    backsubstitute!(x_e, x_r, structure, C_data, ws, s_r, s_e)

on host arrays, as the reference's linear system holds them. The solution must equal a dense FP64 solve of the full
damped system: backward error <= 1e-13 and forward error <= 1e-8 (test/schur_problems.jl:20-22 bounds the
reference's at 1e-9 on better-conditioned fixtures), in FP64 and with conditioning scales; a singular point
returns false with the lowest failing block (1-based) and leaves S and g_S untouched; bad damping arguments throw
before anything is written.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

import dropin_shim as shim

pytestmark = pytest.mark.gpu


def _system(bls, ncams=40, npoints=1500, seed=None):
    spec = bls.scenes.scaled_down(bls.scenes.workload("sparse_1000x200k"), ncams, npoints, seed=seed)
    return bls.scenes.hessian_problem(spec)


def _full_dense(p):
    """The damped full system H + lambda diag(scaling) of the problem, dense: R (mapped onto S's pattern, upper blocks
    with full diagonal blocks), the point blocks E and the couplings C."""
    st, pat = p.structure, p.pattern
    nr, ne = st.nr, st.ne
    H = np.zeros((nr + ne, nr + ne))
    Rs = np.zeros(pat.nnz)
    m = p._r_to_s >= 0
    Rs[p._r_to_s[m]] = p.R[m]
    for j in range(nr):
        for q in range(pat.S_colptr[j], pat.S_colptr[j + 1]):
            i = pat.S_rowval[q]
            if i <= j:
                H[i, j] = H[j, i] = Rs[q]
    for e in range(st.neblocks):
        o, b0 = st.eoffsets[e], nr + st.boffsets_e[e]
        H[b0:b0 + 3, b0:b0 + 3] = p.E[o:o + 9].reshape(3, 3, order="F")
        for c in range(st.eliminated_ptr[e], st.eliminated_ptr[e + 1]):
            blk = p.C[st.coffsets[c]:st.coffsets[c] + 18].reshape(3, 6, order="F")
            r0 = st.boffsets_r[st.entry_retained[c]]
            H[b0:b0 + 3, r0:r0 + 6] = blk
            H[r0:r0 + 6, b0:b0 + 3] = blk.T
    H[np.arange(nr), np.arange(nr)] += p.lam * p.scaling_r
    H[nr + np.arange(ne), nr + np.arange(ne)] += p.lam * p.scaling_e
    return H


def _prepare(bls, p):
    p._r_to_s = bls.build_r_to_s_map(p.structure, p.pattern)
    return p


def _schur_solve(bls, p, ws, s_r=None, s_e=None):
    """schur_solve!'s body over the shim, on host arrays (the reference's SparseSchurLinearSystem fields)."""
    st, pat = p.structure, p.pattern
    S_nzval = np.zeros(pat.nnz)
    g_S = np.zeros(st.nr)
    shim.reset_schur_sparse(S_nzval, p.R, p._r_to_s, pat.diag_inds, p.scaling_r, p.lam, ws, s_r, None)
    ok = shim.reduce_schur_sparse(S_nzval, g_S, p.b_r, p.b_e, p.scaling_e, p.lam, st, p.E, p.C, pat.block_colptr, pat.block_rowval,
                                  pat.block_row_offsets, pat.col_heights, ws, s_r, s_e)
    if not ok:
        return None
    # the caller's own factorisation of S (upper triangle stored; CHOLMOD in the reference, scipy here)
    S = sp.csc_matrix((S_nzval, pat.S_rowval, pat.S_colptr), shape=(st.nr, st.nr))
    U = sp.triu(S)
    Sf = (U + sp.triu(U, 1).T).tocsc()
    x_r = spla.spsolve(Sf, g_S)
    x_e = np.zeros(st.ne)
    shim.backsubstitute(x_e, x_r, st, p.C, ws, s_r, s_e)
    return x_r, x_e


@pytest.mark.parametrize("scaled", [False, True], ids=["unit", "conditioned"])
def test_schur_solve_through_the_shim(bls, scaled):
    p = _prepare(bls, _system(bls))
    st = p.structure
    ws = shim.GPUSchurWorkspace(bls, st, p.pattern, p._r_to_s, torch.float64)
    rng = np.random.default_rng(3)
    s_r = np.ldexp(1.0, rng.integers(-3, 4, st.nr)) if scaled else None
    s_e = np.ldexp(1.0, rng.integers(-3, 4, st.ne)) if scaled else None
    x_r, x_e = _schur_solve(bls, p, ws, s_r, s_e)
    H = _full_dense(p)
    b = np.concatenate([p.b_r, p.b_e])
    if scaled:
        # the conditioned system in the scaled variables y (x = s .* y): (s H s) y = s b
        s = np.concatenate([s_r, s_e])
        # damping is formed on the scaled diagonal: lambda scaling s^2, the same as s (H + lambda D) s
        y = np.linalg.solve(s[:, None] * H * s[None, :], s * b)
    else:
        y = np.linalg.solve(H, b)
    x = np.concatenate([x_r, x_e])
    # the point blocks' singular values reach 1e-4 (cond(H) ~ 1e8 with the conditioning scales), so the dense
    # reference itself is accurate to ~1e-8 only: the backward error is the tight check, the forward error the loose one
    A, rhs = (s[:, None] * H * s[None, :], s * b) if scaled else (H, b)
    assert np.linalg.norm(A @ x - rhs) / (np.linalg.norm(A, 2) * np.linalg.norm(x)) < 1e-13
    assert np.linalg.norm(x - y) / np.linalg.norm(y) < 1e-8


def test_shim_failure_and_argument_errors(bls):
    p = _prepare(bls, _system(bls, 30, 800, seed=11))
    st, pat = p.structure, p.pattern
    ws = shim.GPUSchurWorkspace(bls, st, pat, p._r_to_s, torch.float64)
    E = p.E.copy()
    v = np.array([1.0, -2.0, 0.5])
    for e in (6, 13):
        E[9 * e:9 * e + 9] = np.outer(v, v).ravel(order="F")
    S_nzval, g_S = np.full(pat.nnz, 7.0), np.full(st.nr, 9.0)
    shim.reset_schur_sparse(S_nzval, p.R, p._r_to_s, pat.diag_inds, p.scaling_r, p.lam, ws)
    ok = shim.reduce_schur_sparse(S_nzval, g_S, p.b_r, p.b_e, np.zeros_like(p.scaling_e), 0.0, st, E, p.C, pat.block_colptr,
                                  pat.block_rowval, pat.block_row_offsets, pat.col_heights, ws)
    assert not ok and ws.failed_block == 7
    assert np.all(S_nzval == 7.0) and np.all(g_S == 9.0)
    bad = p.scaling_r.copy()
    bad[4] = -1.0
    with pytest.raises(shim.ArgumentError):
        shim.reset_schur_sparse(S_nzval, p.R, p._r_to_s, pat.diag_inds, bad, p.lam, ws)
    with pytest.raises(shim.ArgumentError):
        shim.reduce_schur_sparse(S_nzval, g_S, p.b_r, p.b_e, p.scaling_e, float("nan"), st, p.E, p.C, pat.block_colptr,
                                 pat.block_rowval, pat.block_row_offsets, pat.col_heights, ws)
    assert np.all(S_nzval == 7.0) and np.all(g_S == 9.0)
