"""The learned block preconditioner on the device against its FP64 oracle (oracle/gnn_oracle.py, whose gradient is
pinned by finite differences), and what training gains.

Graph features and edge weights (FP64 linear algebra) within 1e-10; the FP32 network's outputs, loss and gradient
within 1e-4 relative (FP32 activations and atomically summed weight gradients); the BF16-in/FP32-accumulate inference
within 3e-2 of the FP64 outputs (BF16 keeps 8 bits). Training on reduced systems that the plain Schur path produced from
seeded scenes, measured on held-out ones: PCG with the learned blocks still stops on the FP64 residual 1e-8 (the network
changes the iteration count, not the solution).
"""
import numpy as np
import pytest
import torch

import gnn_oracle as go
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


def reduced(bls, ncams, npoints, seed):
    spec = bls.scenes.scaled_down(bls.scenes.workload("pcg_10000x1M"), ncams=ncams, npoints=npoints, seed=seed)
    p = bls.scenes.hessian_problem(spec)
    st, pat = p.structure, p.pattern
    ws = bls.SchurReductionWorkspace(st, pat)
    S = torch.zeros(pat.nnz, dtype=torch.float64, device=DEV)
    g = torch.zeros(st.nr, dtype=torch.float64, device=DEV)
    bls.reset_schur_sparse(S, cu(p.R), None, None, cu(p.scaling_r), p.lam, ws)
    assert bls.reduce_schur_sparse(S, g, cu(p.b_r), cu(p.b_e), cu(p.scaling_e), p.lam, st, cu(p.E), cu(p.C), None, None, None, None, ws)
    return st, pat, S, g


def edges_of(pat, n):
    return [(int(pat.block_rowval[k]), c) for c in range(n) for k in range(int(pat.block_colptr[c]), int(pat.block_colptr[c + 1]))
            if int(pat.block_rowval[k]) != c]


def random_params(seed, scale=0.3):
    rng = np.random.default_rng(seed)
    n = go.H * go.F + go.H + go.NL * (2 * go.H * go.H + go.H) + go.T * go.H + go.T
    return (scale * rng.standard_normal(n) / np.sqrt(go.H)).astype(np.float32)


@pytest.fixture(scope="module")
def small(bls):
    st, pat, S, g = reduced(bls, 30, 1500, seed=77)
    A = csc_to_dense_upper(st.nr, pat.S_colptr, pat.S_rowval, S.cpu().numpy())
    pws = bls.PCGWorkspace(st, pat)
    net = bls.gnn.LearnedPreconditioner(pws)
    assert net.prepare(S)
    return st, pat, S, g, A, pws, net, edges_of(pat, st.nrblocks)


def test_features_and_forward(bls, small):
    st, pat, S, g, A, pws, net, edges = small
    p32 = random_params(3)
    B = net.blocks(cu(p32), bf16=False).cpu().numpy().reshape(-1, 6, 6)
    t, f, e = (x.cpu().numpy() for x in net.outputs())
    L, enorm, feat, nb = go.graph(A, edges)
    assert relerr(e, enorm) <= 1e-10
    assert relerr(f, feat) <= 1e-6
    M = go.agg_matrix(st.nrblocks, enorm, nb)
    ot, _ = go.forward(p32.astype(np.float64), feat, M)
    assert relerr(t, ot) <= 1e-4
    oB = go.preconditioner_blocks(p32.astype(np.float64), A, edges)
    assert relerr(B.transpose(0, 2, 1), oB) <= 1e-4      # device blocks are column-major
    # BF16 inference
    net.blocks(cu(p32), bf16=True)
    tb = net.outputs()[0].cpu().numpy()
    assert relerr(tb, ot) <= 3e-2


def test_untrained_is_block_jacobi(bls, small):
    st, pat, S, g, A, pws, net, edges = small
    p0 = bls.gnn.init_params(0).cpu().numpy()
    assert np.all(p0[-(21 * 64 + 21):] == 0)
    B = net.blocks(cu(p0), bf16=True).cpu().numpy().reshape(-1, 6, 6)
    for b in range(st.nrblocks):
        np.testing.assert_allclose(B[b], np.linalg.inv(A[6 * b:6 * b + 6, 6 * b:6 * b + 6]), rtol=1e-9, atol=1e-12)


def test_loss_and_gradient(bls, small):
    st, pat, S, g, A, pws, net, edges = small
    p32 = random_params(5)
    z = np.random.default_rng(9).standard_normal((3, st.nr))
    loss, grad = net.loss_grad(cu(p32), cu(z))
    oloss, ograd = go.loss_grad(p32.astype(np.float64), A, edges, z)
    assert abs(loss - oloss) <= 1e-5 * oloss
    assert relerr(grad.cpu().numpy(), ograd) <= 1e-4


def test_training_gain(bls):
    """Train on reduced systems of seeded scenes (the plain Schur path's output) and measure the gain on held-out ones.

    On this workload family (random N(0, 1) Jacobians, no gauge freedom) the block-Jacobi-preconditioned spectrum is
    already tight (loss Z N2 / N1^2 within a few percent of 1), and a block-diagonal correction has next to nothing to
    gain: the test records the held-out loss and the PCG iteration counts, and checks that the learned blocks keep PCG
    on the same FP64 answer (residual <= 1e-8) at no more than one extra iteration."""
    torch.manual_seed(0)
    train_sys, test_sys = [], []
    for k in range(6):
        nc = 40 + 10 * k
        st, pat, S, g = reduced(bls, nc, 3 * nc, seed=500 + k)
        pws = bls.PCGWorkspace(st, pat)
        net = bls.gnn.LearnedPreconditioner(pws)
        assert net.prepare(S)
        train_sys.append(net)
    for k in range(2):
        st, pat, S, g = reduced(bls, 60, 180, seed=900 + k)
        pws = bls.PCGWorkspace(st, pat)
        net = bls.gnn.LearnedPreconditioner(pws)
        assert net.prepare(S)
        test_sys.append((net, S, g))
    p0 = bls.gnn.init_params(0)
    gen = torch.Generator(device=DEV)
    gen.manual_seed(123)
    probes = [torch.randn(32, n.pcg.structure.nr, dtype=torch.float64, device=DEV, generator=gen) for n, _, _ in test_sys]
    before = [n.loss_grad(p0, z)[0] for (n, _, _), z in zip(test_sys, probes)]
    params, losses = bls.gnn.train(train_sys, p0.clone(), steps=240, lr=2e-3, probes=4, seed=1)
    assert all(np.isfinite(losses))
    after = [n.loss_grad(params, z)[0] for (n, _, _), z in zip(test_sys, probes)]
    for (net, S, g), lb, la in zip(test_sys, before, after):
        net.prepare(S)
        _, bj = net.pcg.solve(S, g, tol=1e-8)
        B = net.blocks(params, bf16=True)
        x, lr = net.pcg.solve(S, g, tol=1e-8, preconditioner=B)
        assert bj.converged and lr.converged and lr.rel_residual <= 1e-8
        assert lr.iterations <= bj.iterations + 1
        print(f"held-out loss {lb:.5f} -> {la:.5f}; PCG iterations block-Jacobi {bj.iterations}, learned {lr.iterations}")


def test_trained_parameters_ratio(bls):
    """The committed parameters (train_gnn.py: 32 seeded scenes of the 1M-point workload's family, 1,000 to 5,000
    cameras) on a held-out 2,000-camera scene of that family: PCG to 1e-8 with the learned blocks against block-Jacobi.
    The measured ratios are printed; a gain is asserted only where one exists (fewer iterations), otherwise the learned
    blocks must keep PCG on the same FP64 answer at no more iterations. On this family the ratio is 1.0 in iterations
    and above 1 in time (the blocks' inference adds to an already tight block-Jacobi solve), against the 0.6 target."""
    from pathlib import Path
    pfile = Path(bls.__file__).resolve().parent / "gnn_pcg_params.npy"
    params = torch.from_numpy(np.load(pfile)).to(DEV)
    net, S, g = bls.gnn.scene_system(2000, 200_000, seed=91_000)
    bls.gnn.pcg_comparison(net, S, g, params)   # warm-up
    cmp_ = bls.gnn.pcg_comparison(net, S, g, params)
    bj, lr = cmp_["block_jacobi"], cmp_["learned"]
    print(f"iterations {bj['iterations']} -> {lr['iterations']} (ratio {cmp_['iteration_ratio']:.3f}); "
          f"seconds {bj['seconds']:.2e} -> {lr['seconds']:.2e} (ratio {cmp_['time_ratio']:.3f}; target 0.6)")
    assert bj["converged"] and lr["converged"] and lr["rel_residual"] <= 1e-8
    if lr["iterations"] < bj["iterations"]:
        assert cmp_["iteration_ratio"] < 1.0
    else:
        assert lr["iterations"] == bj["iterations"]
