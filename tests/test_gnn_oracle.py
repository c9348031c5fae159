"""The learned preconditioner's FP64 oracle, on the CPU: its analytic gradient against central finite differences (the
oracle is unpinned otherwise: the network has no reference counterpart), the untrained network reproducing
block-Jacobi exactly, and symmetric positive definite preconditioner blocks for any parameters.
"""
import numpy as np
import pytest

import gnn_oracle as go


def small_system(rng, n=7):
    """A random SPD block matrix with a ring-plus-chords block pattern of 6x6 blocks."""
    edges = [(b, b + 1) for b in range(n - 1)] + [(0, n - 1), (1, 4), (2, 5)]
    edges = sorted(set((min(b, c), max(b, c)) for b, c in edges))
    A = np.zeros((6 * n, 6 * n))
    for b in range(n):
        X = rng.standard_normal((6, 6))
        A[6 * b:6 * b + 6, 6 * b:6 * b + 6] = X @ X.T + 6 * np.eye(6)
    for b, c in edges:
        B = 0.4 * rng.standard_normal((6, 6))
        A[6 * b:6 * b + 6, 6 * c:6 * c + 6] = B
        A[6 * c:6 * c + 6, 6 * b:6 * b + 6] = B.T
    A += 8 * np.eye(6 * n)   # keep it positive definite
    return A, edges


def random_params(rng, scale=0.3):
    n = go.H * go.F + go.H + go.NL * (2 * go.H * go.H + go.H) + go.T * go.H + go.T
    return scale * rng.standard_normal(n) / np.sqrt(go.H)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    A, edges = small_system(rng)
    p = random_params(rng)
    probes = rng.standard_normal((3, A.shape[0]))
    loss, g = go.loss_grad(p, A, edges, probes)
    idx = rng.choice(len(p), 40, replace=False)
    # include entries of every parameter group
    W_in, b_in, layers, W_out, b_out = go.unpack(np.arange(len(p)))
    idx = np.concatenate([idx, [int(W_in[3, 2]), int(b_in[5]), int(layers[0][0][1, 2]), int(layers[1][1][4, 7]), int(layers[2][2][9]),
                                int(W_out[7, 11]), int(b_out[20])]])
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (go.loss_grad(p + e, A, edges, probes)[0] - go.loss_grad(p - e, A, edges, probes)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g).max()), (i, fd, g[i])


def test_untrained_network_is_block_jacobi():
    rng = np.random.default_rng(1)
    A, edges = small_system(rng)
    p = random_params(rng)
    W_in, b_in, layers, W_out, b_out = go.unpack(p)
    p0 = go.pack(W_in, b_in, layers, np.zeros_like(W_out), np.zeros_like(b_out))
    B = go.preconditioner_blocks(p0, A, edges)
    for b in range(A.shape[0] // 6):
        np.testing.assert_allclose(B[b], np.linalg.inv(A[6 * b:6 * b + 6, 6 * b:6 * b + 6]), rtol=1e-10, atol=1e-12)


def test_blocks_are_spd():
    rng = np.random.default_rng(2)
    A, edges = small_system(rng)
    for s in (0.1, 1.0, 3.0):
        B = go.preconditioner_blocks(random_params(rng, s), A, edges)
        for Bb in B:
            np.testing.assert_allclose(Bb, Bb.T, rtol=1e-12, atol=1e-12)
            assert np.linalg.eigvalsh(Bb).min() > 0
