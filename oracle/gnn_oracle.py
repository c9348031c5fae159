"""FP64 numpy restatement of the learned block preconditioner (test infrastructure only: tests/ use it as the checker
of the device kernels). There is no reference counterpart for the network: its parity is unpinned, and this oracle's
own gradient is pinned by central finite differences (tests/test_gnn_oracle.py).

Definitions (the same as the device code): L_b = chol(S_bb); E_bc = L_b^-1 S_bc L_c^-T for every off-diagonal block of
the pattern; edge weight a_bc = ||E_bc||_F; node features f_b = [log1p(e_b,0..5), log1p(sum e_b), log1p(deg_b)/4] with
e_b,i the row energies; mean aggregation m_b = sum_c a_bc h_c / sum_c a_bc; h0 = relu(W_in f + b_in),
h_l = relu(W_s h_(l-1) + W_m m_(l-1) + b), t = W_out h3 + b_out; G_b = I + lower(t_b); M = G S^ G' with
S^ = L^-1 S L^-T; over probes z, loss = Z N2 / N1^2 with N1 = sum z'Mz, N2 = sum |Mz|^2, Z = sum |z|^2 (an estimate
of n sum(lambda^2) / (sum lambda)^2 over M's spectrum: 1 when it is a single point, and blind to a uniform scaling of
the preconditioner, as CG is); preconditioner block B_b = L_b^-T G_b' G_b L_b^-1.
"""
from __future__ import annotations

import numpy as np

F, H, T, NL = 8, 64, 21, 3
LOWER = [(i, j) for i in range(6) for j in range(i + 1)]   # row-major lower triangle order of t


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0

    def take(k, shape):
        nonlocal o
        a = p[o:o + k].reshape(shape)
        o += k
        return a
    W_in, b_in = take(H * F, (H, F)), take(H, (H,))
    layers = []
    for _ in range(NL):
        layers.append((take(H * H, (H, H)), take(H * H, (H, H)), take(H, (H,))))
    W_out, b_out = take(T * H, (T, H)), take(T, (T,))
    assert o == len(p)
    return W_in, b_in, layers, W_out, b_out


def pack(W_in, b_in, layers, W_out, b_out):
    parts = [W_in.ravel(), b_in]
    for Ws, Wm, b in layers:
        parts += [Ws.ravel(), Wm.ravel(), b]
    parts += [W_out.ravel(), b_out]
    return np.concatenate(parts)


def graph(A, edges):
    """A: the dense symmetric reduced matrix (6n x 6n); edges: (b, c) pairs, b < c, of the off-diagonal pattern blocks.
    Returns (L blocks [n,6,6], edge weights [E], features [n,8], neighbour lists [(c, edge)] per node)."""
    n = A.shape[0] // 6
    L = np.stack([np.linalg.cholesky(A[6 * b:6 * b + 6, 6 * b:6 * b + 6]) for b in range(n)])
    energy = np.zeros((n, 6))
    enorm = np.zeros(len(edges))
    nb = [[] for _ in range(n)]
    for e, (b, c) in enumerate(edges):
        X = np.linalg.solve(L[b], A[6 * b:6 * b + 6, 6 * c:6 * c + 6])
        E = np.linalg.solve(L[c], X.T).T
        enorm[e] = np.sqrt((E ** 2).sum())
        energy[b] += (E ** 2).sum(axis=1)
        energy[c] += (E ** 2).sum(axis=0)
        nb[b].append((c, e))
        nb[c].append((b, e))
    deg = np.array([len(x) for x in nb], np.float64)
    feat = np.concatenate([np.log1p(energy), np.log1p(energy.sum(axis=1))[:, None], (np.log1p(deg) * 0.25)[:, None]], axis=1)
    return L, enorm, feat, nb


def agg_matrix(n, enorm, nb):
    """The aggregation as a dense n x n matrix M (m = M h)."""
    M = np.zeros((n, n))
    for b in range(n):
        a = sum(enorm[e] for _, e in nb[b])
        if a > 0:
            for c, e in nb[b]:
                M[b, c] += enorm[e] / a
    return M


def forward(p, feat, M):
    W_in, b_in, layers, W_out, b_out = unpack(p)
    pre0 = feat @ W_in.T + b_in
    h = [np.maximum(pre0, 0)]
    m, pre = [], [pre0]
    for Ws, Wm, b in layers:
        mi = M @ h[-1]
        z = h[-1] @ Ws.T + mi @ Wm.T + b
        m.append(mi)
        pre.append(z)
        h.append(np.maximum(z, 0))
    t = h[-1] @ W_out.T + b_out
    return t, dict(h=h, m=m, pre=pre)


def G_blocks(t):
    n = t.shape[0]
    G = np.tile(np.eye(6), (n, 1, 1))
    for q, (i, j) in enumerate(LOWER):
        G[:, i, j] += t[:, q]
    return G


def block_apply(Bs, x, transpose=False):
    n = Bs.shape[0]
    xb = x.reshape(n, 6)
    return np.einsum("bji,bj->bi" if transpose else "bij,bj->bi", Bs, xb).reshape(-1)


def loss_and_dt(t, A, L, probes):
    """The loss Z N2 / N1^2 (N1 = sum z'Mz, N2 = sum |Mz|^2, Z = sum |z|^2, M = G S^ G') and its gradient in t:
    dL/dG = (Z / N1^2) (2 sum (y w' + z s') - 4 (N2 / N1) sum z w') with w = S^ G' z, y = G w, s = S^ G' y."""
    n = t.shape[0]
    G = G_blocks(t)
    Linv = np.linalg.inv(L)
    def Shat(x):
        return block_apply(Linv, A @ block_apply(Linv, x, transpose=True))
    N1 = N2 = Z = 0.0
    dA = np.zeros((n, 6, 6))
    dB = np.zeros((n, 6, 6))
    outer = lambda a, b: np.einsum("bi,bj->bij", a.reshape(n, 6), b.reshape(n, 6))
    for z in probes:
        w = Shat(block_apply(G, z, transpose=True))
        y = block_apply(G, w)
        s = Shat(block_apply(G, y, transpose=True))
        Z += z @ z
        N1 += z @ y
        N2 += y @ y
        dA += outer(y, w) + outer(z, s)
        dB += outer(z, w)
    loss = Z * N2 / N1 ** 2
    dG = (Z / N1 ** 2) * (2 * dA - 4 * (N2 / N1) * dB)
    dt = np.stack([dG[:, i, j] for (i, j) in LOWER], axis=1)
    return loss, dt


def backward(p, feat, M, cache, dt):
    W_in, b_in, layers, W_out, b_out = unpack(p)
    h, m, pre = cache["h"], cache["m"], cache["pre"]
    gW_out = dt.T @ h[-1]
    gb_out = dt.sum(axis=0)
    dh = dt @ W_out
    glayers = []
    for l in range(NL - 1, -1, -1):
        Ws, Wm, b = layers[l]
        dpre = dh * (pre[l + 1] > 0)
        glayers.append((dpre.T @ h[l], dpre.T @ m[l], dpre.sum(axis=0)))
        dh = dpre @ Ws + M.T @ (dpre @ Wm)
    glayers.reverse()
    dpre0 = dh * (pre[0] > 0)
    return pack(dpre0.T @ feat, dpre0.sum(axis=0), glayers, gW_out, gb_out)


def loss_grad(p, A, edges, probes):
    L, enorm, feat, nb = graph(A, edges)
    M = agg_matrix(A.shape[0] // 6, enorm, nb)
    t, cache = forward(p, feat, M)
    loss, dt = loss_and_dt(t, A, L, probes)
    return loss, backward(p, feat, M, cache, dt)


def preconditioner_blocks(p, A, edges):
    L, enorm, feat, nb = graph(A, edges)
    M = agg_matrix(A.shape[0] // 6, enorm, nb)
    t, _ = forward(p, feat, M)
    G = G_blocks(t)
    C = G @ np.linalg.inv(L)
    return np.einsum("bki,bkj->bij", C, C)
