"""A learned correction to the 6x6 block-Jacobi preconditioner of PCG on the reduced system (no reference counterpart).

LearnedPreconditioner(structure, pattern) wraps the device graph network of csrc/gnn.cu over the camera covisibility
graph (the block pattern of S): 3 message-passing layers of width 64, node features from the block-Jacobi-normalised
couplings, and per block a lower-triangular correction T_b; the preconditioner block is L_b^-T (I+T_b)'(I+T_b) L_b^-1.
It is trained (train_step: the device loss and gradient, then Adam, all in this project's kernels) on reduced systems
that the plain Schur path produces from seeded scenes, and applied through PCGWorkspace.solve(preconditioner=...).
The network changes the iteration count only: PCG still stops on the explicit FP64 residual of S x = g.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import BLS_NOT_PD, ArgumentError, check, dptr, ptr64
from .layout import SchurPattern, SchurStructure
from .pcg import PCGWorkspace
from .reduction import _dev, _dtype_code, context

def param_count() -> int:
    return int(_lib.gpu().bls_gnn_param_count())


def init_params(seed: int = 0, device: int = 0) -> torch.Tensor:
    """He-initialised hidden layers, a zero output layer (so the untrained network is exactly block-Jacobi)."""
    rng = np.random.default_rng(seed)
    F, H, T, L = 8, 64, 21, 3
    p = []
    p.append(rng.standard_normal(H * F) * np.sqrt(2.0 / F))
    p.append(np.zeros(H))
    for _ in range(L):
        p.append(rng.standard_normal(H * H) * np.sqrt(1.0 / H))
        p.append(rng.standard_normal(H * H) * np.sqrt(1.0 / H))
        p.append(np.zeros(H))
    p.append(np.zeros(T * H))
    p.append(np.zeros(T))
    v = np.concatenate(p).astype(np.float32)
    assert len(v) == param_count()
    return torch.from_numpy(v).to(torch.device("cuda", device))


class LearnedPreconditioner:
    """The network's graph for one pattern (built on a PCGWorkspace of the same structure and pattern)."""

    def __init__(self, pcg: PCGWorkspace):
        self.pcg = pcg
        pat = pcg.pattern
        self._keep = [np.ascontiguousarray(a, np.int64) for a in (pat.block_colptr, pat.block_rowval, pat.block_row_offsets,
                                                                  pat.col_heights, pat.S_colptr)]
        h = C.c_void_p()
        check(_lib.gpu().bls_gnn_create(pcg.handle, *[ptr64(a) for a in self._keep], C.byref(h)))
        self._h = h
        self.n = pcg.structure.nrblocks
        self.nedges = int(_lib.gpu().bls_gnn_edge_count(h))
        self._S = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and _lib._gpu is not None:
            _lib.gpu().bls_gnn_destroy(h)
            self._h = None

    @property
    def handle(self):
        context(self.pcg.device)
        return self._h

    def prepare(self, S: torch.Tensor) -> bool:
        """The graph features of S; False if a diagonal block of S is not positive definite."""
        T = _dtype_code(_dev(S, "S.nzval", self.pcg.pattern.nnz))
        fb = C.c_int64(0)
        rc = check(_lib.gpu().bls_gnn_prepare(self.handle, T, dptr(S), C.byref(fb)))
        self._S = S
        return rc != BLS_NOT_PD

    def blocks(self, params: torch.Tensor, *, bf16: bool = True) -> torch.Tensor:
        """Inference: the preconditioner blocks (36 float64 per block) for the prepared S."""
        _dev(params, "params", param_count(), torch.float32)
        out = torch.empty(36 * self.n, dtype=torch.float64, device=params.device)
        check(_lib.gpu().bls_gnn_forward(self.handle, dptr(params), int(bf16), dptr(out)))
        return out

    def outputs(self):
        """(t [n, 21], features [n, 8], edge weights [nedges]) of the last forward / prepare."""
        dev = torch.device("cuda", self.pcg.device)
        t = torch.empty(21 * self.n, dtype=torch.float32, device=dev)
        f = torch.empty(8 * self.n, dtype=torch.float32, device=dev)
        e = torch.empty(max(self.nedges, 1), dtype=torch.float64, device=dev)
        check(_lib.gpu().bls_gnn_outputs(self.handle, dptr(t), dptr(f), dptr(e)))
        return t.view(self.n, 21), f.view(self.n, 8), e[: self.nedges]

    def loss_grad(self, params: torch.Tensor, probes: torch.Tensor, grad: torch.Tensor | None = None):
        """(loss, grad) of the training objective on the prepared S for the given probes [P, nr] (float64)."""
        if self._S is None:
            raise ArgumentError("prepare(S) first")
        nr = self.pcg.structure.nr
        if probes.dim() != 2 or probes.shape[1] != nr:
            raise ArgumentError(f"probes must be [P, {nr}]")
        probes = _dev(probes.contiguous(), "probes", None, torch.float64)
        if grad is None:
            grad = torch.empty(param_count(), dtype=torch.float32, device=params.device)
        loss = C.c_double(0.0)
        check(_lib.gpu().bls_gnn_loss_grad(self.handle, _dtype_code(self._S), dptr(self._S), dptr(params), dptr(probes), probes.shape[0],
                                           C.byref(loss), dptr(grad)))
        return float(loss.value), grad


class Adam:
    """Adam on a flat FP32 parameter vector (the project's own update kernel)."""

    def __init__(self, params: torch.Tensor, lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8):
        self.p = params
        self.m = torch.zeros_like(params)
        self.v = torch.zeros_like(params)
        self.lr, self.b1, self.b2, self.eps = lr, betas[0], betas[1], eps
        self.t = 0

    def step(self, grad: torch.Tensor) -> None:
        self.t += 1
        check(_lib.gpu().bls_adam_step(context(self.p.device.index or 0), dptr(self.p), dptr(grad), dptr(self.m), dptr(self.v), self.p.numel(),
                                       self.lr, self.b1, self.b2, self.eps, self.t))


def train(systems, params: torch.Tensor | None = None, *, steps: int = 200, lr: float = 3e-3, probes: int = 4, seed: int = 0,
          log_every: int = 0):
    """Train on reduced systems [(LearnedPreconditioner prepared on S), ...]: each step one system, `probes` Gaussian
    probe vectors, the device loss and gradient, one Adam step. Returns (params, losses)."""
    if params is None:
        params = init_params(seed, systems[0].pcg.device)
    opt = Adam(params, lr=lr)
    gen = torch.Generator(device=params.device)
    gen.manual_seed(seed)
    losses = []
    grad = torch.empty_like(params)
    for k in range(steps):
        net = systems[k % len(systems)]
        z = torch.randn(probes, net.pcg.structure.nr, dtype=torch.float64, device=params.device, generator=gen)
        loss, _ = net.loss_grad(params, z, grad)
        losses.append(loss)
        opt.step(grad)
        if log_every and k % log_every == 0:
            print(f"step {k}: loss {loss:.5f}")
    return params, losses


def scene_system(ncams: int, npoints: int, seed: int, *, device: int = 0):
    """A reduced system of the 1M-point workload's distributions (pcg_10000x1M's generator on `ncams` cameras and
    `npoints` points: window +-60, k = 2 + Geom(0.15), camera column scales over four decades, lambda 1e-5), produced by
    the plain mixed Schur path on the device, with its PCG workspace and network graph prepared on the FP32 S.
    Returns (LearnedPreconditioner, S, g)."""
    from . import scenes
    from .reduction import SchurReductionWorkspace, reduce_schur_sparse, reset_schur_sparse
    spec = scenes.scaled_down(scenes.workload("pcg_10000x1M"), ncams=ncams, npoints=npoints, seed=seed)
    p = scenes.hessian_problem(spec)
    st, pat = p.structure, p.pattern
    dev = torch.device("cuda", device)
    f = lambda a, t=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=t)
    ws = SchurReductionWorkspace(st, pat, device=device)
    S = torch.zeros(pat.nnz, dtype=torch.float32, device=dev)
    g = torch.zeros(st.nr, dtype=torch.float64, device=dev)
    reset_schur_sparse(S, f(p.R), None, None, f(p.scaling_r, torch.float64), p.lam, ws)
    if not reduce_schur_sparse(S, g, f(p.b_r, torch.float64), f(p.b_e, torch.float64), f(p.scaling_e, torch.float64), p.lam, st, f(p.E),
                               f(p.C), None, None, None, None, ws):
        raise ArgumentError(f"the scene's point block {ws.failed_block} is singular")
    net = LearnedPreconditioner(PCGWorkspace(st, pat, device=device))
    if not net.prepare(S):
        raise ArgumentError("a diagonal block of the reduced system is not positive definite")
    return net, S, g


def pcg_comparison(net: LearnedPreconditioner, S: torch.Tensor, g: torch.Tensor, params: torch.Tensor, *, tol: float = 1e-8) -> dict:
    """Block-Jacobi PCG against PCG with the learned blocks on one prepared system: iterations, device seconds (the
    learned side including its BF16 inference of the blocks) and the final FP64 residuals."""
    out = {}
    for name in ("block_jacobi", "learned"):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        B = net.blocks(params, bf16=True) if name == "learned" else None
        _, res = net.pcg.solve(S, g, tol=tol, preconditioner=B)
        b.record()
        torch.cuda.synchronize()
        out[name] = {"iterations": res.iterations, "seconds": a.elapsed_time(b) / 1e3, "rel_residual": res.rel_residual,
                     "converged": res.converged}
    out["iteration_ratio"] = out["learned"]["iterations"] / max(out["block_jacobi"]["iterations"], 1)
    out["time_ratio"] = out["learned"]["seconds"] / out["block_jacobi"]["seconds"]
    return out


def train_on_scenes(n_scenes: int = 48, ncams=(1000, 5000), points_per_camera: int = 100, *, steps: int = 600, lr: float = 2e-3,
                    probes: int = 4, seed: int = 0, device: int = 0, log_every: int = 0):
    """Train the network on `n_scenes` seeded scenes of the 1M-point workload's family with camera counts drawn
    uniformly from `ncams` (points_per_camera points per camera, as the 1M-point scene has), their reduced systems
    from the plain Schur path (scene_system). Returns (params, losses, systems)."""
    rng = np.random.default_rng(seed)
    systems = []
    for i in range(n_scenes):
        nc = int(rng.integers(ncams[0], ncams[1] + 1))
        net, _, _ = scene_system(nc, points_per_camera * nc, seed=70_000 + 97 * seed + i, device=device)
        systems.append(net)
    params, losses = train(systems, None, steps=steps, lr=lr, probes=probes, seed=seed, log_every=log_every)
    return params, losses, systems
