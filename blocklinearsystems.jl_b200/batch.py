"""Many independent elimination problems of uneven sizes as one device reduction (no reference counterpart: the
reference reduces one system per call; here a batch is the disjoint union of the problems' layouts).

BatchedReduction(problems) concatenates the problems' SchurStructure / build_schur_pattern layouts with offsets (block
indices, coupling and point-block offsets, S positions, the r -> s map), so one plan, one reset and one reduction cover
every problem: the union's S is block diagonal by problem, and each kernel launch spans the whole batch. Each
problem's damping lambda_p is folded into its scalings (lambda_p * scaling, formed in FP64 exactly as the kernels form
lambda * scaling; the batch runs with lambda = 1), so every problem's result is the one its own call would give.
Each problem fails on its own (problem_status): a singular point in problem p leaves p's S reset and its g_S as it was,
and the other problems are reduced, as separate reference calls would. autotune() times the phase-2 schedules that
keep that (the block-column owned schedule with staged point operands at several unit sizes, the block-owned pair
lists) and keeps the fastest; capture() records reset + reduce of the batch as one CUDA graph that step() replays.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .reduction import SchurReductionWorkspace, reduce_schur_sparse, reset_reduce_schur_sparse_host, reset_schur_sparse


@dataclass
class UnionLayout:
    """The fields of SchurStructure and SchurPattern that a device plan reads, for the disjoint union of problems."""
    nrblocks: int
    neblocks: int
    nr: int
    ne: int
    E_length: int
    C_length: int
    r_dims: np.ndarray
    e_dims: np.ndarray
    eliminated_ptr: np.ndarray
    entry_retained: np.ndarray
    coffsets: np.ndarray
    eoffsets: np.ndarray
    block_colptr: np.ndarray
    block_rowval: np.ndarray
    block_row_offsets: np.ndarray
    col_heights: np.ndarray
    S_colptr: np.ndarray
    S_rowval: np.ndarray
    diag_inds: np.ndarray
    R_length: int
    r_to_s_map: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.S_colptr[-1])


def union_layout(problems) -> tuple[UnionLayout, dict]:
    """The union layout of HessianProblems (scenes.hessian_problem, sparse) and each problem's offsets."""
    from .layout import build_r_to_s_map
    cat = lambda xs: np.concatenate(xs).astype(np.int64)
    off = dict(rb=[0], eb=[0], nr=[0], ne=[0], E=[0], C=[0], coup=[0], blk=[0], nnz=[0], R=[0])
    parts = {k: [] for k in ("r_dims", "e_dims", "eptr", "eret", "coff", "eoff", "bcol", "brow", "broff", "colh", "Scol", "Srow", "diag", "rts")}
    for i, p in enumerate(problems):
        st, pat = p.structure, p.pattern
        o = {k: v[-1] for k, v in off.items()}
        parts["r_dims"].append(st.r_dims)
        parts["e_dims"].append(st.e_dims)
        parts["eptr"].append((st.eliminated_ptr if i == 0 else st.eliminated_ptr[1:]) + o["coup"])
        parts["eret"].append(st.entry_retained + o["rb"])
        parts["coff"].append(st.coffsets + o["C"])
        parts["eoff"].append(st.eoffsets + o["E"])
        parts["bcol"].append((pat.block_colptr if i == 0 else pat.block_colptr[1:]) + o["blk"])
        parts["brow"].append(pat.block_rowval + o["rb"])
        parts["broff"].append(pat.block_row_offsets)
        parts["colh"].append(pat.col_heights)
        parts["Scol"].append((pat.S_colptr if i == 0 else pat.S_colptr[1:]) + o["nnz"])
        parts["Srow"].append(pat.S_rowval + o["nr"])
        parts["diag"].append(pat.diag_inds + o["nnz"])
        m = build_r_to_s_map(st, pat)
        parts["rts"].append(np.where(m >= 0, m + o["nnz"], -1))
        off["rb"].append(o["rb"] + st.nrblocks)
        off["eb"].append(o["eb"] + st.neblocks)
        off["nr"].append(o["nr"] + st.nr)
        off["ne"].append(o["ne"] + st.ne)
        off["E"].append(o["E"] + st.E_length)
        off["C"].append(o["C"] + st.C_length)
        off["coup"].append(o["coup"] + len(st.entry_retained))
        off["blk"].append(o["blk"] + len(pat.block_rowval))
        off["nnz"].append(o["nnz"] + pat.nnz)
        off["R"].append(o["R"] + pat.R_length)
    U = UnionLayout(nrblocks=off["rb"][-1], neblocks=off["eb"][-1], nr=off["nr"][-1], ne=off["ne"][-1], E_length=off["E"][-1],
                    C_length=off["C"][-1], r_dims=cat(parts["r_dims"]), e_dims=cat(parts["e_dims"]), eliminated_ptr=cat(parts["eptr"]),
                    entry_retained=cat(parts["eret"]), coffsets=cat(parts["coff"]), eoffsets=cat(parts["eoff"]),
                    block_colptr=cat(parts["bcol"]), block_rowval=cat(parts["brow"]), block_row_offsets=cat(parts["broff"]),
                    col_heights=cat(parts["colh"]), S_colptr=cat(parts["Scol"]), S_rowval=cat(parts["Srow"]), diag_inds=cat(parts["diag"]),
                    R_length=off["R"][-1], r_to_s_map=cat(parts["rts"]))
    return U, {k: np.asarray(v, np.int64) for k, v in off.items()}


class BatchedReduction:
    """reset_schur_sparse + reduce_schur_sparse of every problem of a batch in one plan (mixed form with float32, FP64
    with float64 storage)."""

    def __init__(self, problems, dtype=torch.float32, *, device: int = 0):
        self.problems = problems
        self.dtype = dtype
        self.U, self.off = union_layout(problems)
        U = self.U
        self.ws = SchurReductionWorkspace(U, U, U.r_to_s_map, device=device)
        # each problem fails on its own, as its own reduce_schur_sparse! call would
        from . import _lib
        from ._lib import check, ptr64
        offs = [np.ascontiguousarray(self.off[k], np.int64) for k in ("eb", "rb", "nr", "nnz")]
        check(_lib.gpu().bls_schur_plan_set_problems(self.ws._h, len(problems), *[ptr64(a) for a in offs]))
        dev = torch.device("cuda", device)
        f = lambda xs, t=dtype: torch.from_numpy(np.ascontiguousarray(np.concatenate(xs))).to(device=dev, dtype=t)
        self.E = f([p.E for p in problems])
        self.C = f([p.C for p in problems])
        self.R = f([p.R for p in problems])
        self.b_r = f([p.b_r for p in problems], torch.float64)
        self.b_e = f([p.b_e for p in problems], torch.float64)
        # each problem's lambda folded into its scalings; the batch runs with lambda = 1
        self.sc_r = f([p.lam * p.scaling_r for p in problems], torch.float64)
        self.sc_e = f([p.lam * p.scaling_e for p in problems], torch.float64)
        self.S = torch.zeros(U.nnz, dtype=dtype, device=dev)
        self.g = torch.zeros(U.nr, dtype=torch.float64, device=dev)
        self.nobs = int(sum(p.nobs for p in problems))
        self.graph = None
        self.schedule = "pairs"
        self.stage_unit = 16

    def run(self, sync: bool = True) -> bool:
        reset_schur_sparse(self.S, self.R, None, None, self.sc_r, 1.0, self.ws)
        return reduce_schur_sparse(self.S, self.g, self.b_r, self.b_e, self.sc_e, 1.0, self.U, self.E, self.C, None, None, None, None,
                                   self.ws, sync=sync)

    STAGE_UNITS = (8, 16, 24, 32)

    def autotune(self, reps: int = 5) -> dict:
        """Time the phase-2 schedules that keep per-problem failure on the batch, after a warm-up run each, and keep
        the fastest: the block-column owned schedule with staged point operands at each unit size of STAGE_UNITS
        (pairs per thread between two writes to the column tile; keys "stage/8", ...) and the block-owned pair lists
        ("pairs"). The schedule is left at the winner (stage_unit holds its unit size)."""
        times = {}

        def timed(key):
            self.run()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                self.run(sync=False)
            b.record()
            torch.cuda.synchronize()
            times[key] = a.elapsed_time(b) / reps

        self.ws.set_kernel("stage")
        for u in self.STAGE_UNITS:
            self.ws.set_stage_unit(u)
            timed(f"stage/{u}")
        self.ws.set_kernel("pairs")
        timed("pairs")
        best = min(times, key=times.get)
        self.schedule = best.split("/")[0]
        if self.schedule == "stage":
            self.stage_unit = int(best.split("/")[1])
            self.ws.set_stage_unit(self.stage_unit)
        self.ws.set_kernel(self.schedule)
        self.graph = None
        return times

    def capture(self) -> None:
        """Record reset + reduce of the whole batch as one CUDA graph (replayed by step())."""
        self.run()   # first run outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.run(sync=False)
        torch.cuda.current_stream().wait_stream(s)
        self.graph = g

    def step(self) -> None:
        """One batch reduction: the captured graph when there is one, else the launches."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self.run(sync=False)

    def run_host(self, S_h: torch.Tensor, g_h: torch.Tensor, host: dict) -> bool:
        """reset + reduce of the whole batch from host buffers (`host`: E, C, R, b_r, b_e, sc_r, sc_e laid out as this
        batch's device inputs, with each lambda folded into the scalings), S and g_S copied back into S_h and g_h. One
        call: the library copies the inputs stage by stage while the earlier stages are reduced (page-locked buffers)."""
        return reset_reduce_schur_sparse_host(S_h, g_h, host["R"], host["sc_r"], 1.0, host["b_r"], host["b_e"], host["sc_e"], self.U,
                                              host["E"], host["C"], self.ws)

    def problem_status(self) -> np.ndarray:
        """Per problem of the last batch reduction (synchronises): 0, or the problem's lowest failing eliminated block
        (1-based, local to the problem), as that problem's own reduce_schur_sparse! call reports it. A failing problem
        keeps its reset S and its g_S; the other problems are reduced."""
        from . import _lib
        from ._lib import ptr64
        out = np.zeros(len(self.problems), np.int64)
        rc = _lib.gpu().bls_schur_plan_problem_status(self.ws._h, ptr64(out))
        if rc < 0:
            _lib.check(rc)
        return out

    def ok(self) -> bool:
        """Verdict of the last batch reduction (synchronises): True when the arguments were valid and no problem's
        eliminated block failed (see problem_status for the problems that did)."""
        return self.ws.query_status() and not self.problem_status().any()

    def problem_S(self, i: int) -> torch.Tensor:
        return self.S[int(self.off["nnz"][i]):int(self.off["nnz"][i + 1])]

    def problem_g(self, i: int) -> torch.Tensor:
        return self.g[int(self.off["nr"][i]):int(self.off["nr"][i + 1])]
