"""Batched reduction of uneven problems (the batched workload's distributions, scaled down) through one plan over the
disjoint union of their layouts, against the oracle run problem by problem.

Each problem's S and g_S slice of the batch within 1e-12 relative of its own FP64 oracle reduction (with its own
lambda), and within 1e-4 in the mixed form (on the same FP32-rounded inputs); the captured CUDA graph reproduces the
direct launches; the autotuner's choice is the faster schedule; a failing point block fails its own problem only.
"""
import numpy as np
import pytest
import torch

import oracle as orc

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def problems(bls):
    ps = []
    for i in range(10):
        spec = bls.scenes.workload("batched_256", i)
        spec = bls.scenes.scaled_down(spec, ncams=min(spec.ncams, 12 + 7 * i), npoints=min(spec.npoints, 400 + 150 * i))
        ps.append(bls.scenes.hessian_problem(spec))
    return ps


def oracle_reduce(bls, p, dtype):
    sc = bls.scenes.Scene(p.spec)
    bs, el, ptr, idx = sc.description()
    ost = orc.Structure.from_description(bs, (ptr, idx), el)
    opat = orc.Pattern(ost)
    cast = (lambda a: a.astype(np.float32).astype(np.float64)) if dtype == torch.float32 else (lambda a: a)
    S, g = np.zeros(opat.nnz), np.zeros(ost.nr)
    orc.reset_schur_sparse(ost, opat, S, cast(p.R), p.scaling_r, p.lam)
    ok, fb = orc.reduce_schur_sparse(ost, opat, orc.Work(ost, 1), S, g, p.b_r, p.b_e, p.scaling_e, p.lam, cast(p.E), cast(p.C))
    assert ok
    return S, g


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_batch_matches_each_problem(bls, problems, dtype):
    B = bls.batch.BatchedReduction(problems, dtype)
    assert B.run()
    tol = 1e-12 if dtype == torch.float64 else 1e-4
    for i, p in enumerate(problems):
        oS, og = oracle_reduce(bls, p, dtype)
        assert relerr(B.problem_S(i).double().cpu().numpy(), oS) <= tol, i
        assert relerr(B.problem_g(i).cpu().numpy(), og) <= tol, i


def _corrupt_problem4(B):
    """A singular point block in problem 4 (its 6th point: E = 0 and no damping)."""
    e_off = int(B.off["eb"][4])
    eo = int(B.U.eoffsets[e_off + 5])
    B.E[eo:eo + 9] = 0.0
    B.sc_e[int(B.off["ne"][4]) + 15:int(B.off["ne"][4]) + 18] = 0.0


@pytest.mark.parametrize("schedule", ["stage", "pairs"])
def test_graph_autotune_and_per_problem_failure(bls, problems, schedule):
    """The autotuner times the schedules that keep per-problem failure and keeps the faster; the captured graph
    reproduces the launches; a singular point in problem 4 fails problem 4 alone, as its own reference call would
    (src/schur_reduction.jl:233-257): its S stays the reset system and its g_S untouched, its 6th block is reported
    (1-based, local to the problem), and every other problem is still reduced."""
    B = bls.batch.BatchedReduction(problems, torch.float32)
    times = B.autotune(reps=3)
    assert set(times) == {f"stage/{u}" for u in B.STAGE_UNITS} | {"pairs"} and 24 in B.STAGE_UNITS
    best = min(times, key=times.get)
    assert B.schedule == best.split("/")[0] and (B.schedule == "pairs" or B.stage_unit == int(best.split("/")[1]))
    B.ws.set_kernel(schedule)
    assert B.run()
    S0, g0 = B.S.clone(), B.g.clone()
    B.capture()
    B.S.zero_()
    B.g.zero_()
    B.step()
    assert B.ok() and not B.problem_status().any()
    assert relerr(B.S.double().cpu().numpy(), S0.double().cpu().numpy()) <= 1e-6
    assert relerr(B.g.cpu().numpy(), g0.cpu().numpy()) <= 1e-12
    # the reset system of the batch (what a failing problem keeps)
    S_reset = torch.zeros_like(B.S)
    bls.reset_schur_sparse(S_reset, B.R, None, None, B.sc_r, 1.0, B.ws)
    _corrupt_problem4(B)
    B.g.fill_(7.0)
    B.step()
    st = B.problem_status()
    assert not B.ok()
    assert st[4] == 6 and np.count_nonzero(st) == 1, st
    a, b = int(B.off["nnz"][4]), int(B.off["nnz"][5])
    assert torch.equal(B.S[a:b], S_reset[a:b])
    assert torch.all(B.problem_g(4) == 7.0)
    for i in range(len(problems)):
        if i == 4:
            continue
        a, b = int(B.off["nnz"][i]), int(B.off["nnz"][i + 1])
        assert relerr(B.S[a:b].double().cpu().numpy(), S0[a:b].double().cpu().numpy()) <= 1e-6, i
        assert relerr(B.problem_g(i).cpu().numpy(), g0[int(B.off["nr"][i]):int(B.off["nr"][i + 1])].cpu().numpy()) <= 1e-12, i


def test_host_buffer_batch_matches_device_run(bls, problems):
    """The whole batch from page-locked host buffers in one call (stage-by-stage copies) gives the device run's S and
    g; with problem 4 failing, only the problems that succeeded are copied back (problem 4's host S and g_S keep the
    caller's values) and the failure is reported in problem 4 alone."""
    B = bls.batch.BatchedReduction(problems, torch.float32)
    assert B.run()
    host = {k: getattr(B, k).cpu().pin_memory() for k in ("E", "C", "R", "b_r", "b_e", "sc_r", "sc_e")}
    hS = torch.empty_like(B.S, device="cpu").pin_memory()
    hg = torch.empty_like(B.g, device="cpu").pin_memory()
    assert B.run_host(hS, hg, host)
    assert relerr(hS.double().numpy(), B.S.double().cpu().numpy()) <= 1e-6
    assert relerr(hg.numpy(), B.g.cpu().numpy()) <= 1e-12
    S_ok, g_ok = hS.clone(), hg.clone()
    _corrupt_problem4(B)
    host["E"].copy_(B.E.cpu())
    host["sc_e"].copy_(B.sc_e.cpu())
    hS.fill_(3.0)
    hg.fill_(5.0)
    assert B.run_host(hS, hg, host)            # the call succeeds; the verdicts are per problem
    st = B.problem_status()
    assert st[4] == 6 and np.count_nonzero(st) == 1, st
    a, b = int(B.off["nnz"][4]), int(B.off["nnz"][5])
    assert torch.all(hS[a:b] == 3.0) and torch.all(hg[int(B.off["nr"][4]):int(B.off["nr"][5])] == 5.0)
    for i in range(len(problems)):
        if i == 4:
            continue
        a, b = int(B.off["nnz"][i]), int(B.off["nnz"][i + 1])
        assert relerr(hS[a:b].double().numpy(), S_ok[a:b].double().numpy()) <= 1e-6, i
