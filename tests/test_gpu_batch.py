"""Batched reduction of uneven problems (the batched workload's distributions, scaled down) through one plan over the
disjoint union of their layouts, against the oracle run problem by problem.

Each problem's S and g_S slice of the batch within 1e-12 relative of its own FP64 oracle reduction (with its own
lambda), and within 1e-4 in the mixed form (on the same FP32-rounded inputs); the captured CUDA graph reproduces the
direct launches; the autotuner's choice is the faster schedule; a failing point block is reported in its problem's range.
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


def test_graph_autotune_and_failure(bls, problems):
    B = bls.batch.BatchedReduction(problems, torch.float32)
    times = B.autotune(reps=3)
    assert set(times) == {"pairs", "columns", "lanes", "tiles", "points"} and B.schedule == min(times, key=times.get)
    assert B.run()
    S0, g0 = B.S.clone(), B.g.clone()
    B.capture()
    B.S.zero_()
    B.g.zero_()
    B.step()
    assert B.ok()
    assert relerr(B.S.double().cpu().numpy(), S0.double().cpu().numpy()) <= 1e-6
    assert relerr(B.g.cpu().numpy(), g0.cpu().numpy()) <= 1e-12
    # a singular point block in problem 4 (its 6th point): reported in that problem's range, 1-based
    e_off = int(B.off["eb"][4])
    eo = int(B.U.eoffsets[e_off + 5])
    B.E[eo:eo + 9] = 0.0
    B.sc_e[int(B.off["ne"][4]) + 15:int(B.off["ne"][4]) + 18] = 0.0
    B.step()
    assert not B.ok()
    assert B.ws.failed_block == e_off + 6


def test_host_buffer_batch_matches_device_run(bls, problems):
    """The whole batch from page-locked host buffers in one call (stage-by-stage copies) gives the device run's S and g."""
    B = bls.batch.BatchedReduction(problems, torch.float32)
    assert B.run()
    host = {k: getattr(B, k).cpu().pin_memory() for k in ("E", "C", "R", "b_r", "b_e", "sc_r", "sc_e")}
    hS = torch.empty_like(B.S, device="cpu").pin_memory()
    hg = torch.empty_like(B.g, device="cpu").pin_memory()
    assert B.run_host(hS, hg, host)
    assert relerr(hS.double().numpy(), B.S.double().cpu().numpy()) <= 1e-6
    assert relerr(hg.numpy(), B.g.cpu().numpy()) <= 1e-12
