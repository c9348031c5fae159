"""Parity at the benchmarked sizes: the full sparse_1000x200k, qr_500x100k and pcg_10000x1M scenes on the device
against the oracle (the reference's algorithm restated on the CPU, threaded over every host core).

Schur: FP64 S and g_S within 1e-12 relative of the oracle (test/schur.jl:223-237 and :399-400 bound the reference's
own solutions and its threaded sums at 1e-12 / 1e-13); the mixed form (FP32 storage and accumulation, FP64 inverse,
z and gradient) against the FP64 oracle on the same FP32-rounded inputs, S within 1e-4 and g_S within 1e-6
(test/precision.jl:21,44,107 accepts Float32 results at sqrt(eps(Float32)) ~ 3e-4). Every phase-2 schedule the plan
can be set to is checked at full size on the 200k-point scene; the 1M-point scene runs the default schedule.
QR: FP64 factored tables, residual, J~'J~ and J~'r~ within 1e-11; the mixed form's unique quantities (J~'J~, J~'r~)
within 1e-6 (the sign of a near-zero Householder pivot may differ from FP64's, so the tables themselves are another
valid factorisation).
"""
import os

import numpy as np
import pytest
import torch

import oracle as orc

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
CORES = os.cpu_count() or 1


def cu(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(DEV)


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


_SCENES = {}


def hessian_scene(bls, name):
    """The full scene, its oracle layout and the oracle's FP64 reduction of the FP64 inputs and of the FP32-rounded
    inputs (computed once per scene and shared by the tests)."""
    if name in _SCENES:
        return _SCENES[name]
    spec = bls.scenes.workload(name)
    p = bls.scenes.hessian_problem(spec)
    bs, el, ptr, idx = bls.scenes.Scene(spec).description()
    ost = orc.Structure.from_description(bs, (ptr, idx), el, nchunks=CORES, min_work=4096)
    opat = orc.Pattern(ost)
    work = orc.Work(ost, CORES, False)
    ref = {}
    for key, cast in (("f64", np.float64), ("f32", np.float32)):
        E, Cd, R = (a.astype(cast).astype(np.float64) for a in (p.E, p.C, p.R))
        oS, og = np.zeros(opat.nnz), np.zeros(ost.nr)
        orc.reset_schur_sparse(ost, opat, oS, R, p.scaling_r, p.lam)
        ok, fb = orc.reduce_schur_sparse(ost, opat, work, oS, og, p.b_r, p.b_e, p.scaling_e, p.lam, E, Cd, nthreads=CORES)
        assert ok, fb
        ref[key] = (oS, og)
    _SCENES[name] = (p, ref)
    return _SCENES[name]


def device_reduce(bls, p, dtype, kernel=None):
    st, pat = p.structure, p.pattern
    ws = bls.SchurReductionWorkspace(st, pat)
    if kernel is not None:
        ws.set_kernel(kernel)
    S = torch.zeros(pat.nnz, dtype=dtype, device=DEV)
    g = torch.zeros(st.nr, dtype=torch.float64, device=DEV)
    bls.reset_schur_sparse(S, cu(p.R, dtype), None, None, cu(p.scaling_r), p.lam, ws)
    ok = bls.reduce_schur_sparse(S, g, cu(p.b_r), cu(p.b_e), cu(p.scaling_e), p.lam, st, cu(p.E, dtype), cu(p.C, dtype),
                                 None, None, None, None, ws)
    assert ok, ws.failed_block
    return S.double().cpu().numpy(), g.cpu().numpy(), ws


@pytest.mark.parametrize("kernel", [None, "stage", "pairs", "columns", "lanes", "tiles", "points"])
def test_sparse_1000x200k_full(bls, kernel):
    p, ref = hessian_scene(bls, "sparse_1000x200k")
    S, g, _ = device_reduce(bls, p, torch.float64, kernel)
    assert relerr(S, ref["f64"][0]) < 1e-12
    assert relerr(g, ref["f64"][1]) < 1e-12
    S, g, _ = device_reduce(bls, p, torch.float32, kernel)
    assert relerr(S, ref["f32"][0]) < 1e-4
    assert relerr(g, ref["f32"][1]) < 1e-6


def test_pcg_10000x1M_full(bls):
    """The 1M-point scene (10,000 cameras, 7.66M observations, camera column scales over four decades): the default
    schedule's FP64 and mixed S and g_S against the oracle at full size."""
    p, ref = hessian_scene(bls, "pcg_10000x1M")
    S, g, _ = device_reduce(bls, p, torch.float64)
    assert relerr(S, ref["f64"][0]) < 1e-12
    assert relerr(g, ref["f64"][1]) < 1e-12
    S, g, _ = device_reduce(bls, p, torch.float32)
    e_s, e_g = relerr(S, ref["f32"][0]), relerr(g, ref["f32"][1])
    print(f"pcg_10000x1M mixed: S {e_s:.2e}, g_S {e_g:.2e}")
    assert e_s < 1e-4
    assert e_g < 1e-6
    del _SCENES["pcg_10000x1M"]


def test_qr_500x100k_full(bls):
    spec = bls.scenes.workload("qr_500x100k")
    p = bls.scenes.jacobian_problem(spec)
    j = p.structure
    bs, el, ptr, idx = bls.scenes.Scene(spec).description()
    o = orc.QRStructure.from_description(bs, (ptr, idx), np.full(len(ptr) - 1, 2), el, nchunks=CORES)
    pairs = bls.free_block_pairs(j)
    pat = bls.build_schur_pattern(j.schur, pairs)
    opat = orc.Pattern(o.st, pairs)
    nr = j.schur.nr
    for dtype in (torch.float64, torch.float32):
        npdt = np.float64 if dtype == torch.float64 else np.float32
        Rw = p.Rw.astype(npdt)
        ws = bls.QRReductionWorkspace(j, pat, dtype)
        J = bls.SchurBlockJacobian(j, dtype, data=cu(Rw), r=cu(p.Rr))
        assert bls.reduce_qr(ws, J, cu(p.scaling_e), p.lam)
        Ss = torch.zeros(pat.nnz, dtype=dtype, device=DEV)
        gs = torch.zeros(nr, dtype=torch.float64, device=DEV)
        bls.reduced_normal_sparse(Ss, gs, ws, pat)
        F, Fr = np.zeros(o.raw_length), np.zeros(o.residual_length)
        ok, fb = orc.reduce_qr(o, F, Fr, Rw.astype(np.float64), p.Rr, p.scaling_e, p.lam, nthreads=CORES)
        assert ok, fb
        oS, og = np.zeros(opat.nnz), np.zeros(nr)
        orc.reduced_normal_sparse(o, opat, oS, og, F, Fr)
        if dtype == torch.float64:
            assert relerr(ws.factored.double().cpu().numpy(), F) < 1e-11
            assert relerr(ws.fres.cpu().numpy(), Fr) < 1e-11
            tol = 1e-11
        else:
            tol = 1e-6
        e_s, e_g = relerr(Ss.double().cpu().numpy(), oS), relerr(gs.cpu().numpy(), og)
        print(f"qr_500x100k {dtype}: J~'J~ {e_s:.2e}, J~'r~ {e_g:.2e}")
        assert e_s < tol and e_g < tol
